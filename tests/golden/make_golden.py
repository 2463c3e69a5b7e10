"""Generate golden outputs of the REFERENCE archive imager on a B200.

The reference's archive/FIPkernels.cu is compiled unmodified for sm_100a by `make -C oracle ref`
(oracle/_ref/libfipk_ref.so, needs the reference sources to build; the built library travels with
the tree). This script runs its FIpipe on the small configuration's FITS-quartet inputs and writes

    tests/golden/fipk_small.npz   image [256][256] float32, input sha256, K chosen by the oracle rule

Usage (GPU):  python -m tests.golden.make_golden [out_dir]
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def quartet():
    """Visreal, Visimag, Bin [N_s][3], Vin [3][3] (float32), N, cell of the small configuration:
    the collapse and FP64 rotation of the synthetic snapshot, cast to float like the reference's
    FITS inputs (archive/SVD_MFS.py writes them from the same quantities)."""
    from oracle import oracle as O
    from svdimager_b200 import synth
    s = synth.make_snapshot("small")
    vr, vi = O.collapse(s)
    vin, q, sv, _ = O.preprocess64(s)
    b = O.expand_coords(q, sv).astype(np.float32)
    return vr, vi, b, vin.astype(np.float32), s.image_size, s.cell_size


def wide_cell_quartet():
    """Samples inside the grid of a 128^2 image at cell 8e-3 rad (40,000 samples, a 5-source sky
    plus noise, Vin an in-plane rotation). At this cell the reference's FP32 degree-based SIN
    reprojection is accurate to ~1e-5 pixel (its rounding error scales as 1/cell), so the whole
    archive path can be compared at 1e-5."""
    rng = np.random.default_rng(11)
    N, cell = 128, 8e-3
    n = 40000
    r = np.zeros((n, 3))
    r[:, :2] = rng.uniform(-58.0, 58.0, (n, 2))
    r[:, 2] = rng.normal(0, 1e-3, n)
    src = np.array([[3.0, 0.1, -0.2], [1.0, -0.3, 0.05], [0.5, 0.25, 0.3], [2.0, 0.0, 0.0],
                    [0.7, -0.1, -0.35]])
    ph = -2 * np.pi * (np.outer(r[:, 0], src[:, 1]) + np.outer(r[:, 1], src[:, 2]))
    vis = (np.exp(1j * ph) @ src[:, 0]) + rng.normal(0, 0.05, n) + 1j * rng.normal(0, 0.05, n)
    th = 0.4
    v = np.array([[np.cos(th), np.sin(th), 0.0], [-np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
    return (vis.real.astype(np.float32), vis.imag.astype(np.float32), r.astype(np.float32),
            v.astype(np.float32), N, cell)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main(out_dir):
    from oracle import oracle as O
    visr, visi, b, v, N, cell = quartet()
    img = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    img2 = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    imgp = O.run_reference_fipipe(visr, visi, b, v, N, cell, precise=True)
    assert np.any(img != 0) and np.any(imgp != 0), "reference FIpipe returned an empty image"
    sc = O.slab_config_fipk(b[:, 2], v.astype(np.float64), N, cell)
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "fipk_small.npz")
    # image: the reference as its own Makefile builds it (--use_fast_math);
    # image_precise: the same source built without --use_fast_math.
    np.savez_compressed(path, image=img, image_rerun=img2, image_precise=imgp,
                        input_sha256=digest(visr, visi, b, v), K=sc.K, N=N, cell=cell)
    print("wrote", path, "K", sc.K, "rerun rel diff",
          float(np.linalg.norm(img - img2) / np.linalg.norm(img)),
          "fast-math vs precise", float(np.linalg.norm(img - imgp) / np.linalg.norm(imgp)))
    visr, visi, b, v, N, cell = wide_cell_quartet()
    img = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    imgp = O.run_reference_fipipe(visr, visi, b, v, N, cell, precise=True)
    assert np.any(img != 0) and np.any(imgp != 0), "reference FIpipe returned an empty image"
    sc = O.slab_config_fipk(b[:, 2], v.astype(np.float64), N, cell)
    path = os.path.join(out_dir, "fipk_widecell.npz")
    np.savez_compressed(path, image=img, image_precise=imgp, input_sha256=digest(visr, visi, b, v),
                        K=sc.K, N=N, cell=cell)
    print("wrote", path, "K", sc.K, "fast-math vs precise",
          float(np.linalg.norm(img - imgp) / np.linalg.norm(imgp)))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
