"""Parity of the B200 path with the oracle (CPU restatement of the reference), with the reference's
own archive imager compiled for sm_100a, and with the FP64 direct DFT. Every call goes through the
C ABI (svdimager_b200.api -> libsvdimager_b200.so).

Tolerances: integer/byte work (flag collapse, tile binning) is bit-exact; images are compared by
relative RMS, sqrt(sum (a-b)^2 / sum b^2), against 1e-5 (FP32 gridding and FFT)."""
import math
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, synth
from tests.conftest import snapshot

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
# Grid planes against the FP64 oracle grid: FP32 ES weights (degree-8 polynomial, <= 1.2e-7) and the tile
# accumulator's fixed-point step (<= 2^-21 of the tile segment's max |v| per contribution).
GRID_TOL = 4e-6


def _scale(cell, G):
    return float(np.float32(cell)) * G


def _slab_config_from_stats(st):
    return O.SlabConfig(st["slab_r3_min"], st["r3_max"], st["max_abs_t3"], st["alpha_max"],
                        st["num_slabs"], st["slab_width"], st["slab_half"], 1.0 / st["slab_half"],
                        st["slab_alpha_max"], st["num_terms"])


@pytest.fixture(scope="module")
def small_run(cuda_device, small_snapshot):
    s = small_snapshot
    e = api.Engine(keep_grid=1)
    img = e.image(s)
    return dict(engine=e, image=img, stats=e.stats(), snap=s)


def test_collapse_bit_exact(small_run):
    s, e = small_run["snap"], small_run["engine"]
    ovr, ovi = O.collapse(s)
    assert np.array_equal(e.buffer(api.BUF_VIS_REAL), ovr)
    assert np.array_equal(e.buffer(api.BUF_VIS_IMAG), ovi)
    both = (s.flag0 != 0) & (s.flag3 != 0)
    assert both.any() and np.all(e.buffer(api.BUF_VIS_REAL)[both] == 0)


def test_rotation_matches_oracle(small_run):
    s, e = small_run["snap"], small_run["engine"]
    vin, q, sv, _ = O.preprocess64(s)
    assert np.array_equal(e.buffer(api.BUF_S), sv)
    assert np.allclose(e.buffer(api.BUF_VIN).reshape(3, 3), vin, atol=1e-12)
    assert np.allclose(e.buffer(api.BUF_Q).reshape(-1, 3), q, rtol=1e-12, atol=1e-9)


def _check_binning(e, st, r, vr, vi, cell, coord_mode=0, edge_mode=0, W=8):
    G, T, T2 = st["grid_size"], st["tile"], st["tile_cols"]
    sc = _slab_config_from_stats(st)
    ntile2 = st["num_keys"] // (sc.num_slabs * ((G + T - 1) // T))
    keys, xq, yq, sa = O.tile_keys(r, _scale(cell, G), G, W, T, edge_mode, sc, coord_mode, records=True,
                                   T2=T2, ntile2=ntile2)
    n_keys = st["num_keys"]
    off = e.buffer(api.BUF_OFFSETS).astype(np.int64)
    kept = keys >= 0
    assert st["num_gridded"] == int(kept.sum())
    assert np.array_equal(np.diff(off), np.bincount(keys[kept], minlength=n_keys))
    rec = e.buffer(api.BUF_RECORDS)
    vin = np.array(st["vin"]).reshape(3, 3)
    inv_det = np.float32(1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0]))
    orec = np.zeros(int(kept.sum()), rec.dtype)
    order = np.argsort(keys[kept], kind="stable")
    orec["xq"] = xq[kept][order]
    orec["yq"] = yq[kept][order]
    orec["vre"] = (vr[kept] * inv_det).astype(np.float32)[order]
    orec["vim"] = (vi[kept] * inv_det).astype(np.float32)[order]
    # records within one key may come in any order: compare per-key sorted
    kk = np.repeat(np.arange(n_keys), np.diff(off))
    a = np.lexsort((rec["vim"], rec["vre"], rec["yq"], rec["xq"], kk))
    b = np.lexsort((orec["vim"], orec["vre"], orec["yq"], orec["xq"], kk))
    assert np.array_equal(rec[a], orec[b])


def test_tile_binning_bit_exact_main(small_run):
    s, e, st = small_run["snap"], small_run["engine"], small_run["stats"]
    r = O.expand_coords(e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S))
    _check_binning(e, st, r, e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG), s.cell_size)


def test_grid_planes_match_oracle(small_run):
    s, e, st = small_run["snap"], small_run["engine"], small_run["stats"]
    G = st["grid_size"]
    r = O.expand_coords(e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S))
    vin = np.array(st["vin"]).reshape(3, 3)
    inv_det = 1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    sc = _slab_config_from_stats(st)
    og = O.grid(r, e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG), _scale(s.cell_size, G), G, sc,
                inv_det)
    grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    assert grid.shape == og.shape
    for p in range(og.shape[0]):
        num = np.linalg.norm(grid[p] - og[p])
        den = np.linalg.norm(og[p])
        if den > 0:
            assert num / den < GRID_TOL, (p, num / den)


def test_main_path_image_matches_oracle(small_run):
    s = small_run["snap"]
    oimg = O.image_sii(s)
    assert small_run["stats"]["num_terms"] == oimg.sc.K == 8
    assert O.rel_rms(small_run["image"], oimg.image) < IMG_TOL


def test_main_path_presplat_and_dft_accuracy(cuda_device, small_snapshot):
    """Rotated-frame image before reprojection against the oracle and against the FP64 direct
    DFT of the same samples (strict inclusion at the grid edge), at every pixel."""
    s = small_snapshot
    with api.Engine(edge_mode=api.EDGE_STRICT, presplat=1) as e:
        R = e.image(s)
    o = O.image_sii(s, edge_mode=1)
    assert O.rel_rms(R, o.pre) < IMG_TOL
    N = s.image_size
    yy, xx = np.mgrid[0:N, 0:N]
    px, py = xx.ravel(), yy.ravel()
    scale = _scale(s.cell_size, o.G)
    inc = O.inclusion_mask(o.r, scale, o.G, edge_mode=1)
    vin, q, sv, _ = O.preprocess64(s)
    inv_det = 1 / abs(o.vin[0, 0] * o.vin[1, 1] - o.vin[0, 1] * o.vin[1, 0])
    d = O.dft_pixels_sep(q, sv, o.vr, o.vi, inv_det, s.num_samples, o.vin, N, float(np.float32(s.cell_size)),
                         px, py, inc).reshape(N, N)
    err = O.rel_rms(R, d)
    print("small: rel RMS vs FP64 DFT", err)
    assert err < IMG_TOL


def test_fipipe_device_path_equals_engine(cuda_device, small_snapshot, small_run):
    s = small_snapshot
    buf = api.preprocess_measurement_set_gpu(s, want_bin=True)
    img = api.FIpipeDevice(buf, s.image_size, s.cell_size)
    api.free_device_preprocess_buffers(buf)
    assert O.rel_rms(img, small_run["image"]) < 1e-6


def _quartet():
    from tests.golden.make_golden import quartet
    return quartet()


def test_fipipe_matches_oracle(cuda_device):
    visr, visi, b, v, N, cell = _quartet()
    img = api.FIpipe(visr, visi, b, v, N, cell)
    o = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=0)
    assert O.rel_rms(img, o.image) < IMG_TOL
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32)) as e:
        img32 = e.fipipe(visr, visi, b, v, N, cell)
        assert e.stats()["num_terms"] == o.sc.K
    o32 = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    assert O.rel_rms(img32, o32.image) < IMG_TOL


def test_fipipe_binning_bit_exact(cuda_device):
    visr, visi, b, v, N, cell = _quartet()
    for cm in (0, 1):
        with api.Engine(api.archive_options(coord_mode=cm)) as e:
            e.fipipe(visr, visi, b, v, N, cell)
            _check_binning(e, e.stats(), b.astype(np.float64), visr, visi, cell, coord_mode=cm)


@pytest.mark.skipif(O.load_reference_fipipe() is None, reason="reference library not built")
def test_fipipe_matches_reference_binary(cuda_device):
    """The reference's own archive imager, compiled unmodified for sm_100a, on the same inputs."""
    visr, visi, b, v, N, cell = _quartet()
    ref = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    ref2 = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    assert np.any(ref != 0), "reference FIpipe returned an empty image (kernel launch failed?)"
    noise = O.rel_rms(ref2, ref)
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32)) as e:
        img32 = e.fipipe(visr, visi, b, v, N, cell)
    img64 = api.FIpipe(visr, visi, b, v, N, cell)
    e32, e64 = O.rel_rms(img32, ref), O.rel_rms(img64, ref)
    print(f"vs reference binary (--use_fast_math): ref32 {e32:.3e} fp64 {e64:.3e} "
          f"reference rerun noise {noise:.3e}")
    # At cell 4e-4 rad the reference's FP32 degree-based SIN reprojection (theta ~ 87 deg, one ulp
    # = 7.6e-6 deg) moves its splat positions by ~3e-4 pixel, in either of its builds, so its
    # image carries ~3e-4 rounding noise here; the 1e-5 parity is shown at a wide cell
    # (test_fipipe_matches_reference_binary_wide_cell), where that noise vanishes.
    assert e32 < 1e-3 and e64 < 1e-3
    refp = O.run_reference_fipipe(visr, visi, b, v, N, cell, precise=True)
    p32, p64 = O.rel_rms(img32, refp), O.rel_rms(img64, refp)
    print(f"vs reference binary (IEEE math): ref32 {p32:.3e} fp64 {p64:.3e}")
    assert p32 < 1e-3 and p64 < 1e-3


def _wide_cell_inputs():
    from tests.golden.make_golden import wide_cell_quartet
    return wide_cell_quartet()


@pytest.mark.skipif(O.load_reference_fipipe() is None, reason="reference library not built")
def test_fipipe_matches_reference_binary_wide_cell(cuda_device):
    visr, visi, b, v, N, cell = _wide_cell_inputs()
    refp = O.run_reference_fipipe(visr, visi, b, v, N, cell, precise=True)
    ref = O.run_reference_fipipe(visr, visi, b, v, N, cell)
    assert np.any(refp != 0)
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32)) as e:
        img32 = e.fipipe(visr, visi, b, v, N, cell)
    img64 = api.FIpipe(visr, visi, b, v, N, cell)
    o = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    vals = {"ref32/ieee": O.rel_rms(img32, refp), "fp64/ieee": O.rel_rms(img64, refp),
            "ref32/fast": O.rel_rms(img32, ref), "oracle/ieee": O.rel_rms(o.image, refp),
            "fast/ieee": O.rel_rms(ref, refp)}
    print("wide cell vs reference binary:", {k: f"{x:.2e}" for k, x in vals.items()})
    assert vals["ref32/ieee"] < IMG_TOL and vals["oracle/ieee"] < IMG_TOL
    assert vals["fp64/ieee"] < IMG_TOL


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fipk_small.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden output absent")
def test_fipipe_matches_reference_golden(cuda_device):
    visr, visi, b, v, N, cell = _quartet()
    z = np.load(GOLDEN)
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32)) as e:
        img = e.fipipe(visr, visi, b, v, N, cell)
    assert O.rel_rms(img, z["image_precise"]) < 1e-3
    assert O.rel_rms(img, z["image"]) < 1e-3
    zw = os.path.join(os.path.dirname(__file__), "golden", "fipk_widecell.npz")
    if os.path.exists(zw):
        from tests.golden.make_golden import wide_cell_quartet
        visr, visi, b, v, N, cell = wide_cell_quartet()
        with api.Engine(api.archive_options(coord_mode=api.COORD_REF32)) as e:
            img = e.fipipe(visr, visi, b, v, N, cell)
        assert O.rel_rms(img, np.load(zw)["image_precise"]) < IMG_TOL


def test_all_flagged_gives_zero_image(cuda_device):
    s = synth.make_snapshot("small", n_rows_limit=400, nchan=4)
    s.flag0[:] = 1
    s.flag3[:] = 1
    with api.Engine() as e:
        img = e.image(s)
    assert np.all(img == 0)


def test_empty_input_is_an_error(cuda_device):
    s = synth.make_snapshot("small", n_rows_limit=10, nchan=2)
    s.num_rows = 0
    with api.Engine() as e:
        with pytest.raises(api.SvdiError) as ei:
            e.image(s)
    assert ei.value.status == 2


def test_edge_clipping_and_integer_positions(cuda_device):
    """Samples whose footprints cross the grid edge (clipped, reference rule) or lie exactly on a
    grid cell (W+1-cell footprint carrying exp(-beta) at both ends) match the oracle."""
    N, cell = 64, 2e-3
    G = 96
    scale = float(np.float32(cell)) * G
    rng = np.random.default_rng(5)
    n = 3000
    b = rng.uniform(-1.0, 1.0, (n, 3)) * (G / 2 + 3) / scale
    b[:, 2] *= 1e-3
    # exact integer grid positions (scale * b integral): fraction 0 in both, one, other axis
    ints = rng.integers(-G // 2 + 5, G // 2 - 5, (300, 2)).astype(np.float64)
    b[:300, :2] = ints / scale
    b[300:400, 0] = ints[:100, 0] / scale
    b[400:500, 1] = ints[100:200, 1] / scale
    b = b.astype(np.float32)
    visr = rng.normal(size=n).astype(np.float32)
    visi = rng.normal(size=n).astype(np.float32)
    v = np.eye(3, dtype=np.float32)
    v[0] = [0.8, 0.6, 0.0]
    v[1] = [-0.6, 0.8, 0.0]
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32, keep_grid=1)) as e:
        img = e.fipipe(visr, visi, b, v, N, cell)
        st = e.stats()
        _check_binning(e, st, b.astype(np.float64), visr, visi, cell, coord_mode=1)
        grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    o = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    inv_det = 1.0 / abs(0.8 * 0.8 + 0.6 * 0.6)
    og = O.grid(b.astype(np.float64), visr, visi, scale, G, o.sc, inv_det, coord_mode=1)
    assert np.linalg.norm(grid - og) / np.linalg.norm(og) < GRID_TOL
    assert O.rel_rms(img, o.image) < IMG_TOL


def _piled_quartet():
    """50,000 samples on one (non-integer) grid position with large, nearly coherent values, beside
    10,000 ordinary samples: the pile's chunks carry a value sum ~2^10 times their maximum, so the
    fixed-point scale is set by the chunk sum (31 - e_sum) and consecutive chunks of the pile cannot
    share one accumulation run without exceeding 2^31."""
    N, cell, G = 64, 2e-3, 96
    scale = float(np.float32(cell)) * G
    rng = np.random.default_rng(11)
    n_pile, n_rest = 50_000, 10_000
    b = np.empty((n_pile + n_rest, 3))
    b[:n_pile] = np.array([7.37, -11.61, 0.0]) / scale
    b[n_pile:] = rng.uniform(-1.0, 1.0, (n_rest, 3)) * (G / 2 - 6) / scale
    b[:, 2] = rng.uniform(-1e-3, 1e-3, n_pile + n_rest)
    visr = np.concatenate([3.0e4 + rng.normal(0, 30.0, n_pile), rng.normal(size=n_rest)]).astype(np.float32)
    visi = np.concatenate([rng.normal(0, 30.0, n_pile), rng.normal(size=n_rest)]).astype(np.float32)
    return visr, visi, b.astype(np.float32), _tilted_basis(), N, cell, G, scale


def _tilted_basis():
    """A rotation about w by 0.3 rad, then a tilt of 0.05 rad (V31, V32 != 0). With an identity
    basis the archive SIN deprojection maps every pixel onto an exact integer position, and whether
    a pixel landing exactly on the splat bound |L| = N/2 - 1 is kept then depends on the last bit
    of its FP64 arithmetic (glibc and CUDA's math differ there); this basis keeps every target at
    least 5e-3 pixel away from that bound."""
    a, t = 0.3, 0.05
    rz = np.array([[np.cos(a), np.sin(a), 0.0], [-np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
    rx = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(t), np.sin(t)], [0.0, -np.sin(t), np.cos(t)]])
    return (rx @ rz).astype(np.float32)


def test_samples_piled_on_one_position(cuda_device):
    """Coincident samples (the domain's collisions): one tile key holds most of the snapshot, the
    chunk-sum bound sets the fixed-point scale and the pile is flushed chunk by chunk. Records are
    bit-exact; grid planes and image match the FP64 oracle."""
    visr, visi, b, v, N, cell, G, scale = _piled_quartet()
    with api.Engine(api.archive_options(coord_mode=api.COORD_REF32, keep_grid=1)) as e:
        img = e.fipipe(visr, visi, b, v, N, cell)
        st = e.stats()
        _check_binning(e, st, b.astype(np.float64), visr, visi, cell, coord_mode=1)
        grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    o = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    V = v.astype(np.float64)
    inv_det = 1.0 / abs(V[0, 0] * V[1, 1] - V[0, 1] * V[1, 0])
    og = O.grid(b.astype(np.float64), visr, visi, scale, G, o.sc, inv_det, coord_mode=1)
    assert np.linalg.norm(grid - og) / np.linalg.norm(og) < GRID_TOL
    assert O.rel_rms(img, o.image) < IMG_TOL


@pytest.mark.parametrize("N", [255, 100, 64])
def test_odd_and_small_image_sizes(cuda_device, N):
    s = synth.make_snapshot("small", n_rows_limit=3000, nchan=8)
    cell = 4e-4 * 256 / N
    with api.Engine() as e:
        img = e.image(s, N, cell)
    o = O.image_sii(s, N, cell)
    assert O.rel_rms(img, o.image) < IMG_TOL


def test_wterm_multi_slab_matches_oracle_and_dft(cuda_device):
    """Non-coplanar snapshot: several w-slabs x Chebyshev terms (tile 32 gridder, K > 1)."""
    s = snapshot("widefield", nchan=4, n_rows_limit=6000, image_size=128, cell_size=6e-4)
    with api.Engine(k_rule=api.KRULE_FIXED, fixed_k=12, target_alpha=2.0, edge_mode=api.EDGE_STRICT,
                    presplat=1) as e:
        R = e.image(s)
        st = e.stats()
    o = O.image_sii(s, edge_mode=1, k_rule=12, target_alpha=2.0)
    assert st["num_slabs"] == o.sc.num_slabs > 1 and st["num_terms"] == 12
    assert O.rel_rms(R, o.pre) < IMG_TOL
    rng = np.random.default_rng(2)
    N = s.image_size
    px, py = rng.integers(0, N, 300), rng.integers(0, N, 300)
    inc = O.inclusion_mask(o.r, _scale(s.cell_size, o.G), o.G, edge_mode=1)
    inv_det = 1 / abs(o.vin[0, 0] * o.vin[1, 1] - o.vin[0, 1] * o.vin[1, 0])
    d = O.dft_pixels(o.r, o.vr, o.vi, inv_det, s.num_samples, o.vin, N, float(np.float32(s.cell_size)), px, py,
                     inc)
    m = np.isfinite(d)
    assert O.rel_rms(R[py, px][m], d[m]) < IMG_TOL


def test_slab_batches_add_signed_sums(cuda_device):
    """Slabs imaged in several batches (max_batch_slabs = 1) give the image of one batch: the
    signed sums of the batches add before |.| is taken."""
    s = snapshot("widefield", nchan=4, n_rows_limit=6000, image_size=128, cell_size=6e-4)
    kw = dict(k_rule=api.KRULE_FIXED, fixed_k=12, target_alpha=2.0, edge_mode=api.EDGE_STRICT)
    with api.Engine(**kw) as e:
        one = e.image(s)
        assert e.stats()["num_slabs"] > 1
    with api.Engine(max_batch_slabs=1, **kw) as e:
        many = e.image(s)
    assert O.rel_rms(many, one) < 1e-6
    with api.Engine(presplat=1, **kw) as e:
        one_p = e.image(s)
    with api.Engine(presplat=1, max_batch_slabs=1, **kw) as e:
        many_p = e.image(s)
    m = np.isfinite(one_p)
    assert np.array_equal(m, np.isfinite(many_p))
    assert O.rel_rms(many_p[m], one_p[m]) < 5e-6  # cuFFT batch shapes differ: FP32 rounding


def test_slab_batching_matches_single_batch_when_one_slab(cuda_device, small_snapshot):
    with api.Engine(max_batch_slabs=1) as e:
        a = e.image(small_snapshot)
    with api.Engine() as e:
        b = e.image(small_snapshot)
    assert O.rel_rms(a, b) < 1e-6


def test_repeat_calls_are_stable(cuda_device, small_snapshot):
    with api.Engine() as e:
        a = e.image(small_snapshot)
        b = e.image(small_snapshot)
    assert O.rel_rms(a, b) < 1e-6


def test_archive_cli_round_trip(cuda_device, tmp_path):
    """sharedlibrary_gpu with FITS inputs (archive/pipe_interface.cpp argv) equals api.FIpipe."""
    from svdimager_b200 import fits
    visr, visi, b, v, N, cell = _quartet()
    paths = {}
    for name, arr in (("Visreal", visr), ("Visimag", visi), ("B", b), ("V", v)):
        paths[name] = str(tmp_path / f"{name}.fits")
        fits.write_fits(paths[name], arr.astype(np.float64))  # SVD_MFS.py writes float64
    out = str(tmp_path / "out.fits")
    exe = os.path.join(os.path.dirname(api.HERE), "svdimager_b200", "bin", "sharedlibrary_gpu")
    r = subprocess.run([exe, paths["Visreal"], paths["Visimag"], paths["B"], paths["V"], str(N), str(len(visr)),
                        repr(cell), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = fits.read_fits(out)
    ref = api.FIpipe(visr, visi, b, v, N, np.float32(cell))
    assert O.rel_rms(img, ref) < 1e-6


def test_archive_cli_writes_sin_wcs_on_request(cuda_device, tmp_path):
    """With SVDI_FITS_WCS="ra,dec" the CLIs add SIN world coordinates to the header; the image
    itself is unchanged (the reference writes bare images, which stays the default)."""
    from svdimager_b200 import fits
    visr, visi, b, v, N, cell = _quartet()
    paths = {}
    for name, arr in (("Visreal", visr), ("Visimag", visi), ("B", b), ("V", v)):
        paths[name] = str(tmp_path / f"{name}.fits")
        fits.write_fits(paths[name], arr.astype(np.float64))
    exe = os.path.join(os.path.dirname(api.HERE), "svdimager_b200", "bin", "sharedlibrary_gpu")
    outs = {}
    for tag, extra in (("bare", {}), ("wcs", {"SVDI_FITS_WCS": "150.5,-30.25"})):
        outs[tag] = str(tmp_path / f"{tag}.fits")
        env = {k: val for k, val in os.environ.items() if k != "SVDI_FITS_WCS"}
        env.update(extra)
        r = subprocess.run([exe, paths["Visreal"], paths["Visimag"], paths["B"], paths["V"], str(N), str(len(visr)),
                            repr(cell), outs[tag]], capture_output=True, text=True, env=env)
        assert r.returncode == 0, r.stderr
    with open(outs["wcs"], "rb") as f:
        hdr, _ = fits.read_header(f.read())
    with open(outs["bare"], "rb") as f:
        bare, _ = fits.read_header(f.read())
    assert "CTYPE1" not in bare
    assert hdr["CTYPE1"] == "RA---SIN" and hdr["CTYPE2"] == "DEC--SIN"
    assert hdr["CRVAL1"] == 150.5 and hdr["CRVAL2"] == -30.25 and hdr["CRPIX1"] == N // 2 + 1
    assert abs(hdr["CDELT2"] - math.degrees(float(np.float32(cell)))) < 1e-12
    assert O.rel_rms(fits.read_fits(outs["wcs"]), fits.read_fits(outs["bare"])) < 1e-6


def test_integrated_cli_round_trip(cuda_device, tmp_path):
    """svd_integrated_imager_gpu on a snapshot bundle equals the engine on the same snapshot."""
    from svdimager_b200 import bundle, fits
    s0 = synth.make_snapshot("small", n_rows_limit=2000, nchan=8, snapshot_index=0)
    s1 = synth.make_snapshot("small", n_rows_limit=2000, nchan=8, snapshot_index=1)
    p = str(tmp_path / "obs.ms")
    bundle.write_bundle(p, [s1, s0])
    out = str(tmp_path / "img.fits")
    exe = os.path.join(os.path.dirname(api.HERE), "svdimager_b200", "bin", "svd_integrated_imager_gpu")
    r = subprocess.run([exe, p, "128", "8e-4", "1", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "Found 2 TIME snapshot(s)" in r.stderr
    img = fits.read_fits(out)
    with api.Engine() as e:
        ref = e.image(s1, 128, 8e-4)
    assert O.rel_rms(img, ref) < 1e-6


def test_precision_config_properties(cuda_device):
    """The headline configuration (8.4M samples, 2048^2): flag mask, sample accounting and
    accuracy against the FP64 DFT at random pixels (strict inclusion)."""
    s = snapshot("precision")
    with api.Engine(edge_mode=api.EDGE_STRICT, presplat=1, k_rule=api.KRULE_TARGET,
                    target_error=1e-7) as e:
        R = e.image(s)
        st = e.stats()
        vr, vi = e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG)
        q, sv = e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S)
    ovr, ovi = O.collapse(s)
    assert np.array_equal(vr, ovr) and np.array_equal(vi, ovi)
    vin = np.array(st["vin"]).reshape(3, 3)
    r = O.expand_coords(q, sv)
    G = st["grid_size"]
    inc = O.inclusion_mask(r, _scale(s.cell_size, G), G, edge_mode=1)
    assert st["num_gridded"] == int(inc.sum())
    rng = np.random.default_rng(7)
    N = s.image_size
    npix = 256
    px, py = rng.integers(0, N, npix), rng.integers(0, N, npix)
    inv_det = 1 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    d = O.dft_pixels_sep(q, sv, vr, vi, inv_det, s.num_samples, vin, N, float(np.float32(s.cell_size)), px, py, inc)
    err = O.rel_rms(R[py, px], d)
    print("precision: K", st["num_terms"], "slabs", st["num_slabs"], "rel RMS vs FP64 DFT", err)
    assert err < IMG_TOL


@pytest.mark.parametrize("K", [2, 3, 5])
def test_fixed_order_tile32_matches_oracle(cuda_device, small_snapshot, K):
    """Fixed Chebyshev orders on 32x32 tiles: the gridder covers K terms with its 8-, 4-, 2- and
    1-term variants (K = 2: one two-term pass; 3: two plus one; 5: four plus one)."""
    s = small_snapshot
    with api.Engine(k_rule=api.KRULE_FIXED, fixed_k=K, tile=32) as e:
        img = e.image(s)
        st = e.stats()
    assert st["num_terms"] == K and st["tile"] == 32
    o = O.image_sii(s, k_rule=K)
    assert O.rel_rms(img, o.image) < IMG_TOL


@pytest.mark.parametrize("bad", ["nan_under_flag", "inf"])
def test_non_finite_visibility_makes_a_nan_image(cuda_device, bad):
    """A NaN under a flag (the reference multiplies it by the flag's zero weight,
    SVDIntegratedImager.cu:606-612, and NaN * 0 is NaN) or an Inf in one gridded sample: the
    reference's float atomics carry it into the grid and its FFT into every moment cell, so every
    pixel the reprojection reaches is non-finite. The oracle does the same arithmetic in FP64;
    the non-finite pixels of this path's image are exactly the oracle's, and the rest are 0."""
    import dataclasses
    s0 = snapshot("small", n_rows_limit=3000, nchan=8)
    s = dataclasses.replace(s0, vis0_real=s0.vis0_real.copy(), flag0=s0.flag0.copy(),
                            flag3=s0.flag3.copy())
    k = int(np.argmin(np.abs(s.uvw[:, :2]).sum(axis=1)))   # shortest baseline, channel 0: gridded
    s.flag3[k] = 0
    if bad == "nan_under_flag":
        s.vis0_real[k], s.flag0[k] = np.float32(np.nan), 1
    else:
        s.vis0_real[k], s.flag0[k] = np.float32(np.inf), 0
    with api.Engine() as e:
        img = e.image(s)
    with np.errstate(invalid="ignore", over="ignore"):
        o = O.image_sii(s)
    bad_gpu, bad_orc = ~np.isfinite(img), ~np.isfinite(o.image)
    assert bad_orc.sum() > img.size // 4
    assert np.array_equal(bad_gpu, bad_orc)
    assert np.all(img[~bad_gpu] == 0) and np.all(o.image[~bad_orc] == 0)
