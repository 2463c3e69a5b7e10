"""The FITS quartet for the archive entry (svdimager_b200.mfs) against a restatement of the
reference's pre-processor archive/SVD_MFS.py:33-106 with scikit-learn's PCA, and through the
archive CLI. Tolerances: the axes agree in FP64 (1e-9), Bin to float32 rounding, Min to 1e-12
relative, the collapsed visibilities to float32 rounding, the CLI image to 1e-6 relative RMS."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, fits, mfs, synth

pytestmark = pytest.mark.gpu


def _svd_mfs(snap):
    """archive/SVD_MFS.py:33-106 on a snapshot's arrays (float64 numpy, scikit-learn PCA)."""
    from sklearn.decomposition import PCA
    R, C = snap.num_rows, snap.num_channels
    nu = snap.frequencies_hz.astype(np.float64)
    uvw = snap.uvw.astype(np.float64)
    D = np.column_stack([(uvw[:, a:a + 1] * nu / mfs.C_LIGHT).ravel(order="F") for a in range(3)])
    pca = PCA(3)
    pca.fit(D)
    V = pca.components_
    B1 = pca.transform(D)
    M = np.mean(D, axis=0)
    Bin = B1 + np.array([np.dot(M, V[k]) for k in range(3)])[None, :]  # Bin[:, k] - dot(-M, V[k])
    f0 = snap.flag0.reshape(C, R).T != 0
    f3 = snap.flag3.reshape(C, R).T != 0
    w0 = snap.weight0.reshape(C, R).T.astype(np.float64) * (~f0)
    w3 = snap.weight3.reshape(C, R).T.astype(np.float64) * (~f3)
    v0 = (snap.vis0_real + 1j * snap.vis0_imag.astype(np.float64)).reshape(C, R).T
    v3 = (snap.vis3_real + 1j * snap.vis3_imag.astype(np.float64)).reshape(C, R).T
    ws = w0 + w3
    safe = np.where(ws > 0, ws, 1.0)
    vis = np.where(ws > 0, (v0 * w0 + v3 * w3) / safe, 0.0)
    return vis.real.ravel(order="F"), vis.imag.ravel(order="F"), Bin, V, M


def test_quartet_matches_the_reference_preprocessor(cuda_device):
    s = synth.make_snapshot("small")
    q = mfs.quartet(s)
    vr, vi, Bin, V, M = _svd_mfs(s)
    assert np.max(np.abs(q["Vin"] - V)) < 1e-9
    assert np.max(np.abs(q["Min"][0] - M)) <= 1e-12 * np.max(np.abs(M))
    scale = np.max(np.abs(Bin))
    assert np.max(np.abs(q["Bin"] - Bin)) <= 2e-7 * scale
    vmax = np.max(np.abs(vr))
    assert np.max(np.abs(q["Visreal"] - vr)) <= 2e-7 * vmax
    assert np.max(np.abs(q["Visimag"] - vi)) <= 2e-7 * vmax


def test_written_quartet_images_through_the_archive_cli(cuda_device, tmp_path):
    s = synth.make_snapshot("small", n_rows_limit=3000)
    paths = mfs.write_quartet(s, str(tmp_path), index=0)
    assert sorted(os.path.basename(p) for p in paths.values()) == [
        "Bin0.fits", "Min0.fits", "Vin0.fits", "Visimag0.fits", "Visreal0.fits"]
    b = fits.read_fits(paths["Bin"])
    assert b.shape == (s.num_rows * s.num_channels, 3)
    out = str(tmp_path / "img.fits")
    exe = os.path.join(os.path.dirname(api.HERE), "svdimager_b200", "bin", "sharedlibrary_gpu")
    r = subprocess.run([exe, paths["Visreal"], paths["Visimag"], paths["Bin"], paths["Vin"], str(s.image_size),
                        str(s.num_rows * s.num_channels), repr(s.cell_size), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    q = mfs.quartet(s)
    ref = api.FIpipe(q["Visreal"], q["Visimag"], q["Bin"], q["Vin"].astype(np.float32), s.image_size,
                     np.float32(s.cell_size))
    assert O.rel_rms(fits.read_fits(out), ref) < 1e-6
