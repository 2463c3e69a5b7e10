"""The archive entry's inputs from a snapshot: the FITS quartet of archive/SVD_MFS.py.

SVD_MFS.py (archive/SVD_MFS.py:1-106) reads a Measurement Set with casacore, scales UVW by
frequency (rows x channels flattened channel-major), finds the principal axes with scikit-learn's
PCA, collapses polarisations 0 and 3 with FLAG and WEIGHT_SPECTRUM, and writes Bin{i}.fits
(the baselines in the PCA frame, not centred), Min{i}.fits (their mean), Vin{i}.fits (the axes as
rows) and Visreal{i}.fits / Visimag{i}.fits, all float64. Here the same quantities come from the
library's device preprocessing (svdi_preprocess_measurement_set: FP64 rotation, collapse); the
axes take scikit-learn's sign convention (the largest |entry| of every axis positive, sklearn's
svd_flip) instead of the main path's array-centre orientation, and Bin's columns follow them."""
from __future__ import annotations

import os

import numpy as np

from . import api, fits

C_LIGHT = 299792458.0


def quartet(snap):
    """{"Visreal", "Visimag" (float32 [N_s]), "Bin" (float32 [N_s][3]), "Vin" (float64 [3][3]),
    "Min" (float64 [1][3])} of a snapshot (synth.Snapshot or a bundle snapshot)."""
    bufs = api.preprocess_measurement_set_gpu(snap, want_bin=True)
    try:
        b = bufs.buf
        n = int(b.num_samples)
        vr = api.copy_to_host(np.empty(n, np.float32), b.d_vis_real)
        vi = api.copy_to_host(np.empty(n, np.float32), b.d_vis_imag)
        bn = api.copy_to_host(np.empty((n, 3), np.float32), b.d_bin)
        V = api.copy_to_host(np.empty((3, 3), np.float64), b.d_vin64)
    finally:
        bufs.free()
    for k in range(3):  # scikit-learn's axis signs
        j = int(np.argmax(np.abs(V[k])))
        if V[k, j] < 0:
            V[k] = -V[k]
            bn[:, k] = -bn[:, k]
    uvw = np.asarray(snap.uvw, np.float64)
    s = np.asarray(snap.frequencies_hz, np.float64) / C_LIGHT
    mean = uvw.sum(axis=0) * s.sum() / n  # mean of b = uvw_row f_chan / c over all samples
    return {"Visreal": vr, "Visimag": vi, "Bin": bn, "Vin": V, "Min": mean[None, :]}


def write_quartet(snap, directory: str, index: int = 0):
    """Write Bin{index}.fits, Min{index}.fits, Vin{index}.fits, Visreal{index}.fits and
    Visimag{index}.fits (float64, as SVD_MFS.py) into `directory`; returns their paths."""
    q = quartet(snap)
    paths = {}
    for name in ("Bin", "Min", "Vin", "Visreal", "Visimag"):
        paths[name] = os.path.join(directory, f"{name}{index}.fits")
        fits.write_fits(paths[name], np.asarray(q[name], np.float64))
    return paths
