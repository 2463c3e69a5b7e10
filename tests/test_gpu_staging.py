"""Pageable host copies through the engine's pinned staging ring (host_stage.cu) against plain
copies from pinned memory. The archive entry stages pageable inputs of 4 MB or more in 16 MB
chunks through a three-slot ring and downloads a pageable image of 4 MB or more the same way;
pinned arrays take a single cudaMemcpyAsync each.

A 4.7 M-sample quartet (Visreal 19 MB: two chunks; Bin 56 MB: four; the ring wraps twice) made of
the small quartet repeated with a different visibility phase and baseline scale per copy, so that a
chunk written to the wrong place changes the image: the device copy of Visreal/Visimag is
bit-identical to the host arrays, and the image from pageable buffers equals the image from pinned
buffers to 1e-6 relative RMS (float atomics in the gridder's tile flush make the last bits
run-dependent)."""
import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api

pytestmark = pytest.mark.gpu

N = 2048  # a 16.8 MB image: one full chunk and a short one


def _big_quartet(reps=36):
    from tests.golden.make_golden import quartet
    vr, vi, b, v, n0, cell = quartet()
    rng = np.random.default_rng(5)
    vis = vr.astype(np.complex64) + 1j * vi.astype(np.complex64)
    VR, VI, B = [], [], []
    for k in range(reps):
        ph = np.exp(1j * rng.uniform(0, 2 * np.pi)).astype(np.complex64)
        w = vis * ph
        VR.append(w.real.astype(np.float32))
        VI.append(w.imag.astype(np.float32))
        B.append((b * np.float32(1.0 - 0.015 * k)).astype(np.float32))
    # the small configuration's field of view at N pixels
    return np.concatenate(VR), np.concatenate(VI), np.concatenate(B), v, cell * n0 / N


def _pinned_copy(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
    arr = t.numpy()
    arr[...] = a
    return t, arr


def test_staged_archive_copies_equal_pinned_copies(cuda_device):
    vr, vi, b, v, cell = _big_quartet()
    n = vr.shape[0]
    assert n * 4 > 16 << 20 and b.nbytes > 3 * (16 << 20)
    keep = []
    pinned = []
    for a in (vr, vi, b):
        t, arr = _pinned_copy(a)
        keep.append(t)
        pinned.append(arr)
    t_out, out_pinned = _pinned_copy(np.zeros((N, N), np.float32))
    keep.append(t_out)
    with api.Engine(api.archive_options()) as e:
        img_pageable = e.fipipe(vr, vi, b, v, N, cell)
        assert np.array_equal(e.buffer(api.BUF_VIS_REAL), vr)
        assert np.array_equal(e.buffer(api.BUF_VIS_IMAG), vi)
        terms = e.stats()["num_terms"]
        e.fipipe(pinned[0], pinned[1], pinned[2], v, N, cell, out=out_pinned)
        img_pinned = out_pinned.copy()
        assert e.stats()["num_terms"] == terms
        # pinned inputs, pageable output; then pageable inputs again after the ring has wrapped
        img_mixed = e.fipipe(pinned[0], pinned[1], pinned[2], v, N, cell)
        img_again = e.fipipe(vr, vi, b, v, N, cell)
    assert np.abs(img_pinned).max() > 0
    for img in (img_pageable, img_mixed, img_again):
        err = O.rel_rms(img, img_pinned)
        print("rel RMS", err)
        assert err < 1e-6
