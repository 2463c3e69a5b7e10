"""Allocation-free binning entry point (svdi_bin_samples_noalloc).

It serves callers that cannot allocate device memory while they run (a real-time correlator loop
with a memory budget fixed at start-up, or a framework that owns the device's memory pool), so it
keeps its scratch in a static device array instead of calling cudaMalloc. This file is collected
last so that a stop-at-first-failure run has already run every other test. The check: two calls
in a row, each compared with the engine's own binning of the same samples (integer work:
bit-exact per tile key)."""
import ctypes

import numpy as np
import pytest

from svdimager_b200 import api

pytestmark = pytest.mark.gpu


def _engine_binning(visr, visi, b, v, N, cell, tile):
    with api.Engine(api.archive_options(coord_mode=api.COORD_FP64, tile=tile)) as e:
        e.fipipe(visr, visi, b, v, N, cell)
        st = e.stats()
        assert st["num_terms"] == 1 and st["num_slabs"] == 1
        return e.buffer(api.BUF_OFFSETS), e.buffer(api.BUF_RECORDS), st


def _sorted_per_key(offsets, rec):
    kk = np.repeat(np.arange(len(offsets) - 1), np.diff(offsets.astype(np.int64)))
    return rec[np.lexsort((rec["vim"], rec["vre"], rec["yq"], rec["xq"], kk))]


def test_noalloc_binning_matches_engine_twice(cuda_device):
    import torch
    from tests.golden.make_golden import quartet
    visr, visi, b, v, N, cell = quartet()
    tile = 64
    off_ref, rec_ref, st = _engine_binning(visr, visi, b, v, N, cell, tile)
    V = v.astype(np.float64)
    inv_det = float(np.float32(1.0 / abs(V[0, 0] * V[1, 1] - V[0, 1] * V[1, 0])))
    n = len(visr)
    G = (3 * N + 1) // 2
    n_keys = ((G + tile - 1) // tile) ** 2
    assert n_keys <= api.NOALLOC_MAX_KEYS
    dev = cuda_device
    tb = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    tr = torch.from_numpy(visr).to(dev)
    ti = torch.from_numpy(visi).to(dev)
    rec = torch.empty(n * 16, dtype=torch.uint8, device=dev)
    off = torch.empty(n_keys + 1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        rec.fill_(0xAB)
        off.fill_(-1)
        torch.cuda.synchronize(dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        api.bin_samples_noalloc(tb.data_ptr(), tr.data_ptr(), ti.data_ptr(), n, N, cell, tile, inv_det,
                                rec.data_ptr(), off.data_ptr(), n_keys + 1, stream)
        torch.cuda.synchronize(dev)
        if call == 1:  # the first call may load the module; later calls take no device memory
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "the call allocated device memory"
        o = off.cpu().numpy().view(np.uint32)
        assert np.array_equal(o, off_ref), f"call {call}: offsets differ"
        total = int(o[-1])
        assert total == st["num_gridded"]
        r = rec.cpu().numpy()[: total * 16].view(rec_ref.dtype)
        assert np.array_equal(_sorted_per_key(o, r), _sorted_per_key(off_ref, rec_ref)), f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_device):
    import torch
    t = torch.zeros(16, device=cuda_device)
    with pytest.raises(api.SvdiError) as ei:
        # N = 8192 at tile 32: 384^2 tile keys > SVDI_NOALLOC_MAX_KEYS
        api.bin_samples_noalloc(t.data_ptr(), t.data_ptr(), t.data_ptr(), 4, 8192, 1e-4, 32, 1.0,
                                t.data_ptr(), t.data_ptr(), 10 ** 6, 0)
    assert ei.value.status == 6 and "allocation-free limit" in ei.value.message
