"""Batches imaged by one CUDA-graph launch, the FP64 direct-DFT accuracy probe, and the autotuner.

The batch replays exactly the device work of the per-snapshot engine with each snapshot's recorded
plan, so its images equal the engine's images up to the order of floating-point atomic adds
(relative RMS < 1e-6). The probe and the oracle both evaluate the FP64 DFT (the oracle with a
channel recurrence), so they agree to ~1e-10."""
import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, autotune, synth

pytestmark = pytest.mark.gpu

N, CELL = 256, 4e-4


def _upload(snaps, torch):
    dev = torch.device("cuda", 0)
    keep, descs = [], []
    for s in snaps:
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in s.arrays().items()}
        keep.append(t)
        descs.append(api.device_ms(s.num_rows, s.num_channels, t, s.array_center_x))
    return keep, descs


@pytest.fixture(scope="module")
def stream5():
    return synth.batching_stream(5, n_rows_limit=3000)


def test_dft_probe_matches_oracle(cuda_device, small_snapshot):
    s = small_snapshot
    with api.Engine(edge_mode=api.EDGE_STRICT, presplat=1) as e:
        R = e.image(s)
        vin = np.array(e.stats()["vin"]).reshape(3, 3)
        q, sv = e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S)
        vr, vi = e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG)
        G = e.stats()["grid_size"]
        rng = np.random.default_rng(3)
        px, py = rng.integers(0, s.image_size, 64), rng.integers(0, s.image_size, 64)
        probe = e.dft_pixels(px, py)
    inc = O.inclusion_mask(O.expand_coords(q, sv), float(np.float32(s.cell_size)) * G, G, edge_mode=1)
    inv_det = 1 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    d = O.dft_pixels_sep(q, sv, vr, vi, inv_det, s.num_samples, vin, s.image_size,
                         float(np.float32(s.cell_size)), px, py, inc)
    m = np.isfinite(d)
    assert np.array_equal(m, np.isfinite(probe))
    assert np.max(np.abs(probe[m] - d[m])) <= 1e-9 * np.max(np.abs(d[m]))
    assert O.rel_rms(R[py, px][m], probe[m]) < 1e-5


def _batch_vs_single(stream5, **opts):
    import torch
    keep, descs = _upload(stream5, torch)
    imgs = torch.zeros((len(descs), N, N), dtype=torch.float32, device="cuda")
    single = torch.zeros((N, N), dtype=torch.float32, device="cuda")
    with api.Engine(edge_mode=api.EDGE_STRICT, **opts) as ref:
        refs = []
        for d in descs:
            ref.image_device(d, N, CELL, single.data_ptr())
            refs.append(single.cpu().numpy().copy())
    e = api.Engine(edge_mode=api.EDGE_STRICT, **opts)
    b = api.Batch(e, descs, N, CELL, imgs.data_ptr())
    imgs.zero_()
    b.launch()
    b.check()
    out1 = imgs.cpu().numpy().copy()
    for i in range(len(descs)):
        assert O.rel_rms(out1[i], refs[i]) < 1e-6, i
    b.launch()
    b.check()
    assert O.rel_rms(imgs.cpu().numpy(), out1) < 1e-6
    return keep, descs, imgs, b, e, out1


def test_batch_matches_single_images(cuda_device, stream5):
    keep, descs, imgs, b, e, out1 = _batch_vs_single(stream5)
    plans = [b.plan(i) for i in range(len(descs))]
    assert all(p["num_slabs"] >= 1 and p["num_terms"] >= 1 for p in plans)
    # refill snapshot 0's visibilities in place: the image scales linearly, the others stay
    for k in ("vis0_real", "vis0_imag", "vis3_real", "vis3_imag"):
        keep[0][k].mul_(2.0)
    b.launch()
    b.check()
    out2 = imgs.cpu().numpy()
    assert O.rel_rms(out2[0], 2.0 * out1[0]) < 1e-6
    assert O.rel_rms(out2[1:], out1[1:]) < 1e-6
    b.close()
    e.close()


def test_large_batch_splits_in_two_halves(cuda_device):
    """A batch of 17 snapshots runs as two halves (8 and 9 snapshots) on two engines whose graphs
    launch side by side: every image equals the engine's, a second launch repeats them, the plan of
    a snapshot in either half is the engine's and the batch is wide."""
    snaps = synth.batching_stream(17, n_rows_limit=2000)
    keep, descs, imgs, b, e, out1 = _batch_vs_single(snaps)
    assert b.wide
    with api.Engine(edge_mode=api.EDGE_STRICT) as ref:
        import torch
        single = torch.zeros((N, N), dtype=torch.float32, device="cuda")
        for i in (0, 8, 16):
            ref.image_device(descs[i], N, CELL, single.data_ptr())
            torch.cuda.synchronize()
            st = ref.stats()
            assert b.plan(i) == {"num_slabs": st["num_slabs"], "num_terms": st["num_terms"]}
    b.close()
    e.close()


def test_batch_is_wide(cuda_device, stream5):
    keep, descs, imgs, b, e, out1 = _batch_vs_single(stream5)
    assert b.wide
    b.close()
    e.close()


def test_wide_batch_with_mixed_chebyshev_orders(cuda_device, stream5):
    """A snapshot with a large w range (elevated stations) beside two of the batching stream: the
    error-target rule gives them different Chebyshev orders and slab counts, so the batch grids two
    groups of tile keys (32 x 32 tiles, Chebyshev arguments per record) with one launch each; every
    image equals the engine's."""
    wf = synth.make_snapshot("widefield", n_rows_limit=3000, nchan=8)
    snaps = [stream5[0], wf, stream5[1]]
    keep, descs, imgs, b, e, out1 = _batch_vs_single(snaps, k_rule=api.KRULE_TARGET, target_error=1e-6)
    assert b.wide
    plans = [b.plan(i) for i in range(len(descs))]
    assert len({p["num_terms"] for p in plans}) > 1, plans
    b.close()
    e.close()


def test_wide_batch_integer_gridder_mixed_chebyshev_orders(cuda_device, stream5):
    """The mixed-order batch on the integer tensor-core gridder: each group of tile keys is gridded
    by one launch per Chebyshev term (the multi-term group reads the records' Chebyshev arguments);
    every image equals the engine's."""
    wf = synth.make_snapshot("widefield", n_rows_limit=3000, nchan=8)
    snaps = [stream5[0], wf, stream5[1]]
    keep, descs, imgs, b, e, out1 = _batch_vs_single(snaps, gridder=api.GRIDDER_TC_I8,
                                                     k_rule=api.KRULE_TARGET, target_error=1e-6)
    assert b.wide
    plans = [b.plan(i) for i in range(len(descs))]
    assert max(p["num_terms"] for p in plans) > 1, plans
    b.close()
    e.close()


@pytest.mark.parametrize("gridder", [api.GRIDDER_TC, api.GRIDDER_TC_I8])
def test_batch_tensor_core_gridder(cuda_device, stream5, gridder):
    """Wide batch on a tensor-core gridder (split FP16 and exact integer): one gridder launch over
    the tile keys of all snapshots; every image equals the engine's."""
    keep, descs, imgs, b, e, out1 = _batch_vs_single(stream5, gridder=gridder, k_rule=api.KRULE_FIXED,
                                                     fixed_k=1)
    assert b.wide
    b.close()
    e.close()


def test_engine_holds_one_batch(cuda_device, stream5):
    import torch
    keep, descs = _upload(stream5[:2], torch)
    imgs = torch.zeros((2, N, N), dtype=torch.float32, device="cuda")
    with api.Engine() as e:
        b = api.Batch(e, descs, N, CELL, imgs.data_ptr())
        with pytest.raises(api.SvdiError):
            api.Batch(e, descs, N, CELL, imgs.data_ptr())
        b.close()
        b2 = api.Batch(e, descs, N, CELL, imgs.data_ptr())
        b2.close()


def test_autotune_picks_an_accurate_fast_option(cuda_device, stream5):
    import torch
    keep, descs = _upload(stream5[:2], torch)
    out = torch.zeros((N, N), dtype=torch.float32, device="cuda")
    cands = autotune.candidates(supports=(6, 8), sigmas=(1.5, 2.0), tiles=(64,))
    best, trials = autotune.tune(descs, N, CELL, out, cands=cands, repeats=3)
    assert len(trials) == len(cands) + 1   # the default options are always tried
    chosen = [t for t in trials if t.options["support"] == best["support"] and t.options["sigma"] == best["sigma"]
              and t.options["gridder"] == best["gridder"] and t.options["tile"] == best["tile"]][0]
    assert chosen.error <= 1e-5
    fastest = min(t.ms for t in trials if t.error <= 1e-5 and np.isfinite(t.ms))
    is_default = all(chosen.options.get(k) == v for k, v in autotune.DEFAULT_CANDIDATE.items())
    # the fastest accurate candidate, or the default options when nothing beats them by the margin
    assert chosen.ms == fastest or (is_default and fastest > 0.97 * chosen.ms)
