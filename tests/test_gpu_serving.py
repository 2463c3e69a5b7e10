"""Serving loop (svdi_server_*): continuous batching over resident engines.

Each request's image must be the same whether it runs alone or concurrently with others
(overlapping on the GPU in other slots); failures are isolated to their request; requests that can
never fit the HBM budget are refused at submission."""
import time

import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, synth

pytestmark = pytest.mark.gpu

MIX_TOL = 1e-6  # float reductions across tile segments may round differently between runs


def _mix():
    """Snapshots of different layouts, channel counts, flag fractions and image sizes."""
    out = []
    out.append((synth.make_snapshot("small"), 256, 4e-4))
    out.append((synth.make_snapshot("small", nchan=8, flag_fraction_rows=0.3, snapshot_index=1), 512, 2e-4))
    out.append((synth.make_snapshot("batching", nchan=16, hour_angle=0.5, flag_fraction_rows=0.0,
                                    flag_fraction_samples=0.2, snapshot_index=2), 1024, 1e-4))
    out.append((synth.make_snapshot("batching", nchan=32, hour_angle=-1.0, flag_fraction_rows=0.1,
                                    snapshot_index=3), 512, 2e-4))
    out.append((synth.make_snapshot("small", nchan=4, snapshot_index=4), 256, 4e-4))
    return out


@pytest.fixture(scope="module")
def mix():
    return _mix()


@pytest.fixture(scope="module")
def alone(cuda_device, mix):
    imgs = []
    with api.Engine() as e:
        for s, N, cell in mix:
            imgs.append(e.image(s, N, cell).copy())
    return imgs


def test_same_result_alone_and_in_the_mix(alone, mix):
    with api.Server(num_slots=4) as srv:
        tickets = []
        for rep in range(2):
            for i, (s, N, cell) in enumerate(mix):
                tickets.append((i, srv.submit(s, N, cell)))
        slots = set()
        for i, t in tickets:
            img, info = srv.wait(t, timeout_s=120)
            assert info["status"] == 0
            slots.add(info["slot"])
            assert O.rel_rms(img, alone[i]) < MIX_TOL, (i, O.rel_rms(img, alone[i]))
    assert len(slots) > 1  # requests ran concurrently in several slots


def test_injected_host_fault_is_isolated(alone, mix):
    with api.Server(num_slots=2, fault_every=3) as srv:
        tickets = [srv.submit(s, N, cell) for s, N, cell in mix]
        for k, t in enumerate(tickets):
            if t % 3 == 0:
                with pytest.raises(api.SvdiError) as ei:
                    srv.wait(t, timeout_s=120)
                assert ei.value.status == 7 and "injected" in ei.value.message
            else:
                img, info = srv.wait(t, timeout_s=120)
                assert O.rel_rms(img, alone[k]) < MIX_TOL


def test_admission_refuses_requests_beyond_the_budget(cuda_device, mix):
    s, N, cell = mix[0]
    with api.Server(num_slots=1, hbm_budget=16 << 20) as srv:
        with pytest.raises(api.SvdiError) as ei:
            srv.submit(s, N, cell)
        assert ei.value.status == 5 and "budget" in ei.value.message


def _estimate(s, N, planes=8):
    """The server's device-memory estimate of a request (server.cu request_bytes)."""
    G = int(np.ceil(1.5 * N)) + 8
    return s.num_samples * 54 + s.num_rows * 36 + planes * G * G * 8 + N * N * 4 + (64 << 20)


def test_tight_budget_counts_resident_buffers_and_drains(alone, mix):
    """Engines keep their buffers between requests, so a slot stays charged the largest request it
    has served. With a budget that holds the largest request once and a half, three slots can never
    hold two large requests' buffers at once: the charge never exceeds the budget, idle slots give
    their buffers back when nothing fits, and every request still completes with the same image."""
    big = max(_estimate(s, N) for s, N, _ in mix)
    budget = big * 3 // 2
    with api.Server(num_slots=3, hbm_budget=budget) as srv:
        tickets = [(i, srv.submit(s, N, cell)) for rep in range(2) for i, (s, N, cell) in enumerate(mix)]
        peak = 0
        for i, t in tickets:
            img, info = srv.wait(t, timeout_s=120)
            peak = max(peak, srv.stats()["hbm_in_use"])
            assert info["status"] == 0
            assert O.rel_rms(img, alone[i]) < MIX_TOL
        assert 0 < peak <= budget


def test_malformed_requests_are_refused(cuda_device, mix):
    s, N, cell = mix[0]
    with api.Server(num_slots=1) as srv:
        with pytest.raises(api.SvdiError):
            srv.submit(s, 0, cell)
        with pytest.raises(api.SvdiError):
            srv.submit(s, N, -1.0)


def test_poisson_stream_latencies(cuda_device, mix):
    """A Poisson stream at 50 requests/s of the mixed snapshots: every request completes and
    reports queueing/run/total latency; p50 <= p99."""
    rng = np.random.default_rng(3)
    lat = []
    with api.Server(num_slots=4) as srv:
        t0 = time.perf_counter()
        arrivals = np.cumsum(rng.exponential(1 / 50.0, 40))
        tickets = []
        for a in arrivals:
            while time.perf_counter() - t0 < a:
                time.sleep(0.0005)
            s, N, cell = mix[rng.integers(len(mix))]
            tickets.append(srv.submit(s, N, cell))
        for t in tickets:
            _, info = srv.wait(t, timeout_s=120)
            lat.append(info["latency_ms"])
    p50, p99 = np.percentile(lat, 50), np.percentile(lat, 99)
    print(f"serving: {len(lat)} requests at 50/s, p50 {p50:.2f} ms, p99 {p99:.2f} ms")
    assert 0 < p50 <= p99
