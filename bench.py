"""Benchmark of the snapshot imaging path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config precision]

Workload (default): the precision configuration -- 512 stations, 130,816 baselines x 64 channels =
8,372,224 visibilities, one snapshot, 2048^2 image, cell 5e-5 rad; synthetic seeded data
(svdimager_b200.synth). A step images one snapshot from its raw Measurement-Set arrays (float UVW,
frequencies, polarisations 0/3, flags, WEIGHT_SPECTRUM): FP64 SVD rotation, flag/weight collapse,
tile binning, gridding, cuFFT, Chebyshev recombination, grid correction, reprojection.

`value` is snapshots/s with the inputs resident in HBM (device API; --lanes engines on their own
streams take the snapshots in turn, so consecutive snapshots overlap); `e2e` is the same through the
streaming host API (server: three resident engines, four snapshots in flight) with pinned host
buffers, host->device upload and device->host image read inside every step; `e2e.sync` is one
blocking host call per snapshot. The inputs (219 MB) exceed the 126 MB L2, so no flush is needed
between steps.

Multi-GPU: replicas only -- every rank images its own snapshot stream on its own GPU; no data-path
collective. value = snapshots of all ranks / max over ranks of the timed region.

--impl reference: the reference algorithm's CPU restatement (oracle: collapse, rotation, ES
gridding, FFT, recombination, reprojection; the same Chebyshev rule as this arm) on all host cores,
rank 0, one whole snapshot per step.
Its line also carries `reference_binary`: the reference's own GPU imager (archive FIpipe, compiled
from its source for sm_100a) timed per call on the same snapshot; our arm's `fipipe` key times our
FIpipe on the same inputs.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "snapshots/s at 2048^2, 8.4M vis, <=1e-5 rel RMS vs FP64 DFT; p50/p99 latency"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(1.0)  # nvidia-smi's start-up (driver queries) finishes before the timed region
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    from svdimager_b200 import replicas
    return replicas.init_from_env("nccl", timeout_s=120)


def serving_phase(api, big, n_requests, rate, device, seed=5, gridder=0):
    """Poisson stream (rate/s) of mixed requests through a 4-slot server: the 512-station
    headline snapshot at 2048^2, a 256-station 32-channel snapshot at 1024^2 and a 128-station
    16-channel snapshot at 512^2. Returns latency percentiles and sustained throughput."""
    from svdimager_b200 import synth
    mix = [(big, big.image_size, big.cell_size),
           (synth.make_snapshot("batching", nchan=32, flag_fraction_rows=0.0, flag_fraction_samples=0.15,
                                snapshot_index=7), 1024, 1e-4),
           (synth.make_snapshot("small", snapshot_index=8), 512, 2e-4)]
    import torch
    for s, _, _ in mix:  # host arrays in pinned memory, as a correlator's receive buffers would be
        for k, v in s.arrays().items():
            setattr(s, k, torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy())
    rng = np.random.default_rng(seed)
    lat, queue, run = [], [], []
    with api.Server(num_slots=4, device=device, edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET,
                    target_error=1e-6, gridder=gridder) as srv:
        for s, N, cell in mix:  # warm every slot's plans and buffers
            for t in [srv.submit(s, N, cell) for _ in range(4)]:
                srv.wait(t, 120)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
        t0 = time.perf_counter()
        tickets = []
        for a in arrivals:
            while time.perf_counter() - t0 < a:
                time.sleep(0.0002)
            s, N, cell = mix[int(rng.integers(len(mix)))]
            tickets.append(srv.submit(s, N, cell))
        for t in tickets:
            _, info = srv.wait(t, 120)
            lat.append(info["latency_ms"])
            queue.append(info["queue_ms"])
            run.append(info["run_ms"])
        wall = time.perf_counter() - t0
    return {"requests": n_requests, "offered_rate_per_s": rate, "slots": 4,
            "mix": "512 st x 64 ch @2048^2, 256 st x 32 ch @1024^2, 128 st x 16 ch @512^2",
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "queue_p99_ms": round(float(np.percentile(queue, 99)), 3),
            "run_p50_ms": round(float(np.percentile(run, 50)), 3),
            "sustained_snapshots_per_s": round(n_requests / wall, 2)}


GRIDDER_DTYPE = {"tc": "f16 hi+lo operands, f32 accumulation", "tc_bf16": "bf16 hi+lo operands, f32 accumulation",
                 "tc_i8": "u8 x s8 operands (22-bit fixed point as three byte digits), s32 accumulation"}
GRIDDER_LABEL = {"tc": "tcgen05 split-precision (FP16 hi+lo)", "tc_bf16": "tcgen05 split-precision (BF16 hi+lo)",
                 "tc_i8": "tcgen05 exact integer (kind::i8, three byte digits)"}


def algorithmic_bytes(n_samples, n_rows, n_chan, planes, G, N):
    """Algorithmic bytes of one snapshot: 26 B per sample (two polarisations complex64, two flag
    bytes, two weights), 24 B per row (FP64 uvw), 8 B per channel, 32 B per moment-plane cell (one
    grid write, one FFT read, one FFT write, one recombination read) and 4 B per image pixel."""
    return 26 * n_samples + 24 * n_rows + 8 * n_chan + 32 * planes * G * G + 4 * N * N


def grid_kernel_bytes(n_gridded, planes, G):
    """Algorithmic bytes of the gridding stage: one 16 B record read per gridded sample and one
    8 B write per moment-plane cell."""
    return 16 * n_gridded + 8 * planes * G * G


def batching_phase(api, local, n_snapshots=256, launches=3, seed_offset=0):
    """Configuration B: n snapshots of the 256-station layout (hour angles over +-3 h, 16/32/64
    channels, 0-40 % sample flags) imaged at 1024^2, cell 1e-4 rad, from one CUDA graph per batch.
    The autotuner picks the options on three representative snapshots; the same batch is also
    timed with the default options. Returns the batch figures."""
    import torch
    from svdimager_b200 import autotune, synth
    t_gen = time.perf_counter()
    snaps = synth.batching_stream(n_snapshots, seed_offset=seed_offset)
    t_gen = time.perf_counter() - t_gen
    dev = torch.device("cuda", local)
    keep, descs = [], []
    for sn in snaps:
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in sn.arrays().items()}
        keep.append(t)
        descs.append(api.device_ms(sn.num_rows, sn.num_channels, t, sn.array_center_x))
    N, cell = 1024, 1e-4
    nvis = np.array([sn.num_samples for sn in snaps])
    order = np.argsort(nvis)
    reps = [descs[i] for i in (order[0], order[len(order) // 2], order[-1])]
    scratch = torch.zeros((N, N), dtype=torch.float32, device=dev)
    t_tune = time.perf_counter()
    best, trials = autotune.tune(reps, N, cell, scratch, device=local, repeats=3)
    t_tune = time.perf_counter() - t_tune
    chosen = [t for t in trials if all(t.options[k] == best[k] for k in ("support", "sigma", "gridder", "tile"))][0]
    imgs = torch.zeros((n_snapshots, N, N), dtype=torch.float32, device=dev)
    # an explicit stream: the graphs are launched on it and the events recorded on it (a null
    # stream would launch them on the engine's own stream, outside the timed events)
    stream = torch.cuda.Stream(dev)
    out = {"snapshots": n_snapshots, "image": f"{N}^2, cell {cell} rad", "total_vis": int(nvis.sum()),
           "vis_per_snapshot": [int(nvis.min()), int(nvis.max())], "generation_s": round(t_gen, 1),
           "autotune": {"seconds": round(t_tune, 2), "candidates": len(trials),
                        "chosen": {"gridder": "tc" if best["gridder"] == api.GRIDDER_TC else "fp32",
                                   "tile": best["tile"], "support": best["support"], "sigma": best["sigma"],
                                   "beta": round(best["beta"], 4),
                                   "chebyshev_terms": sorted(set(chosen.num_terms)),
                                   "w_slabs": sorted(set(chosen.num_slabs)),
                                   "rel_rms_vs_fp64_dft": chosen.error, "ms_per_snapshot": round(chosen.ms, 4)}}}
    for name, opts in (("tuned", best), ("default", dict(device=local, edge_mode=api.EDGE_STRICT,
                                                          k_rule=api.KRULE_TARGET, target_error=1e-6))):
        e = api.Engine(**opts)
        t_cap = time.perf_counter()
        b = api.Batch(e, descs, N, cell, imgs.data_ptr())
        t_cap = time.perf_counter() - t_cap
        b.launch(stream.cuda_stream)
        b.check()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # an NVTX range names the timed launches for a kernel-level profile (ncu --nvtx)
        torch.cuda.nvtx.range_push(f"config_b_{name}")
        for _ in range(launches):
            b.launch(stream.cuda_stream)
        torch.cuda.nvtx.range_pop()
        e1.record(stream)
        b.check()
        ms = e0.elapsed_time(e1) / launches
        out[name] = {"ms_per_batch": round(ms, 3), "snapshots_per_s": round(n_snapshots / (ms * 1e-3), 1),
                     "vis_per_s": round(float(nvis.sum()) / (ms * 1e-3), 1), "graph_launches_per_batch": 1,
                     "plan_and_capture_s": round(t_cap, 2)}
        b.close()
        e.close()
    # the same 256 snapshots as two batches (alternate snapshots) on two engines whose launches run
    # on their own streams at the same time (each batch of 128 is itself two halves)
    halves = [descs[0::2], descs[1::2]]
    engines = [api.Engine(**best) for _ in halves]
    himgs = [torch.zeros((len(h), N, N), dtype=torch.float32, device=dev) for h in halves]
    batches = [api.Batch(e, h, N, cell, im.data_ptr()) for e, h, im in zip(engines, halves, himgs)]
    streams = [torch.cuda.Stream(dev) for _ in halves]
    for b, st_ in zip(batches, streams):
        b.launch(st_.cuda_stream)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for st_ in streams:
        st_.wait_event(e0)
    for _ in range(launches):
        for b, st_ in zip(batches, streams):
            b.launch(st_.cuda_stream)
    for st_ in streams:
        stream.wait_stream(st_)
    e1.record(stream)
    for b in batches:
        b.check()
    ms = e0.elapsed_time(e1) / launches
    out["tuned_two_streams"] = {"ms_per_batch": round(ms, 3), "snapshots_per_s": round(n_snapshots / (ms * 1e-3), 1),
                                "vis_per_s": round(float(nvis.sum()) / (ms * 1e-3), 1),
                                "graph_launches_per_batch": len(batches)}
    for b, e in zip(batches, engines):
        b.close()
        e.close()
    return out


def widefield_phase(api, local, npix=256):
    """Configuration W: the 512-station layout at 30 deg elevation, 64 channels, 4096^2 image over
    a 0.3 rad field. ES support W and the Chebyshev error target are swept; each point reports the
    device time, the moment planes used and the relative RMS error of the rotated-frame image
    against the library's FP64 direct DFT at random pixels."""
    import torch
    from svdimager_b200 import synth
    sn = synth.make_snapshot("widefield")
    dev = torch.device("cuda", local)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in sn.arrays().items()}
    d = api.device_ms(sn.num_rows, sn.num_channels, t, sn.array_center_x)
    N, cell = sn.image_size, sn.cell_size
    img = torch.zeros((N, N), dtype=torch.float32, device=dev)
    rng = np.random.default_rng(5)
    px, py = rng.integers(0, N, npix), rng.integers(0, N, npix)
    from svdimager_b200 import autotune

    def point(W, tgt, gridder=api.GRIDDER_FP32):
        opts = dict(device=local, edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET, target_error=tgt,
                    support=W, sigma=1.5, beta=autotune.es_beta(W, 1.5), gridder=gridder)
        with api.Engine(presplat=1, **opts) as e:
            e.image_device(d, N, cell, img.data_ptr())
            R = img.cpu().numpy()
            ref = e.dft_pixels(px, py)
            m = np.isfinite(ref)
            err = float(np.sqrt(np.sum((R[py, px][m] - ref[m]) ** 2) / np.sum(ref[m] ** 2)))
        with api.Engine(**opts) as e:
            e.image_device(d, N, cell, img.data_ptr())
            ms, ms_grid = [], []
            for _ in range(3):
                e.image_device(d, N, cell, img.data_ptr())
                ms.append(e.stats()["ms_total"])
                ms_grid.append(e.stats()["ms_grid"])
            st = e.stats()
        return {"support": W, "cheb_target": tgt, "w_slabs": st["num_slabs"],
                "chebyshev_terms": st["num_terms"], "planes": st["num_planes"],
                "ms": round(float(np.median(ms)), 3), "ms_gridding": round(float(np.median(ms_grid)), 3),
                "tensor_core": bool(st["used_tc"]), "rel_rms_vs_fp64_dft": err}

    points = [point(W, tgt) for W in (6, 8, 10, 12) for tgt in (1e-5, 1e-6, 1e-7)]
    ok = [p for p in points if p["rel_rms_vs_fp64_dft"] <= 1e-5]
    best = min(ok, key=lambda p: p["ms"]) if ok else None
    # the exact integer tensor-core gridder on the same snapshot (one launch per Chebyshev term)
    tc = point(8, 1e-6, api.GRIDDER_TC_I8)
    tc["gridder"] = "tc_i8 (u8 x s8 digits, int32 accumulate; one launch per Chebyshev term)"
    return {"workload": f"widefield: {sn.num_rows} baselines x {sn.num_channels} channels = {sn.num_samples} vis, "
                        f"{N}^2 image, cell {cell:.3e} rad (0.3 rad field), 30 deg elevation",
            "pixels": npix, "sweep": points, "fastest_within_1e-5": best, "tensor_core": tc}


def archive_quartet(snap, eng, api):
    """The archive entry's inputs for `snap` (`FIpipe`, pipe_interface.cpp:8): collapsed
    visibilities, rotated baselines Bin [N_s][3] (float) and Vin (float), taken from the engine's
    own preprocessing of the snapshot, in pageable host memory as the archive CLI passes them."""
    with api.Engine(device=eng.options.device) as e:
        e.image(snap)
        vr, vi = e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG)
        q, s = e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S)
        vin = np.array(e.stats()["vin"], np.float64).reshape(3, 3)
    b = (s[:, None, None] * q[None, :, :]).reshape(-1, 3).astype(np.float32)   # idx = row + chan * rows
    return vr.copy(), vi.copy(), np.ascontiguousarray(b), vin.astype(np.float32)


def fipipe_phase(api, eng, snap, steps):
    """Our `FIpipe` (archive semantics: one slab, smallest Chebyshev order within 1e-2) on the
    snapshot's quartet, host buffers in and out, wall clock per call: the same call and inputs as
    the reference binary's timing in the reference arm."""
    vr, vi, b, v = archive_quartet(snap, eng, api)
    N, cell = snap.image_size, snap.cell_size
    with api.Engine(api.archive_options(device=eng.options.device)) as e:
        for _ in range(2):
            e.fipipe(vr, vi, b, v, N, cell)
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            e.fipipe(vr, vi, b, v, N, cell)
            ts.append(time.perf_counter() - t0)
        st = e.stats()
    return {"snapshots_per_s": round(1.0 / float(np.median(ts)), 3),
            "ms_p50": round(float(np.median(ts)) * 1e3, 3), "ms_p99": round(float(np.percentile(ts, 99)) * 1e3, 3),
            "chebyshev_terms": st["num_terms"], "calls": steps,
            "h2d_bytes_per_call": int(vr.nbytes + vi.nbytes + b.nbytes + v.nbytes), "d2h_bytes_per_call": N * N * 4,
            "what": "FIpipe(Visreal, Visimag, Bin, Vin, dirty, N_s, N, cell) from pageable host buffers, wall clock"}


def e2e_stream(api, opts, psnap, N, cell, steps, warmup, dist, dev, slots=3, window=4):
    """End to end through the streaming API: `steps` snapshots submitted to a server with `slots`
    resident engines, at most `window` in flight (a correlator client that hands over the next
    snapshot when a receive buffer frees up). Every request uploads its inputs from pinned host
    memory and reads its image back into a pinned host image; the upload of one request overlaps
    the imaging of another. Timed from the first submit to the last completion."""
    import torch
    outs = [torch.zeros((N, N), dtype=torch.float32).pin_memory().numpy() for _ in range(window)]
    lat = []
    with api.Server(num_slots=slots, **opts) as srv:
        for i in range(max(warmup, slots)):
            srv.wait(srv.submit(psnap, N, cell, out=outs[i % window]), 120)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        inflight = []
        for i in range(steps):
            if len(inflight) == window:
                _, info = srv.wait(inflight.pop(0), 120)
                lat.append(info["latency_ms"])
            inflight.append(srv.submit(psnap, N, cell, out=outs[i % window]))
        for t in inflight:
            _, info = srv.wait(t, 120)
            lat.append(info["latency_ms"])
        sec = time.perf_counter() - t0
    from svdimager_b200 import replicas
    return {"seconds": replicas.max_over_ranks(sec, dist, dev), "slots": slots, "window": window,
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3)}}


def make_workload(config, rank):
    from svdimager_b200 import synth
    return synth.make_snapshot(config, snapshot_index=rank)


def run_ours(args):
    import torch
    from svdimager_b200 import api
    rank, ws, local, dist = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from svdimager_b200 import replicas
    host_cpus = replicas.bind_host_to_gpu(local)  # pinned buffers on the GPU's NUMA node
    snap = make_workload(args.config, rank)
    N, cell = snap.image_size, snap.cell_size
    gridder = {"tc": api.GRIDDER_TC, "tc_bf16": api.GRIDDER_TC_BF16, "tc_i8": api.GRIDDER_TC_I8}.get(
        args.gridder, api.GRIDDER_FP32)
    opts = dict(device=local, edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET, target_error=1e-6,
                gridder=gridder)
    eng = api.Engine(**opts)
    # device-resident inputs
    host = {k: np.ascontiguousarray(v) for k, v in snap.arrays().items()}
    dten = {k: torch.from_numpy(v).to(dev) for k, v in host.items()}
    dms = api.device_ms(snap.num_rows, snap.num_channels, dten, snap.array_center_x)
    out = torch.zeros((N, N), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    # throughput pipelines: engines on their own streams take the snapshots in turn, so one
    # snapshot's FFT and recombination overlap the next one's binning (engine 0 is `eng`)
    lanes = [(eng, torch.cuda.Stream(dev), out)]
    for _ in range(1, max(1, args.lanes)):
        lanes.append((api.Engine(**opts), torch.cuda.Stream(dev), torch.zeros((N, N), dtype=torch.float32, device=dev)))

    def step():
        eng.image_device(dms, N, cell, out.data_ptr(), sp)

    def lane_step(i):
        e_, s_, o_ = lanes[i % len(lanes)]
        e_.image_device(dms, N, cell, o_.data_ptr(), s_.cuda_stream)

    for i in range(max(args.warmup, len(lanes))):
        lane_step(i)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    st = eng.stats()
    lat = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    n_launch0 = api.kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stage = {"ms_preprocess": [], "ms_bin": [], "ms_grid": [], "ms_fft": [], "ms_image": []}
    # throughput: snapshots submitted back to back over the pipelines (the host enqueues the next
    # snapshot while the device images the previous ones); the events bracket every pipeline
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _, s_, _ in lanes:
            s_.wait_event(ev0)
        for i in range(args.steps):
            lane_step(i)
        for _, s_, _ in lanes:
            stream.wait_stream(s_)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    launches = api.kernel_launch_count() - n_launch0
    # latency and per-stage device times: one snapshot at a time
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize(dev)
        lat.append((time.perf_counter() - t0) * 1e3)
        s2 = eng.stats()
        for k in stage:
            stage[k].append(s2[k])
    from svdimager_b200 import replicas
    ms_total = replicas.max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    ms_step = ms_total / args.steps
    value = replicas.aggregate_rate(args.steps, ws, ms_total / 1e3)

    # end-to-end through the host API (pinned host buffers, upload + image read per step)
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in host.items()}
    from types import SimpleNamespace
    psnap = SimpleNamespace(num_rows=snap.num_rows, num_channels=snap.num_channels,
                            array_center_x=snap.array_center_x, image_size=N, cell_size=cell,
                            **{k: v.numpy() for k, v in pinned.items()})
    himg = torch.zeros((N, N), dtype=torch.float32).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        eng.image(psnap, out=himg)
    if dist:
        dist.barrier()
    e2e_lat = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t1 = time.perf_counter()
        eng.image(psnap, out=himg)
        e2e_lat.append((time.perf_counter() - t1) * 1e3)
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e_sync_value = replicas.aggregate_rate(args.steps, ws, e2e_s)
    # streaming through the server: the next snapshot uploads while the previous one images
    # at least 64 requests: with 4 in flight, the window's fill and drain (about two snapshot
    # latencies) stay under a tenth of the timed region also for short --steps runs
    e2e_requests = max(args.steps, 64)
    stream_out = e2e_stream(api, opts, psnap, N, cell, e2e_requests, args.warmup, dist, dev)
    e2e_value = replicas.aggregate_rate(e2e_requests, ws, stream_out["seconds"])
    serving = None if args.no_serving else serving_phase(api, snap, args.serving_requests, 50.0, local,
                                                         gridder=gridder)
    batching = None if args.no_batching else batching_phase(api, local, args.batch_snapshots,
                                                             seed_offset=rank)
    widefield = None if args.no_widefield else widefield_phase(api, local)
    fipipe = None if args.no_fipipe else fipipe_phase(api, eng, snap, max(3, min(args.steps, 10)))
    h2d =int(sum(v.nbytes for v in host.values()))
    d2h = int(N * N * 4)

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    G = st["grid_size"]
    planes = st["num_planes"]
    peak, peak_kind = peaks()
    stage_ms = {k: float(np.median(v)) for k, v in stage.items()}
    # dominant kernel stage of ours (cuFFT is a library call and reported beside it)
    ours = {k: v for k, v in stage_ms.items() if k != "ms_fft"}
    dom = max(ours, key=ours.get)
    if dom == "ms_grid":
        alg = grid_kernel_bytes(st["num_gridded"], planes, G)
        name = (("k_grid_i8" if args.gridder == "tc_i8" else "k_grid_tc") if st["used_tc"] else "k_grid_fp32") \
            + " (+ plane zeroing)"
    elif dom == "ms_bin":
        alg = (26 + 8) * snap.num_samples + 16 * st["num_gridded"]
        name = "k_histogram_sep + k_scan + k_scatter_sep"
    elif dom == "ms_preprocess":
        alg = 26 * snap.num_samples + 8 * snap.num_samples + 36 * snap.num_rows
        name = "k_collapse + rotation"
    else:
        alg = 8 * planes * N * N + 4 * N * N
        name = "k_recombine"
    achieved = alg / (stage_ms[dom] * 1e-3) / 1e9
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of each gridder on
    # this workload, from one-launch ncu --set full captures (fourth imaging call of this bench with
    # --lanes 1 --steps 2 --warmup 3)
    traffic = None
    if dom == "ms_grid" and args.config == "precision":
        traffic = {"k_grid_fp32": 223104512, "k_grid_tc": 225017856, "k_grid_i8": 224812288}.get(name.split()[0])

    cpu = cpu_baseline(snap, eng, api, st, args) if not args.no_cpu else None
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "snapshots/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": GRIDDER_DTYPE[args.gridder] if st["used_tc"] else "f32",
        "data": "synthetic (seeded; 512-station layout, 220-source sky, noise, flags, weights)",
        "config": {
            "workload": f"{args.config}: {snap.num_rows} baselines x {snap.num_channels} channels = "
                        f"{snap.num_samples} vis, one snapshot, {N}^2 image, cell {cell} rad",
            "gridder": GRIDDER_LABEL[args.gridder] if st["used_tc"] else "fp32 fixed-point",
            "grid": G, "planes": planes, "num_slabs": st["num_slabs"], "chebyshev_terms": st["num_terms"],
            "support": 8, "beta": 15.3704324328, "oversampling": 1.5, "tile": st["tile"],
            "k_rule": "target 1e-6", "edges": "strict (samples whose footprint leaves the grid are dropped)",
            "gridded_samples": st["num_gridded"],
            "l2": "inputs 219 MB > 126 MB L2, no flush", "parallelism": f"replicas x{ws}",
            "pipelines": f"{len(lanes)} engines on their own streams, snapshots in turn",
        },
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 4),
                       "p99": round(float(np.percentile(lat, 99)), 4)},
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "e2e": {"value": round(e2e_value, 3), "unit": "snapshots/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "h2d_gbs": round(h2d * e2e_value / ws / 1e9, 2),
                "host_cpus": f"{len(host_cpus)} CPUs of the GPU's NUMA node" if host_cpus else "unbound",
                "api": f"svdi_server submit/wait, {stream_out['slots']} slots, {stream_out['window']} requests "
                       "in flight, pinned host inputs and output images",
                "requests": e2e_requests,
                "latency_ms": stream_out["latency_ms"],
                "sync": {"value": round(e2e_sync_value, 3), "api": "svdi_engine_image_host, one blocking call per step",
                         "latency_ms": {"p50": round(float(np.percentile(e2e_lat, 50)), 3),
                                        "p99": round(float(np.percentile(e2e_lat, 99)), 3)}}},
        "roofline": {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_kind": peak_kind,
                     "limiter": ("warp-instruction issue: the gridder is a shared-memory reduction of 64 "
                                 "cells per sample, its DRAM traffic is small" if dom == "ms_grid" else None),
                     "snapshot_alg_bytes": algorithmic_bytes(snap.num_samples, snap.num_rows,
                                                             snap.num_channels, planes, G, N),
                     "snapshot_frac": round(algorithmic_bytes(snap.num_samples, snap.num_rows,
                                                              snap.num_channels, planes, G, N)
                                            / (ms_step * 1e-3) / 1e9 / peak, 4)},
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    if serving:
        line["serving"] = serving
    if batching:
        line["batching"] = batching
    if widefield:
        line["widefield"] = widefield
    if fipipe:
        line["fipipe"] = fipipe
    if cpu:
        line["cpu_baseline"] = cpu["baseline"]
        line["accuracy"] = cpu["accuracy"]
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(snap, eng, api, st, args):
    """FP64 direct DFT (oracle) on the host cores at a bounded random pixel sample of the same
    snapshot; the same pixels of the device image before reprojection give the accuracy."""
    from oracle import oracle as O
    N, cell = snap.image_size, snap.cell_size
    with api.Engine(device=eng.options.device, edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET,
                    target_error=1e-6, presplat=1, gridder=eng.options.gridder) as e2:
        R = e2.image(snap)
        vr, vi = e2.buffer(api.BUF_VIS_REAL), e2.buffer(api.BUF_VIS_IMAG)
        q, sv = e2.buffer(api.BUF_Q).reshape(-1, 3), e2.buffer(api.BUF_S)
        st2 = e2.stats()
        # the same image against the library's device FP64 direct DFT at 10,000 random pixels
        rng_p = np.random.default_rng(20261203)
        gx, gy = rng_p.integers(0, N, 10000), rng_p.integers(0, N, 10000)
        try:
            probe = e2.dft_pixels(gx, gy)
            pm = np.isfinite(probe)
            diff = R[gy, gx][pm].astype(np.float64) - probe[pm]
            acc_10k = {"pixels": int(pm.sum()),
                       "rel_rms_vs_fp64_dft": float(np.sqrt(np.sum(diff ** 2) / np.sum(probe[pm] ** 2))),
                       "peak_rel_vs_fp64_dft": float(np.max(np.abs(diff)) / np.max(np.abs(probe[pm]))),
                       "reference": "device FP64 direct DFT (svdi_engine_dft_pixels) of the kept samples"}
        except Exception as ex:  # a supplementary figure: its failure must not cost the bench line
            acc_10k = {"error": f"{type(ex).__name__}: {ex}"}
    vin = np.array(st2["vin"]).reshape(3, 3)
    G = st2["grid_size"]
    r = O.expand_coords(q, sv)
    inc = O.inclusion_mask(r, float(np.float32(cell)) * G, G, edge_mode=1)
    inv_det = 1 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    rng = np.random.default_rng(12345)
    npix = args.cpu_pixels
    px, py = rng.integers(0, N, npix), rng.integers(0, N, npix)
    t0 = time.perf_counter()
    d = O.dft_pixels_sep(q, sv, vr, vi, inv_det, snap.num_samples, vin, N, float(np.float32(cell)), px, py, inc)
    dt = time.perf_counter() - t0
    valid = np.isfinite(d)
    err = O.rel_rms(R[py, px][valid], d[valid])
    peak_err = float(np.max(np.abs(R[py, px][valid] - d[valid])) / np.max(np.abs(d[valid])))
    cores = O.lib().orc_num_threads()
    per_pix = dt / npix
    snaps_per_s = 1.0 / (per_pix * st2["valid_pixels"])
    return {
        "baseline": {"value": snaps_per_s, "unit": "snapshots/s", "cores": cores, "kind": "port",
                     "sample": f"FP64 direct DFT of all {snap.num_samples} samples at {npix} random "
                               f"pixels in {dt:.2f} s, extrapolated to {st2['valid_pixels']} pixels"},
        "accuracy": {"rel_rms_vs_fp64_dft": err, "peak_rel_vs_fp64_dft": peak_err, "pixels": int(valid.sum()),
                     "device_dft_10k": acc_10k,
                     "image": "rotated-frame image before reprojection (strict edges)"},
    }


def reference_binary_phase(O, snap, calls):
    """The reference's own GPU imager, its archive `FIpipe` (archive/FIPkernels.cu:679-911,
    compiled unmodified for sm_100a into oracle/_ref), on the snapshot's full quartet from
    pageable host buffers: wall clock per call (its allocations, uploads, host Chebyshev selection,
    cuFFT plan, kernels, download, frees) and its own "Time elapsed" line (FIPkernels.cu:888,
    plan + kernels). Its stdout is captured so that the JSON line stays the only output."""
    fn = O.load_reference_fipipe()
    if fn is None:
        return {"unavailable": "reference library not built (make -C oracle ref)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
    except ImportError:
        return {"unavailable": "torch missing"}
    vr, vi = O.collapse(snap)
    vin, q, sv, _ = O.preprocess64(snap)
    b = np.ascontiguousarray(O.expand_coords(q, sv).astype(np.float32))
    v = np.ascontiguousarray(vin.astype(np.float32).reshape(-1))
    N, cell = snap.image_size, snap.cell_size
    out = np.zeros(N * N, np.float32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    walls = []
    with tempfile.TemporaryFile(mode="w+b") as cap:
        sys.stdout.flush()
        saved = os.dup(1)
        os.dup2(cap.fileno(), 1)
        try:
            for i in range(calls + 1):   # the first call warms the CUDA context and cuFFT
                t0 = time.perf_counter()
                fn(ptr(vr), ptr(vi), ptr(b), ptr(v), ptr(out), vr.shape[0], N, float(cell))
                if i:
                    walls.append(time.perf_counter() - t0)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        cap.seek(0)
        text = cap.read().decode(errors="replace")
    elapsed = [float(m) for m in re.findall(r"Time elapsed: ([0-9.eE+-]+) ms", text)][1:]
    terms = re.findall(r"selected kept terms\s*=\s*(\d+)", text)
    return {"snapshots_per_s": round(1.0 / float(np.median(walls)), 3),
            "ms_p50": round(float(np.median(walls)) * 1e3, 3),
            "ms_self_timed_p50": round(float(np.median(elapsed)), 3) if elapsed else None,
            "chebyshev_terms": int(terms[-1]) if terms else None, "calls": calls,
            "image_nonzero": bool(np.any(out != 0)),
            "what": "reference archive FIpipe (archive/FIPkernels.cu, nvcc -O3 --use_fast_math -maxrregcount=64, "
                    "sm_100a) from pageable host buffers, wall clock; ms_self_timed = its own "
                    "'Time elapsed' (cuFFT plan + kernels)"}


def _row_slice(snap, rows):
    """The first `rows` baseline rows of a snapshot, all channels (idx = row + chan * R)."""
    import dataclasses
    R, C = snap.num_rows, snap.num_channels
    cut = lambda a: np.ascontiguousarray(a.reshape(C, R)[:, :rows].reshape(-1))
    return dataclasses.replace(
        snap, num_rows=rows, uvw=np.ascontiguousarray(snap.uvw[:rows]),
        vis0_real=cut(snap.vis0_real), vis0_imag=cut(snap.vis0_imag), vis3_real=cut(snap.vis3_real),
        vis3_imag=cut(snap.vis3_imag), flag0=cut(snap.flag0), flag3=cut(snap.flag3),
        weight0=cut(snap.weight0), weight3=cut(snap.weight3),
        uvw64=None if snap.uvw64 is None else snap.uvw64[:rows])


def reference_pipeline(O, snap, frac, target_error):
    """One step of the reference algorithm on the host cores (oracle port of SII:635-853 and
    SII:1498-1761, FP64): collapse, SVD rotation, w statistics, slab/Chebyshev selection, ES
    gridding, unnormalised inverse FFT, Chebyshev recombination with grid correction, SIN
    reprojection. frac = 1 images the whole snapshot. frac < 1 runs the same fraction of every
    stage: the snapshot passed in holds that fraction of the rows, the FFT transforms that fraction
    of the plane rows and columns, and recombination and reprojection cover that fraction of the
    image rows. Returns (seconds per stage, slab configuration)."""
    N, cell = snap.image_size, float(np.float32(snap.cell_size))
    t = [time.perf_counter()]
    vr, vi = O.collapse(snap)
    vin, q, sv, _ = O.preprocess64(snap)
    r = O.expand_coords(q, sv)
    t.append(time.perf_counter())
    sc = (O.slab_config_target(r[:, 2], vin, N, cell, target_error) if target_error
          else O.slab_config_sii(r[:, 2], vin, N, cell))
    G = O.grid_size_for(N)
    inv_det = 1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    t.append(time.perf_counter())
    planes = O.grid(r, vr, vi, cell * G, G, sc, inv_det, edge_mode=1)
    t.append(time.perf_counter())
    if frac >= 1.0:
        moments = O.inverse_fft(planes)
    else:
        import scipy.fft
        gf = max(1, int(round(frac * G)))
        planes[:, :gf, :] = scipy.fft.ifft(planes[:, :gf, :], axis=-1, workers=-1)
        planes[:, :, :gf] = scipy.fft.ifft(planes[:, :, :gf], axis=-2, workers=-1)
        moments = planes
    t.append(time.perf_counter())
    rows = (0, N if frac >= 1.0 else max(1, int(round(frac * N))))
    phi = O.es_correction(N, G)
    R = O.recombine(moments, N, cell, vin, sc, phi, snap.num_samples, rows=rows)
    O.reproject(R, N, cell, vin, "sii", rows=rows)
    t.append(time.perf_counter())
    return np.diff(t), sc


def run_reference(args):
    """The reference algorithm on the host cores, rank 0 only: every timed step images one whole
    snapshot of the workload from host memory with the oracle's CPU restatement of the reference
    path (reference_pipeline) on all host threads, with the same Chebyshev rule as this repo's arm
    (error target 1e-6; --ref-bucket-k: the reference's own bucket rule). When the requested steps
    at one snapshot each would take longer than --ref-budget seconds, every step runs the same
    fraction of each stage instead and the rate is that fraction over the step time. The line also
    carries `reference_binary`: the reference's own GPU imager (archive FIpipe, compiled from its
    source for sm_100a) timed per call on the same snapshot."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from svdimager_b200 import synth
    snap = synth.make_snapshot(args.config)
    N, cell = snap.image_size, snap.cell_size
    target = None if args.ref_bucket_k else 1e-6
    # one untimed whole snapshot sizes the steps
    sec_full = float(np.sum(reference_pipeline(O, snap, 1.0, target)[0]))
    frac = min(1.0, args.ref_budget / max(1e-9, sec_full * (args.steps + args.warmup - 1)))
    work = snap if frac >= 1.0 else _row_slice(snap, max(16, int(round(frac * snap.num_rows))))
    if frac < 1.0:
        frac = work.num_rows / snap.num_rows
    for _ in range(args.warmup - 1):
        reference_pipeline(O, work, frac, target)
    stages, ts, sc = [], [], None
    for _ in range(args.steps):
        st, sc = reference_pipeline(O, work, frac, target)
        stages.append(st)
        ts.append(float(np.sum(st)))
    sec = float(np.mean(ts))
    value = frac / sec
    stage_ms = dict(zip(("collapse_rotation", "w_statistics_and_k", "gridding", "fft", "recombine_reproject"),
                        [round(float(x) * 1e3, 2) for x in np.mean(stages, axis=0)]))
    what = ("whole snapshot per step" if frac >= 1.0 else
            f"{frac:.4f} of every stage per step ({work.num_rows} of {snap.num_rows} rows x "
            f"{snap.num_channels} channels, the same fraction of the FFT rows/columns and image rows)")
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "snapshots/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.config}: {snap.num_samples} vis, {N}^2, cell {cell}",
                   "k_rule": "bucket (reference)" if args.ref_bucket_k else "target 1e-6 (as this repo's arm)",
                   "chebyshev_terms": sc.K, "num_slabs": sc.num_slabs, "grid": O.grid_size_for(N),
                   "edges": "strict", "whole_snapshot_s": round(sec_full, 3)},
        "stages_ms": stage_ms,
        "cpu_baseline": {"value": value, "unit": "snapshots/s", "cores": O.lib().orc_num_threads(),
                         "kind": "port",
                         "sample": f"reference algorithm (oracle port, FP64, all host threads): {what}, "
                                   f"from host memory"},
        "e2e": {"value": value, "unit": "snapshots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_binary:
        line["reference_binary"] = reference_binary_phase(O, snap, max(1, min(args.steps, 3)))
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="precision")
    ap.add_argument("--cpu-pixels", type=int, default=3000,
                    help="pixels of the FP64 direct-DFT CPU baseline (about 10 s on 16 host cores)")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="reference arm: seconds of host work the steps may take at most")
    ap.add_argument("--ref-bucket-k", action="store_true",
                    help="reference arm: the reference's bucket Chebyshev rule instead of this repo's target rule")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=150)
    ap.add_argument("--no-batching", action="store_true")
    ap.add_argument("--no-widefield", action="store_true")
    ap.add_argument("--batch-snapshots", type=int, default=256)
    ap.add_argument("--lanes", type=int, default=3,
                    help="engines (each on its own stream) taking the snapshots in turn in the throughput loop")
    ap.add_argument("--no-fipipe", action="store_true", help="skip the archive-entry (FIpipe) timing")
    ap.add_argument("--no-ref-binary", action="store_true",
                    help="reference arm: skip timing the reference's own GPU imager")
    ap.add_argument("--gridder", default="fp32", choices=["tc", "tc_bf16", "tc_i8", "fp32"],
                    help="tc: split-precision tcgen05 gridder (FP16 hi+lo); tc_bf16: the same with BF16 hi+lo; "
                         "tc_i8: exact integer tcgen05 gridder (three byte digits, int32 sums); "
                         "fp32: CUDA-core fixed-point gridder")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
