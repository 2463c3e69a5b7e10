"""Replica plumbing for multi-GPU runs.

Snapshots are independent, so N GPUs run N independent replicas of the imager (one process per
GPU) with no data-path collective. The only cross-rank traffic is timing: every rank times its own
steps with CUDA events between barriers, and the job's time is the maximum over ranks.
"""
from __future__ import annotations

import os
from datetime import timedelta


def init_from_env(backend: str = "nccl", timeout_s: float = 120.0):
    """(rank, world_size, local_rank, dist or None) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    if backend == "nccl":
        import torch
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return rank, ws, local, dist


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world_size: int, seconds_max: float) -> float:
    """Whole-job throughput: units processed by all ranks over the slowest rank's time."""
    return world_size * units_per_rank / seconds_max


def bind_host_to_gpu(device: int = 0) -> list:
    """Restrict this process's CPUs to those NVML reports as closest to GPU `device` (its NUMA
    node), so that pinned host buffers allocated afterwards live next to the GPU's PCIe root and
    host<->device copies do not cross the socket interconnect. Only this process's affinity
    changes; nothing of the GPU. Returns the CPUs bound to ([] when NVML or the affinity call is
    not available, in which case nothing changes)."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(int(device))
            n_words = (os.cpu_count() + 63) // 64
            mask = pynvml.nvmlDeviceGetCpuAffinity(h, n_words)
        finally:
            pynvml.nvmlShutdown()
        cpus = [64 * w + b for w, m in enumerate(mask) for b in range(64) if (int(m) >> b) & 1]
        cpus = [c for c in cpus if c < os.cpu_count()]
        if cpus and hasattr(os, "sched_setaffinity"):
            allowed = os.sched_getaffinity(0)
            chosen = [c for c in cpus if c in allowed]
            if chosen:
                os.sched_setaffinity(0, chosen)
                return chosen
    except Exception:
        pass
    return []
