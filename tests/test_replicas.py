"""Multi-process replica plumbing on CPU (gloo, world_size 2): the timing reduction bench.py uses
for N > 1 GPUs, and failure detection when a rank leaves before a collective (host-side: the
survivor's next collective ends with an error after a short process-group timeout)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker_max(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from svdimager_b200 import replicas
    r, ws, _, dist = replicas.init_from_env("gloo", timeout_s=30)
    v = replicas.max_over_ranks(10.0 * (r + 1), dist)
    out.put((r, v, replicas.aggregate_rate(5, ws, v)))
    dist.barrier()
    dist.destroy_process_group()


def _worker_leaves(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from svdimager_b200 import replicas
    r, ws, _, dist = replicas.init_from_env("gloo", timeout_s=3)
    replicas.max_over_ranks(1.0, dist)  # step 1 completes on both ranks
    if r == 1:
        out.put((1, "left"))
        out.close()
        out.join_thread()
        os._exit(0)  # leaves between steps, nothing in flight
    try:
        replicas.max_over_ranks(2.0, dist)
        out.put((0, "no error"))
    except Exception as ex:  # the survivor learns of it through the collective's timeout / error
        out.put((0, type(ex).__name__))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_worker_max, args=(_free_port(), q), nprocs=2, start_method="spawn")
    res = sorted(q.get(timeout=60) for _ in range(2))
    assert res[0][1] == res[1][1] == 20.0
    assert res[0][2] == pytest.approx(2 * 5 / 20.0)


def test_rank_leaving_is_detected_by_the_survivor():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_leaves, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=90)
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[1] == "left"
    assert res[0] != "no error"


def test_bind_host_to_gpu_with_a_fake_nvml(monkeypatch):
    """The host-side NUMA binding reads the GPU's CPU mask from NVML and restricts this process's
    affinity to it (nothing of the GPU changes); without NVML it leaves the affinity alone."""
    import os
    import sys
    import types
    from svdimager_b200 import replicas
    before = os.sched_getaffinity(0)
    cpu0 = min(before)
    fake = types.SimpleNamespace(
        nvmlInit=lambda: None, nvmlShutdown=lambda: None,
        nvmlDeviceGetHandleByIndex=lambda i: i,
        nvmlDeviceGetCpuAffinity=lambda h, n: [1 << cpu0] + [0] * (n - 1))
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    try:
        assert replicas.bind_host_to_gpu(0) == [cpu0]
        assert os.sched_getaffinity(0) == {cpu0}
    finally:
        os.sched_setaffinity(0, before)
    monkeypatch.setitem(sys.modules, "pynvml", None)  # import fails: nothing changes
    assert replicas.bind_host_to_gpu(0) == []
    assert os.sched_getaffinity(0) == before
