"""The benchmark's multi-rank logic on CPU: two gloo ranks, no GPU.

Each rank owns an independent 64-shot batch (sources shifted per rank); the whole-job value is
every rank's DOF-updates over the slowest rank's time, combined with one MAX all-reduce; the
reference arm runs on rank 0 only.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank), "DG_BENCH_BACKEND": "gloo"})
    r, wsz, local, dist = bench.dist_setup(None)
    assert (r, wsz, local) == (rank, world, rank) and dist.get_backend() == "gloo"
    local_ms = 10.0 * (rank + 1)
    value, t_max = bench.weak_scaling_value(1000.0, 5, local_ms, world, dist, "cpu")
    w = bench.WORKLOADS["multishot"][0](10, rank)
    out[rank] = (value, t_max, float(w.src[0, 0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_weak_scaling_and_distinct_shots():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()  # a server process started by spawn, not fork
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    v0, t0, x0 = out[0]
    v1, t1, x1 = out[1]
    assert t0 == t1 == 20.0                       # max over ranks
    assert v0 == v1 == pytest.approx(2 * 1000.0 * 5 / 0.020)
    assert x0 != x1                               # each rank advances its own shot set


def test_reference_arm_is_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.argparse.Namespace(gpus=2, steps=1, warmup=3, impl="reference", workload="square",
                                    no_cpu_baseline=False)
    assert bench.run_reference_arm(args) == 0     # returns before any work on a non-zero rank
    import torch.distributed as dist
    assert not dist.is_initialized()              # and joins no process group
