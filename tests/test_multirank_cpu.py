"""The benchmark's multi-rank logic on CPU: two gloo ranks, no GPU.

The ranks share one job, as `bench.py --gpus N` runs it: the multi-shot job (64 shots per rank)
is cut into contiguous shot ranges by sharding.shard_shots, the uneven batch's meshes go to ranks
by cost (sharding.shard_meshes); the whole-job value is all ranks' DOF-updates over the slowest
rank's time (a SUM and a MAX all-reduce); every rank's traces reach rank 0 in one gather
(sharding.gather_traces); the reference arm runs on rank 0 only.
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
    import numpy as np

    import bench
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank), "DG_BENCH_BACKEND": "gloo"})
    r, wsz, local, dist = bench.dist_setup(None)
    assert (r, wsz, local) == (rank, world, rank) and dist.get_backend() == "gloo"
    # this rank's share of the multi-shot job and of the uneven batch
    ctor, _, share = bench.WORKLOADS["multishot"]
    (w,) = ctor(10, rank, world)
    ctor_u, _, share_u = bench.WORKLOADS["uneven"]
    mine = ctor_u(10, rank, world)
    # whole-job value: the ranks' different shares over the slowest rank's time
    dof = float(w.dof_per_step() + 1000 * rank)
    local_ms = 10.0 * (rank + 1)
    value, t_max = bench.job_value(dof, 5, local_ms, dist, "cpu")
    # the e2e gather: rank r's traces (shots x 2 x steps x receivers) on rank 0
    traces = np.full((w.shots, 2, 3, 4), float(rank)) + np.arange(24).reshape(2, 3, 4)
    got = bench.gather_job(dist, traces, None)
    out[rank] = (share, share_u, w.src.tolist(), [x.K for x in mine], [x.shots for x in mine], value, t_max,
                 None if got is None else [g.tolist() for g in got])
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_share_one_job():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()  # a server process started by spawn, not fork
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    pkg = bench.pkg()
    r0, r1 = out[0], out[1]
    assert r0[0] == "weak" and r0[1] == "strong"
    # the shot ranges: 64 contiguous shots each, together the job's 128 sources in order
    job = pkg.workloads.layered_multishot(steps=10, shots=128)
    assert len(r0[2]) == len(r1[2]) == 64
    assert np.array_equal(np.array(r0[2] + r1[2]), job.src)
    # the meshes: disjoint, together the 48 of the batch, loads within the costliest mesh
    ws, _ = pkg.workloads.uneven_batch(n_meshes=48, seed=5)
    assert sorted(r0[3] + r1[3]) == sorted(x.K for x in ws) and len(r0[3]) + len(r1[3]) == 48
    cost = [sum(k * s for k, s in zip(r[3], r[4])) for r in (r0, r1)]
    assert abs(cost[0] - cost[1]) <= max(x.K * x.shots for x in ws)
    # value: both ranks' work over the slowest time (MAX 20 ms)
    w0 = 30 * job.K * 64
    assert r0[6] == r1[6] == 20.0
    assert r0[5] == r1[5] == pytest.approx((w0 + w0 + 1000.0) * 5 / 0.020)
    # the gather: rank 0 holds both ranks' traces in rank order, rank 1 nothing
    assert r1[7] is None and len(r0[7]) == 2
    base = np.arange(24).reshape(2, 3, 4)
    for k in range(2):
        assert np.array_equal(np.array(r0[7][k]), np.full((64, 2, 3, 4), float(k)) + base)


def test_reference_arm_is_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.argparse.Namespace(gpus=2, steps=1, warmup=3, impl="reference", workload="square",
                                    no_cpu_baseline=False, variant=0)
    assert bench.run_reference_arm(args) == 0     # returns before any work on a non-zero rank
    import torch.distributed as dist
    assert not dist.is_initialized()              # and joins no process group
