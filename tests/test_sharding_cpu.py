"""Shots and meshes of one job over several ranks (sharding.py), checked on CPU: the partitions'
invariants and balance, and the trace gather between three gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import pkg

sh = pkg.sharding
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("n,world", [(64, 1), (64, 8), (5, 8), (229, 3), (0, 2)])
def test_shot_ranges_cover_every_shot_once(n, world):
    rs = sh.shard_shots(n, world)
    assert len(rs) == world
    assert [s for r in rs for s in r] == list(range(n))
    sizes = [len(r) for r in rs]
    assert max(sizes) - min(sizes) <= 1


def test_mesh_partition_by_cost_is_balanced():
    rng = np.random.default_rng(3)
    K = np.exp(rng.uniform(np.log(5000), np.log(500000), size=48))
    S = rng.integers(1, 9, size=48)
    steps = np.ceil(1.5 / (0.2 / np.sqrt(K)))           # finer meshes take more steps
    costs = [sh.mesh_cost(int(k), int(s), int(t)) for k, s, t in zip(K, S, steps)]
    for world in (1, 2, 4, 8):
        parts = sh.shard_meshes(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(48))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
        if world > 1:   # far better than a split by mesh index
            naive = [sum(costs[i] for i in range(48) if i * world // 48 == r) for r in range(world)]
            assert max(loads) <= max(naive)
    assert sh.shard_meshes([3.0, 3.0, 2.0, 2.0, 2.0], 2) == [[0, 2, 4], [1, 3]]


def _gather_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from conftest import pkg as P
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    shots = P.sharding.shard_shots(7, world)[rank]
    # this rank's traces: [its shots][steps][receivers], values that name shot, step and receiver
    local = np.array([[[1000.0 * s + 10.0 * t + r for r in range(3)] for t in range(4)] for s in shots])
    got = P.sharding.gather_traces(dist, local.reshape(len(shots), 4, 3), root=0)
    if rank == 0:
        whole = np.concatenate(got, axis=0)
        want = np.array([[[1000.0 * s + 10.0 * t + r for r in range(3)] for t in range(4)] for s in range(7)])
        out[rank] = bool(np.array_equal(whole, want)) and [g.shape[0] for g in got] == [len(r) for r in
                                                                                         P.sharding.shard_shots(7, world)]
    else:
        out[rank] = got is None
    dist.barrier()
    dist.destroy_process_group()


def test_trace_gather_between_gloo_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    world = 3
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()  # a server process started by spawn, not fork
    out = mgr.dict()
    procs = [ctx.Process(target=_gather_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    assert all(out[r] for r in range(world))


def _nccl_worker(port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    from conftest import pkg as P
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": "0", "WORLD_SIZE": "1"})
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    local = np.arange(2 * 5 * 3, dtype=np.float64).reshape(2, 5, 3)
    got = P.sharding.gather_traces(dist, local, root=0, device=torch.device("cuda", 0))
    out[0] = len(got) == 1 and bool(np.array_equal(got[0], local))
    dist.destroy_process_group()


@pytest.mark.gpu
def test_trace_gather_over_nccl_single_rank():
    """The gather with CUDA tensors over NCCL (one rank: all this pool's calls have one GPU)."""
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    p = ctx.Process(target=_nccl_worker, args=(port, out))
    p.start()
    p.join(180)
    assert p.exitcode == 0 and out[0]
