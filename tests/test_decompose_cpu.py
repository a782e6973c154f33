"""A mesh split into parts (domain decomposition), checked on the CPU.

The partition, the ghost layers and the exchange plan of `decompose.split` are checked for their
invariants; then the parts run on the CPU oracle, half step by half step, with the ghost values
exchanged in numpy between the halves exactly as `decompose.SplitRun` exchanges them between
contexts, and every owned triangle's fields and every receiver's trace must equal the
undivided oracle run bit for bit.
"""
import numpy as np
import pytest

from conftest import pkg

import oracle

dec = pkg.decompose
FIELDS = ("Vx", "Vz", "Txx", "Tzz", "Txz")


@pytest.fixture(scope="module")
def whole():
    w = pkg.workloads.small_square(n_cells=14, steps=120, shots=2)
    s = pkg.host.build_setup(w, full=True)
    return s, pkg.engine.mesh_from_setup(s)


@pytest.mark.parametrize("P", [2, 3, 5])
def test_partition_and_plan_invariants(whole, P):
    s, mesh = whole
    owner = dec.partition(mesh, P)
    K = s.K
    sizes = np.bincount(owner, minlength=P)
    assert sizes.sum() == K and sizes.max() - sizes.min() <= 2
    parts = dec.split(mesh, owner)
    nb = np.asarray(mesh["Neighbor"]).reshape(K, 3) - 1
    flag = np.asarray(mesh["Edge_flag"]).reshape(K, 3)
    for p in parts:
        local = np.concatenate([p.own, p.ghost])
        # the ghosts are exactly the face neighbours of owned triangles held by other parts
        adj = nb[p.own][flag[p.own] == 1]
        assert np.array_equal(p.ghost, np.unique(adj[owner[adj] != p.index]))
        # owned triangles keep every face and neighbour of the whole mesh
        lnb = np.asarray(p.mesh["Neighbor"]).reshape(-1, 3) - 1
        lfl = np.asarray(p.mesh["Edge_flag"]).reshape(-1, 3)
        n_own = p.own.size
        assert np.array_equal(lfl[:n_own], flag[p.own])
        inner = flag[p.own] == 1
        assert np.array_equal(local[lnb[:n_own]][inner], nb[p.own][inner])
        # what p sends to q is, in the same order, what q receives from p
        for q, ids in p.send.items():
            assert np.array_equal(p.own[ids], parts[q].ghost[parts[q].recv[p.index] - parts[q].own.size])
    assert sorted(np.concatenate([p.receivers for p in parts]).tolist()) == list(range(s.n_rec))


@pytest.mark.parametrize("P", [2, 4])
def test_split_run_on_the_oracle_equals_the_whole_mesh(whole, P):
    s, mesh = whole
    steps = 100
    parts = dec.split(mesh, dec.partition(mesh, P))
    for shot in (0, 1):
        o = oracle.Oracle(mesh, s.dt, s.K)
        rx, rz = o.run(shot, steps, threads=1)
        want = [f.reshape(-1, 6) for f in o.fields]

        ors = [oracle.Oracle(p.mesh, s.dt, p.own.size + p.ghost.size) for p in parts]
        for q in ors:
            q.reset()
        gx = np.zeros((steps, s.n_rec))
        gz = np.zeros((steps, s.n_rec))

        def exchange(planes):
            for p in parts:
                for q, ghost_ids in p.recv.items():
                    src = parts[q].send[p.index]
                    for f in planes:
                        dst = ors[p.index].fields[f].reshape(-1, 6)
                        dst[ghost_ids] = ors[q].fields[f].reshape(-1, 6)[src]

        for t in range(steps):
            for q in ors:
                q.half(shot, t, 0)
            exchange((0, 1))
            for p, q in zip(parts, ors):
                bx = np.zeros(p.receivers.size)
                bz = np.zeros(p.receivers.size)
                q.half(shot, t, 1, bx, bz)
                gx[t, p.receivers] = bx
                gz[t, p.receivers] = bz
            exchange((2, 3, 4))
        for p, q in zip(parts, ors):
            for k in range(5):
                assert np.array_equal(q.fields[k].reshape(-1, 6)[: p.own.size], want[k][p.own]), (shot, k)
        assert np.array_equal(gx, rx) and np.array_equal(gz, rz)
        assert np.abs(rz).max() > 0


def _rank_worker(rank, world, port, out):
    import datetime
    import os
    import sys

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from conftest import pkg as P
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    w = P.workloads.small_square(n_cells=10, steps=5)
    mesh = P.engine.mesh_from_setup(P.host.build_setup(w, full=False), with_ref_ops=False)
    parts = P.decompose.split(mesh, P.decompose.partition(mesh, world))
    me = parts[rank]
    width = 12 * 2  # 12 planes x 2 shots
    send_ids = me.own[me.send_list()]
    send = torch.tensor(np.repeat(send_ids * 1000.0, width) + np.tile(np.arange(width), send_ids.size),
                        dtype=torch.float64)
    recv = torch.full((me.recv_list().size * width,), -1.0, dtype=torch.float64)
    P.decompose.exchange_ranks(dist, me, send, recv, width)
    ghost_ids = np.concatenate([me.own, me.ghost])[me.recv_list()]
    want = np.repeat(ghost_ids * 1000.0, width) + np.tile(np.arange(width), ghost_ids.size)
    out[rank] = bool(np.array_equal(recv.numpy(), want)) and ghost_ids.size > 0
    dist.barrier()
    dist.destroy_process_group()


def test_halo_transfer_between_gloo_ranks():
    """The point-to-point transfer SplitRun uses between ranks (NCCL on GPUs) delivers every
    ghost's values from its owner, into the right slot, with three CPU ranks over gloo."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    world = 3
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()  # a server process started by spawn, not fork
    out = mgr.dict()
    procs = [ctx.Process(target=_rank_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    assert all(out[r] for r in range(world))


def test_epart_file_round_trip(whole, tmp_path):
    """A partition written as a METIS epart file reads back as the same owner array, and a split
    built from it passes the plan checks."""
    s, mesh = whole
    owner = dec.partition(mesh, 3)
    path = str(tmp_path / "model.epart.3")
    pkg.meshgen.write_epart(path, s.K, owner)
    back = dec.read_epart(path, s.K)
    assert np.array_equal(back, owner)
    parts = dec.split(mesh, back)
    assert sum(p.own.size for p in parts) == s.K
    with pytest.raises(ValueError):
        dec.read_epart(path, s.K + 1)
