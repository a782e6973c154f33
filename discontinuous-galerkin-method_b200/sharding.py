"""Shots and meshes of one job spread over several GPUs (one rank each), and the final trace gather.

Shots of a mesh and meshes of a batch are independent: nothing is exchanged while they step, so
a job is cut into per-rank work and the receiver traces are collected once at the end (the
reference runs the shots of a mesh one after the other, DG_leap_Frog_OpenMP.c:397, and the
meshes as separate runs).

* `shard_shots` — contiguous, balanced shot ranges of one mesh;
* `shard_meshes` — meshes to ranks by estimated cost K * shots * steps (longest first, each to
  the least loaded rank), so the slowest rank carries as little as the costs allow;
* `gather_traces` — every rank's traces into rank 0's buffers with one `torch.distributed`
  gather of a padded block (NCCL between GPUs, gloo between CPU processes).
"""
from __future__ import annotations

import numpy as np


def shard_shots(n_shots: int, world: int) -> list[range]:
    """Shot ranges for ranks 0..world-1: contiguous, sizes differing by at most one."""
    if n_shots < 0 or world < 1:
        raise ValueError("need n_shots >= 0 and world >= 1")
    return [range(n_shots * r // world, n_shots * (r + 1) // world) for r in range(world)]


def mesh_cost(K: int, shots: int, steps: int) -> float:
    """Estimated work of one mesh: element-shot updates over its steps."""
    return float(K) * float(shots) * float(steps)


def shard_meshes(costs, world: int) -> list[list[int]]:
    """Mesh indices for each rank: meshes taken from the most to the least costly (ties by
    index), each given to the rank with the least cost so far (ties to the lower rank).  The
    largest load is at most the ideal share plus the costliest mesh."""
    costs = [float(c) for c in costs]
    if world < 1 or any(c < 0 for c in costs):
        raise ValueError("need world >= 1 and non-negative costs")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def gather_traces(comm, local: np.ndarray, root: int = 0, device=None):
    """Gather every rank's float64 array `local` (any shape, first axis = this rank's items, e.g.
    shots) on `root`: returns the list of the ranks' arrays there and None elsewhere.  Sizes and
    trailing shapes travel first (a small gather), then one gather of blocks padded to the
    largest; `device` is where the tensors live (a CUDA device for NCCL, None for CPU/gloo)."""
    import torch

    world, rank = comm.get_world_size(), comm.get_rank()
    local = np.ascontiguousarray(local, dtype=np.float64)
    shape = np.zeros(8, dtype=np.int64)
    if local.ndim > 7:
        raise ValueError("at most 7 dimensions")
    shape[0] = local.ndim
    shape[1:1 + local.ndim] = local.shape
    meta = torch.from_numpy(shape).to(device)
    metas = [torch.zeros_like(meta) for _ in range(world)] if rank == root else None
    comm.gather(meta, metas, dst=root)
    sizes = torch.tensor([local.size], dtype=torch.int64, device=device)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    comm.all_gather(all_sizes, sizes)
    width = max(1, max(int(s.item()) for s in all_sizes))
    block = torch.zeros(width, dtype=torch.float64, device=device)
    block[:local.size] = torch.from_numpy(local.ravel()).to(device)
    blocks = [torch.zeros_like(block) for _ in range(world)] if rank == root else None
    comm.gather(block, blocks, dst=root)
    if rank != root:
        return None
    out = []
    for m, b in zip(metas, blocks):
        m = m.cpu().numpy()
        shp = tuple(int(x) for x in m[1:1 + int(m[0])])
        n = int(np.prod(shp)) if shp else 1
        out.append(b[:n].cpu().numpy().reshape(shp))
    return out
