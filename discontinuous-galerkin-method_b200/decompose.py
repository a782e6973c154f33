"""One mesh split over several contexts (one per GPU): partition, ghost layers, halo exchange.

The reference's MPI driver (DG_leap_Frog_MPI.c:471-617) keeps every array on every rank, takes a
METIS element partition from a file (epart) and all-gathers the stresses and then the
velocities of every partition-boundary triangle to every rank, twice per step (:486-558).
Here each part is a mesh of its own: its triangles plus one layer of ghost triangles (the face
neighbours owned by other parts), built from the whole mesh's set-up arrays, and only the values
a neighbouring part needs travel, point to point:

* `partition` — recursive coordinate bisection of the triangle centroids into balanced parts
  (any owner array works, e.g. a METIS epart file through `read_epart`);
* `split` — the part meshes (dicts for `engine.Engine`) and the exchange plan: for every pair
  of parts the owned triangles one sends and the ghosts the other receives, in the same order.
  A part numbers its triangles boundary (owned, with a face neighbour in another part),
  interior (the other owned ones), ghosts; the owned classes each in Hilbert-curve order;
* `SplitRun` — steps all parts (velocity half, exchange of Vx/Vz, stress half, exchange of
  Txx/Tzz/Txz), either all parts in this process (`comm=None`, buffers copied on the device on a
  transfer stream) or one part per rank with `torch.distributed` point-to-point transfers (NCCL
  on GPUs).  By default each half step runs in two parts (`dg_gpu_half_step_part`): the
  interior triangles while the other half's halo is in transit, then, once the ghosts are
  unpacked, the boundary triangles, whose values are packed and sent at once.

Owned triangles compute exactly what the whole mesh computes (same inputs in the same order), so
fields and traces equal the undivided run bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import engine as eng

_PER_ELEMENT = ("A", "B", "absorb_fun", "Dx", "Dz", "Q")


def centroids(mesh: dict) -> np.ndarray:
    pts = np.asarray(mesh["Point"], dtype=np.float64).reshape(-1, 2)
    tri = np.asarray(mesh["Triangle"], dtype=np.int64).reshape(-1, 3) - 1
    return pts[tri].mean(axis=1)


def partition(mesh: dict, parts: int) -> np.ndarray:
    """Owner part of every triangle: recursive bisection of the centroids along the longer extent,
    split at the element count proportional to the parts on each side (sizes differ by <= 1)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    c = centroids(mesh)
    owner = np.zeros(len(c), dtype=np.int64)

    def rec(idx: np.ndarray, first: int, n: int) -> None:
        if n == 1:
            owner[idx] = first
            return
        left = n // 2
        ext = c[idx].max(axis=0) - c[idx].min(axis=0)
        axis = 0 if ext[0] >= ext[1] else 1
        order = idx[np.lexsort((idx, c[idx, axis]))]
        cut = (len(idx) * left) // n
        rec(order[:cut], first, left)
        rec(order[cut:], first + left, n - left)

    rec(np.arange(len(c)), 0, parts)
    return owner


def read_epart(path: str, K: int | None = None) -> np.ndarray:
    """Owner array from a METIS element-partition file (one 0-based part number per triangle,
    one per line, as the reference's MPI driver reads input_files/mesh/*.epart.N with
    epartinput, DG_leap_Frog_MPI.c:204-207)."""
    with open(path) as f:
        owner = np.array([int(t) for t in f.read().split()], dtype=np.int64)
    if K is not None and owner.size != K:
        raise ValueError("epart has %d entries for %d triangles" % (owner.size, K))
    if owner.size and owner.min() < 0:
        raise ValueError("negative part number in epart")
    return owner


@dataclass
class Part:
    """One part: the mesh dict for `engine.Engine` and the maps back to the whole mesh."""

    index: int
    mesh: dict
    own: np.ndarray            # whole-mesh ids of the owned triangles (local ids 0 .. n_own-1)
    ghost: np.ndarray          # whole-mesh ids of the ghosts (local ids n_own ..)
    receivers: np.ndarray      # whole-mesh receiver indices recorded by this part
    n_boundary: int = 0        # owned triangles with a ghost face neighbour (local ids 0 ..)
    send: dict = field(default_factory=dict)   # peer -> local ids sent to it (order of the buffer)
    recv: dict = field(default_factory=dict)   # peer -> local ids of ghosts received from it

    def send_list(self) -> np.ndarray:
        return np.concatenate([self.send[q] for q in sorted(self.send)] or [np.zeros(0, np.int64)])

    def recv_list(self) -> np.ndarray:
        return np.concatenate([self.recv[q] for q in sorted(self.recv)] or [np.zeros(0, np.int64)])


def hilbert_keys(xz: np.ndarray, bits: int = 16) -> np.ndarray:
    """Index along the Hilbert curve of points quantised to a 2^bits grid over their bounding
    square (the rotate-and-accumulate walk from the coarsest level down)."""
    xz = np.asarray(xz, dtype=np.float64).reshape(-1, 2)
    if xz.shape[0] == 0:
        return np.zeros(0, dtype=np.int64)
    n = 1 << bits
    lo = xz.min(axis=0)
    span = max(float((xz.max(axis=0) - lo).max()), 1e-300)
    x = np.minimum(n - 1, np.floor((xz[:, 0] - lo[0]) / span * (n - 1))).astype(np.int64)
    y = np.minimum(n - 1, np.floor((xz[:, 1] - lo[1]) / span * (n - 1))).astype(np.int64)
    d = np.zeros(x.size, dtype=np.int64)
    s = n >> 1
    while s > 0:
        rx = (x & s) > 0
        ry = (y & s) > 0
        d += s * s * ((3 * rx.astype(np.int64)) ^ ry.astype(np.int64))
        low = ~ry
        flip = low & rx
        x = np.where(flip, n - 1 - x, x)
        y = np.where(flip, n - 1 - y, y)
        x, y = np.where(low, y, x), np.where(low, x, y)
        s >>= 1
    return d


def _position(ids: np.ndarray, query: np.ndarray) -> np.ndarray:
    """Index within `ids` (distinct values, any order) of every value of `query`."""
    order = np.argsort(ids, kind="stable")
    return order[np.searchsorted(ids[order], query)]


def split(mesh: dict, owner: np.ndarray) -> list[Part]:
    """Part meshes with one ghost layer each, and the exchange plan between them."""
    owner = np.asarray(owner, dtype=np.int64)
    K = owner.size
    P = int(owner.max()) + 1
    nb = np.asarray(mesh["Neighbor"], dtype=np.int64).reshape(K, 3) - 1
    flag = np.asarray(mesh["Edge_flag"], dtype=np.int64).reshape(K, 3)
    nn = np.asarray(mesh["Node_Neighbor"], dtype=np.int64).reshape(K, 3, 3)
    tri = np.asarray(mesh["Triangle"], dtype=np.int64).reshape(K, 3)
    inner = flag == 1
    cen = centroids(mesh)
    parts = []
    for p in range(P):
        own = np.flatnonzero(owner == p)
        if own.size == 0:
            raise ValueError("part %d owns no triangle" % p)
        adj = nb[own][inner[own]]
        ghost = np.unique(adj[owner[adj] != p])
        # boundary triangles first, then the interior, each along the Hilbert curve
        is_b = (inner[own] & (owner[nb[own]] != p)).any(axis=1)
        key = hilbert_keys(cen[own])
        own = np.concatenate([own[is_b][np.argsort(key[is_b], kind="stable")],
                              own[~is_b][np.argsort(key[~is_b], kind="stable")]])
        n_boundary = int(is_b.sum())
        local = np.concatenate([own, ghost])
        g2l = np.full(K, -1, dtype=np.int64)
        g2l[local] = np.arange(local.size)
        lnb = g2l[nb[local]]
        lflag = flag[local].copy()
        cut = (lflag == 1) & (lnb < 0)          # a ghost's faces that lead out of the part
        lflag[cut] = 0
        lnb = np.where(lflag == 1, lnb, 0)      # outer faces point at triangle 1, like the reference
        m = dict(mesh)
        m["Triangle"] = tri[local].copy()
        m["Neighbor"] = lnb + 1
        m["Edge_flag"] = lflag
        m["Node_Neighbor"] = nn[local].copy()
        for n in _PER_ELEMENT:
            if n in mesh and mesh[n] is not None:
                m[n] = np.asarray(mesh[n]).reshape(K, -1)[local]
        # a shot whose source triangle another part owns gets a zero source vector here
        src = np.asarray(mesh["source"], dtype=np.int64).reshape(-1, 2).copy()
        fun = np.asarray(mesh["fun"], dtype=np.float64).reshape(-1, 6).copy()
        for s in range(src.shape[0]):
            g = src[s, 0] - 1
            if owner[g] == p:
                src[s, 0] = g2l[g] + 1
            else:
                src[s, 0] = 1
                fun[s] = 0.0
        m["source"], m["fun"] = src, fun
        rec = np.asarray(mesh["receiver"], dtype=np.int64).reshape(-1, 2)
        mine = np.flatnonzero(owner[rec[:, 0] - 1] == p)
        r = rec[mine].copy()
        r[:, 0] = g2l[r[:, 0] - 1] + 1
        m["receiver"] = r
        parts.append(Part(p, m, own, ghost, mine, n_boundary))
    # the plan: p sends to q its owned triangles that are ghosts of q, in whole-mesh id order
    for q in parts:
        by_owner = owner[q.ghost]
        for p in np.unique(by_owner):
            gids = q.ghost[by_owner == p]                    # sorted (ghost is sorted)
            q.recv[int(p)] = q.own.size + np.searchsorted(q.ghost, gids)
            parts[int(p)].send[q.index] = _position(parts[int(p)].own, gids)
    return parts


def slices(lists: dict, width: int) -> dict:
    """Peer -> (begin, end) of its values in a buffer holding `width` values per listed element,
    peers in increasing order."""
    out, at = {}, 0
    for q in sorted(lists):
        n = lists[q].size * width
        out[q] = (at, at + n)
        at += n
    return out


def start_exchange(comm, part: Part, send, recv, width: int) -> list:
    """Start this rank's halo transfer: to every peer its slice of `send`, from every peer into
    its slice of `recv` (tensors of `width` values per listed element), point to point with
    `torch.distributed` (NCCL between GPUs, gloo between CPU processes).  Returns the requests."""
    ops = []
    for q, (a, b) in slices(part.send, width).items():
        ops.append(comm.P2POp(comm.isend, send[a:b], q))
    for q, (a, b) in slices(part.recv, width).items():
        ops.append(comm.P2POp(comm.irecv, recv[a:b], q))
    return comm.batch_isend_irecv(ops) if ops else []


def exchange_ranks(comm, part: Part, send, recv, width: int) -> None:
    """This rank's halo transfer, started and waited for."""
    for r in start_exchange(comm, part, send, recv, width):
        r.wait()


class SplitRun:
    """Steps a mesh split into parts: every part in this process (`comm=None`: all contexts on
    `device`, halos copied between device buffers), or this rank's part only (`comm` = the
    `torch.distributed` module after `init_process_group`; rank r runs part r on `device`).
    `overlap`: run each half step in two parts so that the transfers overlap the interior
    triangles (False: whole half steps with the transfer in between; default: on between ranks,
    off for parts sharing one device, where the transfer is a device copy and the parts share
    the SMs: 2M triangles in 2 parts 0.215 against 0.212 ms/step, in 4 parts 0.383 against 0.349).
    Work is ordered across the contexts' streams and the transfer stream by CUDA events; the
    host does not wait inside `step`."""

    def __init__(self, mesh: dict, parts: int, precision: str = "fp64", *, owner=None, device: int = 0,
                 comm=None, overlap: bool | None = None, **engine_kw):
        import torch

        self.torch = torch
        self.comm = comm
        self.overlap = (comm is not None) if overlap is None else bool(overlap)
        self.pending = {}
        owner = partition(mesh, parts) if owner is None else np.asarray(owner)
        self.owner = owner
        self.parts = split(mesh, owner)
        self.K = owner.size
        self.R = np.asarray(mesh["receiver"]).reshape(-1, 2).shape[0]
        self.S = np.asarray(mesh["fun"]).reshape(-1, 6).shape[0]
        self.dtype = torch.float64 if precision in ("fp64", "fp64_ref") else torch.float32
        self.dev = torch.device("cuda", device)
        mine = range(len(self.parts)) if comm is None else [comm.get_rank()]
        self.engines = {}
        self.buf = {}
        self.streams = {}   # each context's stream (work is ordered across streams by events)
        self.packed = {}    # per part: its send buffer is packed
        self.moved = torch.cuda.Event()  # the transfer has landed
        # keep the part's numbering (boundary, interior, ghosts) inside the engine
        engine_kw.setdefault("reorder", False)
        self.xfer = torch.cuda.Stream(device=self.dev) if comm is None else None
        for p in mine:
            part = self.parts[p]
            e = eng.Engine(part.mesh, precision, device=device, wavefront=-1, **engine_kw)
            e.halo_lists(part.send_list(), part.recv_list())
            self.engines[p] = e
            self.streams[p] = e.stream()
            self.packed[p] = torch.cuda.Event()
            ns, nr = part.send_list().size, part.recv_list().size
            self.buf[p] = {w: (torch.empty(max(ns, 1) * pl * self.S, dtype=self.dtype, device=self.dev),
                               torch.empty(max(nr, 1) * pl * self.S, dtype=self.dtype, device=self.dev))
                           for w, pl in ((0, 12), (1, 18))}

    def close(self):
        for e in self.engines.values():
            e.close()
        self.engines = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _start(self, what: int):
        """Pack the send lists and start the transfer of one half's halo, ordered after the packs
        by events (no host synchronisation)."""
        width = (12 if what == 0 else 18) * self.S
        for p, e in self.engines.items():
            e.halo_pack(what, self.buf[p][what][0].data_ptr(), wait=False)
            self.packed[p].record(self.streams[p])
        if self.comm is None:
            for p in self.engines:
                self.xfer.wait_event(self.packed[p])
            with self.torch.cuda.stream(self.xfer):
                for p in self.engines:
                    for q, (a, b) in slices(self.parts[p].recv, width).items():
                        c, d = slices(self.parts[q].send, width)[p]
                        self.buf[p][what][1][a:b].copy_(self.buf[q][what][0][c:d])
            self.pending[what] = []
        else:
            (p,) = self.engines
            # NCCL's stream follows the current stream, which follows the pack
            self.torch.cuda.current_stream(self.dev).wait_event(self.packed[p])
            self.pending[what] = start_exchange(self.comm, self.parts[p], *self.buf[p][what], width)

    def _finish(self, what: int):
        """Unpack one half's halo into the ghosts once it has landed: the contexts' streams wait
        for the transfer (an event), then unpack ahead of their next launches.  The next pack of
        a buffer is therefore ordered after the transfer that read it, and the next transfer into
        a receive buffer after the unpack that read it."""
        if what not in self.pending:
            return
        for r in self.pending.pop(what):
            r.wait()      # NCCL: the current stream waits for the transfer
        src = self.xfer if self.comm is None else self.torch.cuda.current_stream(self.dev)
        self.moved.record(src)
        for p, e in self.engines.items():
            self.streams[p].wait_event(self.moved)
            e.halo_unpack(what, self.buf[p][what][1].data_ptr())

    def step(self, n: int = 1):
        engines = list(self.engines.values())
        if not self.overlap:
            for _ in range(int(n)):
                for e in engines:
                    e.half_step(0)
                self._start(0)
                self._finish(0)
                for e in engines:
                    e.half_step(1)
                self._start(1)
                self._finish(1)
            return
        interior, boundary = eng.PART_INTERIOR, eng.PART_BOUNDARY
        for _ in range(int(n)):
            for e in engines:                 # needs no ghost: overlaps the stress halo
                e.half_step_part(0, interior)
            self._finish(1)
            for e in engines:
                e.half_step_part(0, boundary)
            self._start(0)
            for e in engines:                 # overlaps the velocity halo
                e.half_step_part(1, interior)
            self._finish(0)
            for e in engines:
                e.half_step_part(1, boundary)
            self._start(1)
        self._finish(1)

    def fetch(self, what: str, shot: int = 0) -> np.ndarray:
        """A field ([K][Np], whole-mesh order) from the parts this process runs (other
        triangles are zero when `comm` is set)."""
        out = np.zeros((self.K, 6))
        for p, e in self.engines.items():
            part = self.parts[p]
            out[part.own] = e.fetch(what, 0, shot).reshape(-1, 6)[: part.own.size]
        return out

    def traces(self, comp: str = "trace_z", shot: int = 0) -> np.ndarray:
        """[steps][R] traces in the whole mesh's receiver order (receivers of other ranks zero)."""
        cols = {}
        steps = 0
        for p, e in self.engines.items():
            if self.parts[p].receivers.size:
                tr = e.fetch(comp, 0, shot)
                steps = tr.shape[0]
                cols[p] = tr
        out = np.zeros((steps, self.R))
        for p, tr in cols.items():
            out[:, self.parts[p].receivers] = tr
        return out
