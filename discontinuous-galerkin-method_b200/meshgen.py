"""Synthetic triangle meshes in the converted Triangle format the DG host code reads.

The reference builds its meshes offline: ``triangle -pqanA`` followed by a MATLAB conversion
that pads the header rows and writes every value with ``save -ascii``
(input_files/mesh/create_mesh_file.m:5-49).  Neither Triangle nor MATLAB is available, so this
module produces meshes of the same kind directly:

* ``jittered_grid``   — a structured grid of cells split into two triangles each, interior
  vertices jittered by a seeded uniform offset (the homogeneous and layered configurations);
* ``delaunay``        — a seeded Delaunay triangulation of jittered points clipped to a domain
  with a curved top (the slope/topography configurations);
* ``read_poly`` / ``from_poly`` — a ``.poly`` planar straight-line graph (input_files/mesh/*.poly)
  triangulated with its segments as mesh edges, regional attributes and holes;
* ``write_converted`` — the ``.ele/.node/.neigh`` triple with the padded header row and the
  ``%16.7e`` MATLAB ``-ascii`` number format that ReadInt/ReadDouble parse
  (fun_save_to_file.c:22-204), 1-based indices, ``-1`` for "no neighbour".

Conventions follow Triangle's: vertices of each triangle counter-clockwise, neighbour ``k``
of a triangle is the one across the edge opposite its vertex ``k`` (fun_DG.c:576-578 rotates
this into the edge-ordered ``Neighbor`` array).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class Mesh:
    points: np.ndarray   # (P, 2) float64, x and z coordinates
    tris: np.ndarray     # (K, 3) int64, 0-based vertex ids, counter-clockwise
    neigh: np.ndarray    # (K, 3) int64, 0-based neighbour opposite vertex k, -1 = none
    attr: np.ndarray     # (K,) int64 region attribute (1-based like Triangle's -A)
    markers: np.ndarray  # (P,) int64 boundary marker (1 on the outer boundary)

    @property
    def K(self) -> int:
        return int(self.tris.shape[0])

    @property
    def P(self) -> int:
        return int(self.points.shape[0])

    def centroids(self) -> np.ndarray:
        return self.points[self.tris].mean(axis=1)


def compute_neighbors(tris: np.ndarray) -> np.ndarray:
    """Neighbour across the edge opposite each local vertex (-1 on the outer boundary)."""
    K = tris.shape[0]
    # edge opposite vertex k joins vertices (k+1)%3 and (k+2)%3
    a = np.concatenate([tris[:, 1], tris[:, 2], tris[:, 0]])
    b = np.concatenate([tris[:, 2], tris[:, 0], tris[:, 1]])
    owner = np.concatenate([np.arange(K)] * 3)
    slot = np.repeat(np.arange(3), K)
    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    key = lo * (int(tris.max()) + 1) + hi
    order = np.argsort(key, kind="stable")
    ks = key[order]
    neigh = np.full((K, 3), -1, dtype=np.int64)
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    if same.size and np.any(np.diff(same) == 1):
        raise ValueError("non-manifold edge: more than two triangles share an edge")
    i0 = order[same]
    i1 = order[same + 1]
    neigh[owner[i0], slot[i0]] = owner[i1]
    neigh[owner[i1], slot[i1]] = owner[i0]
    return neigh


def _orient_ccw(points: np.ndarray, tris: np.ndarray) -> np.ndarray:
    p = points[tris]
    cross = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - \
            (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])
    tris = tris.copy()
    cw = cross < 0
    tris[cw, 1], tris[cw, 2] = tris[cw, 2].copy(), tris[cw, 1].copy()
    return tris


def _rotate(tris: np.ndarray, rng: np.random.Generator | None) -> np.ndarray:
    """Cyclically rotate each triangle's vertex list (keeps orientation).

    Triangle does not promise which vertex comes first; rotating exercises every face/edge
    pairing of the neighbour-matching code (fun_DG.c:557-739, 1195-1276).
    """
    if rng is None:
        return tris
    r = rng.integers(0, 3, size=tris.shape[0])
    idx = (np.arange(3)[None, :] + r[:, None]) % 3
    return np.take_along_axis(tris, idx, axis=1)


def _boundary_markers(P: int, tris: np.ndarray, neigh: np.ndarray) -> np.ndarray:
    markers = np.zeros(P, dtype=np.int64)
    t, k = np.nonzero(neigh < 0)
    for off in (1, 2):
        markers[tris[t, (k + off) % 3]] = 1
    return markers


def jittered_grid(nx: int, nz: int, width: float, height: float, *, jitter: float = 0.1,
                  seed: int = 0, pinned=(), diagonal: str = "random", rotate: bool = True,
                  attr_fn=None) -> Mesh:
    """``nx`` x ``nz`` cells on [0,width] x [0,height], two triangles per cell.

    Interior vertices move by U(-jitter*h, +jitter*h) in x and z (``default_rng(seed)``);
    boundary vertices and the ``pinned`` (x, z) vertices stay on the lattice so sources and
    receivers can be snapped to a vertex as Get_Source/Get_Receiver require (fun_DG.c:304,380).
    """
    rng = np.random.default_rng(seed)
    hx = width / nx
    hz = height / nz
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(nz + 1), indexing="xy")
    x = ii.astype(np.float64) * hx
    z = jj.astype(np.float64) * hz
    dx = rng.uniform(-jitter * hx, jitter * hx, size=x.shape)
    dz = rng.uniform(-jitter * hz, jitter * hz, size=z.shape)
    interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < nz)
    for (px, pz) in pinned:
        interior &= ~((np.abs(x - px) < 1e-9) & (np.abs(z - pz) < 1e-9))
    x = np.where(interior, x + dx, x)
    z = np.where(interior, z + dz, z)
    points = np.stack([x.ravel(), z.ravel()], axis=1)

    vid = lambda i, j: j * (nx + 1) + i  # noqa: E731
    ci, cj = np.meshgrid(np.arange(nx), np.arange(nz), indexing="xy")
    ci = ci.ravel()
    cj = cj.ravel()
    a = vid(ci, cj)
    b = vid(ci + 1, cj)
    c = vid(ci + 1, cj + 1)
    d = vid(ci, cj + 1)
    if diagonal == "random":
        flip = rng.integers(0, 2, size=a.shape[0]).astype(bool)
    elif diagonal == "alternate":
        flip = ((ci + cj) % 2).astype(bool)
    else:
        flip = np.zeros(a.shape[0], dtype=bool)
    t1 = np.where(flip[:, None], np.stack([a, b, d], 1), np.stack([a, b, c], 1))
    t2 = np.where(flip[:, None], np.stack([b, c, d], 1), np.stack([a, c, d], 1))
    tris = np.empty((2 * a.shape[0], 3), dtype=np.int64)
    tris[0::2] = t1
    tris[1::2] = t2
    tris = _orient_ccw(points, tris)
    tris = _rotate(tris, rng if rotate else None)
    neigh = compute_neighbors(tris)
    cen = points[tris].mean(axis=1)
    attr = np.ones(tris.shape[0], dtype=np.int64) if attr_fn is None else \
        np.asarray(attr_fn(cen[:, 0], cen[:, 1]), dtype=np.int64)
    return Mesh(points, tris, neigh, attr, _boundary_markers(points.shape[0], tris, neigh))


def delaunay(width: float, height: float, h: float, *, seed: int = 0, jitter: float = 0.25,
             top=None, pinned=(), attr_fn=None, rotate: bool = True) -> Mesh:
    """Seeded Delaunay triangulation of jittered points with target edge length ``h``.

    ``top(x)`` gives the z of a curved upper surface (default: flat at ``height``); points are
    placed on the four sides (the top following the curve) and, jittered, inside, then
    triangles whose centroid lies above the curve are dropped.
    """
    from scipy.spatial import Delaunay  # setup-time only

    rng = np.random.default_rng(seed)
    if top is None:
        top = lambda xx: np.full_like(np.asarray(xx, dtype=np.float64), height)  # noqa: E731
    nx = int(round(width / h))
    xs = np.linspace(0.0, width, nx + 1)
    ztop = top(xs)
    nzl = int(round(float(np.min(ztop)) / h))
    zs_left = np.linspace(0.0, float(top(np.array([0.0]))[0]), max(nzl, 1) + 1)
    zs_right = np.linspace(0.0, float(top(np.array([width]))[0]), max(nzl, 1) + 1)
    bottom = np.stack([xs, np.zeros_like(xs)], 1)
    upper = np.stack([xs, ztop], 1)
    left = np.stack([np.zeros_like(zs_left), zs_left], 1)[1:-1]
    right = np.stack([np.full_like(zs_right, width), zs_right], 1)[1:-1]
    # interior lattice (offset rows), jittered
    hz = h * np.sqrt(3.0) / 2.0
    rows = []
    zmax = float(np.max(ztop))
    j = 1
    while j * hz < zmax:
        off = 0.5 * h if j % 2 else 0.0
        xr = np.arange(h * 0.5 + off, width - 0.25 * h, h)
        zr = np.full_like(xr, j * hz)
        rows.append(np.stack([xr, zr], 1))
        j += 1
    inner = np.concatenate(rows, 0)
    inner = inner + rng.uniform(-jitter * h, jitter * h, size=inner.shape)
    keep = (inner[:, 0] > 0.3 * h) & (inner[:, 0] < width - 0.3 * h) & (inner[:, 1] > 0.3 * h) & \
           (inner[:, 1] < top(inner[:, 0]) - 0.3 * h)
    inner = inner[keep]
    pin = np.asarray(pinned, dtype=np.float64).reshape(-1, 2)
    if pin.shape[0]:
        # clear jittered points near pinned vertices, then add the pinned ones exactly
        d2 = ((inner[:, None, :] - pin[None, :, :]) ** 2).sum(-1).min(1)
        inner = inner[d2 > (0.5 * h) ** 2]
    pts = np.concatenate([bottom, upper, left, right, inner, pin], 0)
    # drop duplicates (pinned points that coincide with boundary points)
    _, uidx = np.unique(np.round(pts, 6), axis=0, return_index=True)
    pts = pts[np.sort(uidx)]
    tri = Delaunay(pts)
    tris = tri.simplices.astype(np.int64)
    cen = pts[tris].mean(axis=1)
    tris = tris[cen[:, 1] < top(cen[:, 0])]
    # renumber to the used vertices only
    used = np.unique(tris)
    remap = np.full(pts.shape[0], -1, dtype=np.int64)
    remap[used] = np.arange(used.size)
    pts = pts[used]
    tris = remap[tris]
    tris = _orient_ccw(pts, tris)
    tris = _rotate(tris, rng if rotate else None)
    neigh = compute_neighbors(tris)
    cen = pts[tris].mean(axis=1)
    attr = np.ones(tris.shape[0], dtype=np.int64) if attr_fn is None else \
        np.asarray(attr_fn(cen[:, 0], cen[:, 1]), dtype=np.int64)
    return Mesh(pts, tris, neigh, attr, _boundary_markers(pts.shape[0], tris, neigh))


@dataclasses.dataclass
class PSLG:
    """A planar straight-line graph in Triangle's ``.poly`` terms."""

    vertices: np.ndarray   # (V, 2) float64
    segments: np.ndarray   # (E, 2) int64, 0-based vertex ids
    holes: np.ndarray      # (H, 2) float64 seed points of holes
    regions: np.ndarray    # (R, 4) float64: x, z, attribute, maximum triangle area (<= 0: none)


def read_poly(src: str) -> PSLG:
    """Parse a ``.poly`` file (a path or its text): vertex count/dim/attributes/markers, vertex
    lines ``id x z [attributes] [marker]``, ``#segments [#markers]`` and ``id a b [marker]``,
    ``#holes`` and ``id x z``, optionally ``#regions`` and ``id x z attribute max_area`` (the
    inputs of input_files/mesh/*.poly).  Vertex ids may start at 0 or 1; ``#`` starts a comment."""
    text = open(src).read() if os.path.exists(src) else src
    rows = []
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            rows.append(line.split())
    nv = int(float(rows[0][0]))
    at = 1
    ids = []
    verts = np.zeros((nv, 2))
    for k in range(nv):
        r = rows[at + k]
        ids.append(int(float(r[0])))
        verts[k] = float(r[1]), float(r[2])
    at += nv
    idx = {v: k for k, v in enumerate(ids)}
    ne = int(float(rows[at][0]))
    at += 1
    segs = np.zeros((ne, 2), dtype=np.int64)
    for k in range(ne):
        r = rows[at + k]
        segs[k] = idx[int(float(r[1]))], idx[int(float(r[2]))]
    at += ne
    holes = np.zeros((0, 2))
    if at < len(rows):
        nh = int(float(rows[at][0]))
        at += 1
        holes = np.array([[float(r[1]), float(r[2])] for r in rows[at:at + nh]]).reshape(-1, 2)
        at += nh
    regions = np.zeros((0, 4))
    if at < len(rows):
        nr = int(float(rows[at][0]))
        at += 1
        regions = np.array([[float(r[1]), float(r[2]), float(r[3]), float(r[4]) if len(r) > 4 else -1.0]
                            for r in rows[at:at + nr]]).reshape(-1, 4)
    return PSLG(verts, segs, holes, regions)


def from_poly(pslg, h: float | None = None, *, seed: int = 0, jitter: float = 0.25, rotate: bool = True,
              max_rounds: int = 30) -> Mesh:
    """Triangulate a PSLG (what ``triangle -pqanA`` does for the reference, create_mesh_file.m:5):
    triangles whose edges follow every segment, regional attributes, holes removed.

    Points go along every segment (spacing <= h) and on a jittered offset-row lattice of spacing
    h inside; lattice points within a sub-segment's diametral circle are dropped, so every
    sub-segment is a Delaunay edge; a sub-segment that still is not (another segment's points
    encroach on it) is split at its midpoint and the points are triangulated again.  Triangles
    reachable from the convex hull or a hole seed without crossing a segment are removed; each
    region seed's attribute fills the triangles reachable from it.  ``h`` defaults to the edge
    of an equilateral triangle of the smallest regional maximum area (or 1/40 of the extent).
    """
    from scipy.spatial import Delaunay, cKDTree  # set-up time only

    g = read_poly(pslg) if isinstance(pslg, str) else pslg
    rng = np.random.default_rng(seed)
    lo, hi = g.vertices.min(0), g.vertices.max(0)
    if h is None:
        areas = g.regions[:, 3][g.regions[:, 3] > 0] if g.regions.size else np.zeros(0)
        h = float(np.sqrt(4.0 * areas.min() / np.sqrt(3.0))) if areas.size else float((hi - lo).max() / 40.0)
    # sub-segments: consecutive points along each segment
    sub = []        # list of (point a, point b) coordinate pairs
    for a, b in g.segments:
        pa, pb = g.vertices[a], g.vertices[b]
        n = max(1, int(np.ceil(np.linalg.norm(pb - pa) / h - 1e-9)))
        t = np.linspace(0.0, 1.0, n + 1)
        pts = pa[None, :] + t[:, None] * (pb - pa)[None, :]
        sub.extend(zip(pts[:-1], pts[1:]))
    # interior lattice
    hz = h * np.sqrt(3.0) / 2.0
    rows = []
    j = 0
    while lo[1] + j * hz <= hi[1]:
        off = 0.5 * h if j % 2 else 0.0
        xr = np.arange(lo[0] + off, hi[0] + 1e-9, h)
        rows.append(np.stack([xr, np.full_like(xr, lo[1] + j * hz)], 1))
        j += 1
    inner = np.concatenate(rows, 0)
    inner = inner + rng.uniform(-jitter * h, jitter * h, size=inner.shape)

    def key(p):
        return (round(float(p[0]), 9), round(float(p[1]), 9))

    for _ in range(max_rounds):
        seg_pts = {}
        for a, b in sub:
            seg_pts.setdefault(key(a), a)
            seg_pts.setdefault(key(b), b)
        sp = np.array(list(seg_pts.values()))
        mids = np.array([(a + b) / 2 for a, b in sub])
        rad = np.array([np.linalg.norm(b - a) / 2 for a, b in sub])
        # keep lattice points outside every diametral circle and away from segment points
        keep = cKDTree(sp).query(inner)[0] > 0.45 * h
        tree = cKDTree(inner)
        for m, r in zip(mids, rad):
            for i in tree.query_ball_point(m, r * 1.05):
                keep[i] = False
        pts = np.concatenate([sp, inner[keep]], 0)
        tri = Delaunay(pts)
        simp = tri.simplices.astype(np.int64)
        edges = set()
        for t in simp:
            for u, v in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
                edges.add((min(u, v), max(u, v)))
        pid = {key(p): i for i, p in enumerate(pts)}
        missing = []
        for k, (a, b) in enumerate(sub):
            u, v = pid[key(a)], pid[key(b)]
            if (min(u, v), max(u, v)) not in edges:
                missing.append(k)
        if not missing:
            break
        for k in sorted(missing, reverse=True):
            a, b = sub[k]
            m = (a + b) / 2
            sub[k:k + 1] = [(a, m), (m, b)]
    else:
        raise RuntimeError("could not make every segment a mesh edge")
    # barrier edges, then flood fills over the triangle adjacency
    barrier = set()
    for a, b in sub:
        u, v = pid[key(a)], pid[key(b)]
        barrier.add((min(u, v), max(u, v)))
    nbr = tri.neighbors.astype(np.int64)   # scipy: neighbour k lies opposite vertex k

    def edge_of(t, k):
        u, v = simp[t, (k + 1) % 3], simp[t, (k + 2) % 3]
        return (min(u, v), max(u, v))

    def fill(starts, mark, value):
        stack = [s for s in starts if s >= 0 and mark[s] != value]
        for s in stack:
            mark[s] = value
        while stack:
            t = stack.pop()
            for k in range(3):
                n = nbr[t, k]
                if n >= 0 and mark[n] != value and edge_of(t, k) not in barrier:
                    mark[n] = value
                    stack.append(n)

    T = simp.shape[0]
    outside = np.zeros(T, dtype=np.int64)
    hull = [t for t in range(T) for k in range(3) if nbr[t, k] < 0 and edge_of(t, k) not in barrier]
    fill(hull, outside, 1)
    if g.holes.size:
        fill(list(tri.find_simplex(g.holes)), outside, 1)
    attr = np.zeros(T, dtype=np.int64)
    for x, z, a, _area in g.regions:
        fill([int(tri.find_simplex(np.array([[x, z]]))[0])], attr, int(round(a)))
    inside = outside == 0
    tris = simp[inside]
    attr = attr[inside]
    used = np.unique(tris)
    remap = np.full(pts.shape[0], -1, dtype=np.int64)
    remap[used] = np.arange(used.size)
    pts = pts[used]
    tris = remap[tris]
    tris = _orient_ccw(pts, tris)
    tris = _rotate(tris, rng if rotate else None)
    neigh = compute_neighbors(tris)
    return Mesh(pts, tris, neigh, attr, _boundary_markers(pts.shape[0], tris, neigh))


def text_round(x) -> np.ndarray:
    """Round to the 8 significant digits the ``%16.7e`` text format keeps."""
    x = np.asarray(x, dtype=np.float64)
    return np.array([float("%.7e" % v) for v in x.ravel()]).reshape(x.shape)


def snap_to_vertices(mesh: Mesh, positions) -> np.ndarray:
    """Nearest mesh vertex to each (x, z) position, rounded as the text files store it.

    Get_Source / Get_Receiver match positions to vertices within 1e-3 / 1e-2
    (fun_DG.c:304, 380), so sources and receivers are placed exactly on vertices.
    """
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 2)
    out = np.empty_like(pos)
    for i, p in enumerate(pos):
        d2 = ((mesh.points - p) ** 2).sum(1)
        out[i] = mesh.points[int(np.argmin(d2))]
    return text_round(out)


def _save_ascii(path: str, rows: np.ndarray) -> None:
    """MATLAB ``save -ascii``: every value as ``%16.7e``, one row per line."""
    rows = np.asarray(rows, dtype=np.float64)
    with open(path, "w") as f:
        np.savetxt(f, rows, fmt="%16.7e", delimiter="")


def write_converted(mesh: Mesh, prefix: str) -> dict:
    """Write ``prefix.ele``, ``prefix.node`` and ``prefix.neigh`` as create_mesh_file.m does.

    Header rows (create_mesh_file.m:9-16, 23-29, 36-43): ``.ele`` = [K, 3, 1, 0, 0],
    ``.node`` = [P, 2, 0, 1], ``.neigh`` = [K, 3, 0, 0].  Indices are 1-based and ``-1``
    marks a missing neighbour.  The neighbour file is written under the name the C driver
    opens (the MATLAB script's ``model_converted.1.neigh`` never matches it).
    """
    K, P = mesh.K, mesh.P
    if K >= 10**8 or P >= 10**8:
        raise ValueError("the 8-significant-digit text format cannot hold indices >= 1e8")
    d = os.path.dirname(prefix)
    if d:
        os.makedirs(d, exist_ok=True)
    ele = np.zeros((K + 1, 5))
    ele[0, :3] = [K, 3, 1]
    ele[1:, 0] = np.arange(1, K + 1)
    ele[1:, 1:4] = mesh.tris + 1
    ele[1:, 4] = mesh.attr
    node = np.zeros((P + 1, 4))
    node[0, :] = [P, 2, 0, 1]
    node[1:, 0] = np.arange(1, P + 1)
    node[1:, 1:3] = mesh.points
    node[1:, 3] = mesh.markers
    neigh = np.zeros((K + 1, 4))
    neigh[0, :2] = [K, 3]
    neigh[1:, 0] = np.arange(1, K + 1)
    nb = mesh.neigh.copy()
    nb[nb >= 0] += 1
    neigh[1:, 1:4] = nb
    paths = {"ele": prefix + ".ele", "node": prefix + ".node", "neigh": prefix + ".neigh"}
    _save_ascii(paths["ele"], ele)
    _save_ascii(paths["node"], node)
    _save_ascii(paths["neigh"], neigh)
    return paths


def write_epart(path: str, K: int, parts: np.ndarray | None = None) -> None:
    """METIS element-partition file (one integer per line) as ``epartinput`` reads it."""
    parts = np.zeros(K, dtype=np.int64) if parts is None else np.asarray(parts)
    with open(path, "w") as f:
        f.write("\n".join(str(int(p)) for p in parts))
        f.write("\n")
