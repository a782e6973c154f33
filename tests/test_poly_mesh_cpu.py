"""Meshes from planar straight-line graphs (the .poly inputs the reference meshes with Triangle).

Triangle itself is not available, so its output cannot be pinned; these tests check what the
reference's set-up relies on: counter-clockwise triangles that tile the domain exactly, every
segment made of mesh edges, the regional attributes filling the right areas, holes left out,
neighbour maps that agree, and a model built on such a mesh running through the host set-up
and the CPU oracle with the fields staying finite and non-zero.
"""
import numpy as np
import pytest

from conftest import pkg

import oracle

mg = pkg.meshgen

# an L-shaped domain cut by a sloping interface into two regions
L_SHAPE = """
# vertices: id x z
8 2 0 1
1 0 0
2 3000 0
3 3000 1500
4 1800 1500
5 1800 2400
6 0 2400
7 0 900
8 3000 700
9 1
1 1 2 1
2 2 8 1
3 8 3 1
4 3 4 1
5 4 5 1
6 5 6 1
7 6 7 1
8 7 1 1
9 7 8 2
0
2
1 100 100 1 4000
2 100 2000 2 8000
"""

# a square with a square hole
HOLE = """
8 2 0 0
0 0 0
1 1000 0
2 1000 1000
3 0 1000
4 400 400
5 600 400
6 600 600
7 400 600
8
0 0 1
1 1 2
2 2 3
3 3 0
4 4 5
5 5 6
6 6 7
7 7 4
1
0 500 500
1
0 10 10 5 500
"""


def _areas(m):
    p = m.points[m.tris]
    return 0.5 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) -
                  (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))


def _min_angles(m):
    p = m.points[m.tris]
    out = []
    for k in range(3):
        a = p[:, (k + 1) % 3] - p[:, k]
        b = p[:, (k + 2) % 3] - p[:, k]
        c = (a * b).sum(1) / np.linalg.norm(a, axis=1) / np.linalg.norm(b, axis=1)
        out.append(np.degrees(np.arccos(np.clip(c, -1, 1))))
    return np.min(out, 0)


def _edges(m):
    e = set()
    for t in m.tris:
        for k in range(3):
            u, v = int(t[k]), int(t[(k + 1) % 3])
            e.add((min(u, v), max(u, v)))
    return e


@pytest.mark.parametrize("text,area,regions", [
    (L_SHAPE, 3000 * 1500 + 1800 * 900, {1: (900 + 700) / 2 * 3000, 2: 3000 * 1500 + 1800 * 900 - 2.4e6}),
    (HOLE, 1000 * 1000 - 200 * 200, {5: 1000 * 1000 - 200 * 200}),
])
def test_triangulation_tiles_the_domain_and_follows_the_segments(text, area, regions):
    g = mg.read_poly(text)
    m = mg.from_poly(g)
    a = _areas(m)
    assert a.min() > 0
    assert a.sum() == pytest.approx(area, rel=1e-12)
    for attr, want in regions.items():
        assert a[m.attr == attr].sum() == pytest.approx(want, rel=1e-9), attr
    assert _min_angles(m).min() > 15.0
    # every segment is a chain of mesh edges: its length equals the summed edges on it
    E = _edges(m)
    for s0, s1 in g.segments:
        pa, pb = g.vertices[s0], g.vertices[s1]
        d = pb - pa
        t = ((m.points - pa) @ d) / (d @ d)
        off = np.abs((m.points - pa) @ np.array([-d[1], d[0]])) / np.linalg.norm(d)
        on = np.flatnonzero((off < 1e-6) & (t > -1e-9) & (t < 1 + 1e-9))
        chain = on[np.argsort(t[on])]
        assert t[chain[0]] == pytest.approx(0, abs=1e-9) and t[chain[-1]] == pytest.approx(1, abs=1e-9)
        for u, v in zip(chain[:-1], chain[1:]):
            assert (min(u, v), max(u, v)) in E
    # neighbour maps agree both ways
    for t in range(m.K):
        for k in range(3):
            n = m.neigh[t, k]
            if n >= 0:
                assert t in m.neigh[n]


def test_poly_model_runs_through_setup_and_oracle():
    w = pkg.workloads.poly_model(L_SHAPE, {1: (4000.0, 2300.0, 2500.0), 2: (1500.0, 0.0, 1000.0)},
                                 src=[(1500.0, 500.0)], rec=[(x, 2400.0) for x in (100.0, 800.0, 1600.0)],
                                 h=120.0, fp=8.0, steps=300)
    s = pkg.host.build_setup(w, full=True)
    assert s.arrays["receiver"].shape == (3, 2)
    o = oracle.Oracle.from_setup(s)
    o.run(0, w.steps, threads=2)
    v = o.fields[1]
    assert np.all(np.isfinite(v)) and np.abs(v).max() > 0
