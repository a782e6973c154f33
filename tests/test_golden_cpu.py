"""CPU checks pinned to the golden fixtures made by the reference's own C code.

* the restated P2 operators print to the same 8-significant-digit text the reference ships;
* the host set-up library (csrc/dg_host.c) reproduces every set-up array bit for bit,
  from the mesh text files and from memory;
* the CPU oracle (oracle/dg_oracle.c) reproduces the reference's traces, snapshots and final
  fields bit for bit.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import Golden, golden_names, pkg

import oracle

host = pkg.host


def test_operator_text_matches_shipped_files():
    """precompute_matrices.m restated: same text as input_files/precomputed_matrix (to 1e-16)."""
    g = Golden(golden_names()[0])
    mine = host.text_operators()
    for name in ("V", "Vr", "Vs", "FeketeNew", "S1", "S2", "S3"):
        assert np.array_equal(mine[name], g.ops[name]), name
    # inverV: the shipped file carries inversion roundoff (e.g. 5.55e-17) where ours has other
    # roundoff; every entry above 1e-15 is identical
    big = np.abs(g.ops["inverV"]) > 1e-15
    assert np.array_equal(mine["inverV"][big], g.ops["inverV"][big])
    assert np.max(np.abs(mine["inverV"] - g.ops["inverV"])) < 1e-16


def test_text_reader_round_trip(golden):
    """Mesh text files written like create_mesh_file.m, parsed like ReadInt/ReadDouble."""
    with tempfile.TemporaryDirectory() as d:
        pkg.meshgen.write_converted(golden.workload().mesh, os.path.join(d, "mesh"))
        pts, tri, nb, at = host.read_mesh(os.path.join(d, "mesh"))
    assert np.array_equal(pts, golden.z["setup_Point"].reshape(-1, 2))
    assert np.array_equal(tri.ravel(), golden.z["setup_Triangle"])
    assert np.array_equal(nb.ravel(), golden.z["setup_neighbor_in"])
    assert np.array_equal(at, golden.z["setup_attribute"])
    # the in-memory path rounds coordinates the same way
    assert np.array_equal(host.quantize_e7(golden.z["points_raw"]), pts)


INT_NAMES = ["Neighbor", "Edge", "Edge_flag", "Node_Neighbor", "ibe", "source", "receiver"]
FLOAT_NAMES = ["Jacobi", "Jacobi_Edge", "normal1", "normal2", "normal3", "A", "B", "Q", "Dx", "Dz", "S", "absorb_fun",
               "fun"]


def test_host_setup_bit_exact(golden):
    w = golden.workload()
    s = host.build_setup(w, ops=golden.ops)
    assert s.dt == golden.dt and s.t0 == golden.t0
    assert s.absorb_count == golden.z["setup_sizes"][2]
    assert s.absorb_filled == golden.z["setup_sizes"][3]
    for n in INT_NAMES + FLOAT_NAMES:
        assert np.array_equal(s.arrays[n].ravel(), golden.z["setup_" + n]), n


def test_host_setup_from_files(golden):
    w = golden.workload()
    with tempfile.TemporaryDirectory() as d:
        pkg.meshgen.write_converted(w.mesh, os.path.join(d, "mesh"))
        arrays = host.read_mesh(os.path.join(d, "mesh"))
    s = host.build_setup(w, ops=golden.ops, mesh_arrays=arrays)
    for n in INT_NAMES + FLOAT_NAMES:
        assert np.array_equal(s.arrays[n].ravel(), golden.z["setup_" + n]), n


def test_oracle_bit_exact(golden):
    a = golden.setup_arrays()
    o = oracle.Oracle(a, golden.dt, golden.K)
    for m in range(golden.shots):
        o.reset()
        for t0 in range(0, golden.steps, golden.snap_every):
            rx, rz = o.run(m, golden.snap_every, threads=2)
            t1 = t0 + golden.snap_every
            assert np.array_equal(rx, golden.z["shot%d_rec_x" % m][t0:t1])
            assert np.array_equal(rz, golden.z["shot%d_rec_z" % m][t0:t1])
            assert np.array_equal(o.fields[0], golden.z["shot%d_Vx%d" % (m, t1)])
            assert np.array_equal(o.fields[1], golden.z["shot%d_Vz%d" % (m, t1)])
        for f, name in enumerate(("Vx", "Vz", "Txx", "Tzz", "Txz")):
            assert np.array_equal(o.fields[f], golden.z["shot%d_final_%s" % (m, name)]), name


def test_oracle_detects_a_planted_mistake(golden):
    """The checker is sensitive: one flipped neighbour orientation changes the traces."""
    a = golden.setup_arrays()
    nn = a["Node_Neighbor"].reshape(-1, 3, 3).copy()
    e, f = np.argwhere(a["Edge_flag"].reshape(-1, 3) == 1)[len(nn) // 2]
    nn[e, f] = nn[e, f][::-1]
    a["Node_Neighbor"] = nn
    o = oracle.Oracle(a, golden.dt, golden.K)
    rx, _ = o.run(0, golden.steps, threads=2)
    assert not np.array_equal(rx, golden.z["shot0_rec_x"])


@pytest.mark.parametrize("bad", ["missing_file", "short_file", "source_off_mesh"])
def test_host_errors(bad, tmp_path):
    w = pkg.workloads.small_square(n_cells=4, steps=5)
    if bad == "missing_file":
        with pytest.raises(host.HostError):
            host.read_mesh(str(tmp_path / "nope"))
    elif bad == "short_file":
        pkg.meshgen.write_converted(w.mesh, str(tmp_path / "m"))
        txt = open(tmp_path / "m.node").read().splitlines()
        open(tmp_path / "m.node", "w").write("\n".join(txt[: len(txt) // 2]) + "\n")
        with pytest.raises(host.HostError):
            host.read_mesh(str(tmp_path / "m"))
    else:
        w.src = np.array([[123.456, 789.0]])
        with pytest.raises(host.HostError):
            host.build_setup(w)


def test_source_and_receiver_vertex_rules_with_duplicate_vertices():
    """Get_Source takes the FIRST vertex within 1e-3 of the position, Get_Receiver the LAST within
    1e-2 (fun_DG.c:284-418).  A near-duplicate of a receiver vertex placed before every other
    vertex (and used by no triangle) leaves the receivers as they were; a near-duplicate of the
    source vertex there makes the source land on a vertex no triangle holds: NOSOURCE."""
    w = pkg.workloads.small_square(n_cells=8, steps=5)
    base = host.build_setup(w, full=False)
    pts = host.quantize_e7(w.mesh.points)
    tri = (w.mesh.tris + 1).astype(np.int64)
    nb = np.where(w.mesh.neigh >= 0, w.mesh.neigh + 1, -1).astype(np.int64)

    def with_duplicate(xz):
        return (np.vstack([np.asarray(xz, dtype=np.float64)[None, :], pts]), tri + 1, nb)

    r = w.rec[len(w.rec) // 2]
    s = host.build_setup(w, full=False, mesh_arrays=with_duplicate([r[0] + 4e-3, r[1] - 4e-3]))
    assert np.array_equal(s.arrays["receiver"], base.arrays["receiver"])
    assert np.array_equal(s.arrays["source"], base.arrays["source"])
    with pytest.raises(host.HostError) as ei:
        host.build_setup(w, full=False, mesh_arrays=with_duplicate([w.src[0][0] + 5e-4, w.src[0][1]]))
    assert "(-4)" in str(ei.value)


_DIGEST = r"""
import hashlib, importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
P = importlib.import_module("discontinuous-galerkin-method_b200")
w = P.workloads.random_medium(n_cells_x=100, n_cells_z=50, n_rec=101, corr_len=400.0, steps=20)
s = P.host.build_setup(w, full=True, n_steps=20)
h = hashlib.sha1()
for k in sorted(s.arrays):
    a = s.arrays[k]
    if isinstance(a, np.ndarray):
        h.update(k.encode()); h.update(np.ascontiguousarray(a).tobytes())
h.update(repr(s.dt).encode())
print(h.hexdigest())
"""


def test_host_setup_independent_of_thread_count():
    """The set-up's per-element loops run on OpenMP threads; every array (and dt) is the same
    with one thread as with several."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = []
    for n in ("1", "5"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        r = subprocess.run([sys.executable, "-c", _DIGEST, root], env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        out.append(r.stdout.strip())
    assert out[0] == out[1] and len(out[0]) == 40


def test_large_text_files_parallel_reader(tmp_path):
    """Files above 1 MB are parsed in parallel chunks cut at line starts: integers and doubles
    come back exactly as the sequential ReadInt/ReadDouble scan gives them, a row with one number
    too many (it spills into the next row's first slot, which the next row then overwrites) reads
    as the sequential scan reads it, and a missing number is a format error."""
    rng = np.random.default_rng(7)
    rows, cols = 60000, 3
    ints = rng.integers(-1, 10**6, size=(rows, cols)).astype(np.int64)
    ints[ints < 0] = -1                                   # -1 is the only negative the files hold
    path = str(tmp_path / "ints.txt")
    lines = ["".join("%16.7e" % v for v in r) for r in ints]
    lines[123] += "%16.7e" % 5.0                          # one number too many in row 123
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    assert os.path.getsize(path) > (1 << 20)
    out = np.zeros(rows * cols, dtype=np.int64)
    assert host.lib().dgh_read_int_matrix(path.encode(), out.ctypes.data, rows, cols) == rows * cols
    # the sequential scan, restated: slot row * cols + n, stop at the wanted count
    want = np.zeros(rows * cols, dtype=np.int64)
    num = 0
    for m, line in enumerate(lines):
        for n, tok in enumerate(line.split()):
            if num == rows * cols:
                break
            want[m * cols + n] = int(float(tok))
            num += 1
    assert np.array_equal(out, want)
    assert want[-1] == 0 and np.array_equal(want[:-1], ints.ravel()[:-1])   # the extra number took the last slot's turn

    vals = rng.normal(size=(rows, cols)) * 10.0 ** rng.integers(-5, 6, size=(rows, cols))
    dpath = str(tmp_path / "doubles.txt")
    pkg.meshgen._save_ascii(dpath, vals)
    got = np.zeros(rows * cols)
    assert host.lib().dgh_read_matrix(dpath.encode(), got.ctypes.data, rows, cols) == rows * cols
    parse = host.lib().dgh_parse_e7
    toks = [" " * 16 + "%16.7e" % v for v in vals.ravel()[:2000]]
    want = np.array([parse(t.encode(), t.index("e")) for t in toks])
    assert np.array_equal(got[:2000], want)
    assert np.allclose(got, vals.ravel(), rtol=1e-7, atol=0)
    short = str(tmp_path / "short.txt")
    with open(short, "w") as f:
        f.write("\n".join(lines[:-1]) + "\n")
    assert host.lib().dgh_read_int_matrix(short.encode(), out.ctypes.data, rows, cols) < 0


def test_text_and_binary_writers(tmp_path):
    """Save_Data's format ("%0.14f " per value, a line break per row) from the parallel writer and
    its own exact decimal conversion, over several blocks of rows, with the values printf treats
    specially and exact decimal ties (Python's %-formatting, like printf, is correctly rounded,
    ties to even); and the binary dump reads back exactly."""
    rng = np.random.default_rng(11)
    rows, cols = 70001, 3
    m = rng.normal(size=(rows, cols)) * 10.0 ** rng.integers(-15, 4, size=(rows, cols))
    m[5] = [0.0, -0.0, 1e300]
    m[40000] = [np.inf, -np.inf, np.nan]
    m[69999] = [-1e-300, 5e-324, -123456.78901234567]
    # exact decimal ties at the 14th place (odd multiples of 2^-15) round to even, as printf does
    j = 2 * rng.integers(0, 2**30, size=(3000, cols)) + 1
    m[1000:4000] = np.ldexp(j.astype(np.float64), -15) * np.where(rng.integers(0, 2, size=(3000, cols)), 1.0, -1.0)
    m[4000:4100] = 10.0 ** rng.uniform(5, 15.9, size=(100, cols))   # wide integer parts, up to 2^53
    path = str(tmp_path / "snap.txt")
    assert host.lib().dgh_write_matrix(path.encode(), m.ctypes.data, rows, cols) == 0
    want = "".join("".join("%0.14f " % v for v in r) + "\n" for r in m)
    with open(path) as f:
        assert f.read() == want
    rec = m[:, 0].copy()
    assert host.lib().dgh_write_record(path.encode(), rec.ctypes.data, rows) == 0
    with open(path) as f:
        assert f.read() == "".join("%0.14f \n" % v for v in rec)
    bpath = str(tmp_path / "snap.bin")
    assert host.lib().dgh_write_binary(bpath.encode(), m.ctypes.data, m.size) == 0
    back = np.fromfile(bpath, dtype=np.float64).reshape(rows, cols)
    assert np.array_equal(back, m, equal_nan=True)
