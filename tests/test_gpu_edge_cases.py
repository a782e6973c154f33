"""Edge cases of mesh size, shot count and receivers, against the CPU oracle.

* tiny meshes (8 to 72 triangles: fewer elements than one padded group of 32, exactly 32, and
  counts that are not multiples of 32) with 1 to 3 shots, in every precision;
* 130 shots, past the packed kernels' 128 (one (element, shot) per thread);
* a mesh without receivers (recorder blocks absent), on the two-launch and wavefront steps:
  fields equal those of the same run with receivers, and the traces are empty.
"""
import numpy as np
import pytest

from conftest import pkg, rel_l2

import oracle

eng = pkg.engine
pytestmark = pytest.mark.gpu
TOL = {"fp64_ref": 0.0, "fp64": 1e-10, "fp32": 1e-4, "fp32_kahan": 1e-4}


def _oracle_traces(s, shots, steps):
    o = oracle.Oracle.from_setup(s)
    out = []
    for m in shots:
        o.reset()
        out.append(o.run(m, steps, threads=1))
    return out


@pytest.mark.parametrize("precision", ["fp64_ref", "fp64", "fp32", "fp32_kahan"])
@pytest.mark.parametrize("n_cells,shots", [(2, 1), (4, 2), (5, 2), (6, 3)])
def test_tiny_meshes_against_oracle(precision, n_cells, shots):
    steps = 60
    w = pkg.workloads.homogeneous_square(n_cells=n_cells, steps=steps, n_rec=n_cells + 1, shots=shots)
    s = pkg.host.build_setup(w)
    assert s.K == 2 * n_cells * n_cells
    ref = _oracle_traces(s, range(shots), steps)
    with eng.Engine(eng.mesh_from_setup(s), precision) as e:
        e.step(steps)
        for m in range(shots):
            got = np.concatenate([e.fetch("trace_x", 0, m).ravel(), e.fetch("trace_z", 0, m).ravel()])
            want = np.concatenate([ref[m][0].ravel(), ref[m][1].ravel()])
            assert np.abs(want).max() > 0
            if precision == "fp64_ref":
                assert np.array_equal(got, want), m
            else:
                assert rel_l2(got, want) <= TOL[precision], (m, rel_l2(got, want))


def test_more_shots_than_the_packed_kernels_take():
    steps = 60
    w = pkg.workloads.homogeneous_square(n_cells=12, steps=steps, n_rec=13, shots=130)
    s = pkg.host.build_setup(w)
    ref = _oracle_traces(s, (0, 64, 129), steps)
    with eng.Engine(eng.mesh_from_setup(s), "fp32") as e:
        assert e.stats()["kernel_family"] == 1            # one (element, shot) per thread
        e.step(steps)
        for (x, z), m in zip(ref, (0, 64, 129)):
            got = np.concatenate([e.fetch("trace_x", 0, m).ravel(), e.fetch("trace_z", 0, m).ravel()])
            assert rel_l2(got, np.concatenate([x.ravel(), z.ravel()])) <= 1e-4, m


@pytest.mark.parametrize("precision,shots", [("fp32", 1), ("fp64", 2), ("fp32", 16)])
def test_mesh_without_receivers(precision, shots):
    steps = 60
    fields = []
    for n_rec in (13, 0):
        w = pkg.workloads.homogeneous_square(n_cells=12, steps=steps, n_rec=n_rec, shots=shots)
        s = pkg.host.build_setup(w)
        with eng.Engine(eng.mesh_from_setup(s), precision) as e:
            fam = e.stats()["kernel_family"]
            e.step(steps)
            fields.append([e.fetch(f, 0, shots - 1) for f in ("Vx", "Vz", "Txx")])
            if n_rec == 0:
                assert e.fetch("trace_z", 0, 0).size == 0
                tx, tz = e.fetch_traces(0, steps)
                assert tx.size == 0 and tz.size == 0
    assert fam in ((6,) if shots == 16 else (1, 3, 7))
    for a, b in zip(*fields):
        assert np.array_equal(a, b)
    assert np.abs(fields[0][1]).max() > 0


def test_reference_path_rebuilt_operators_equal_arrays_and_oracle(monkeypatch):
    """DG_FP64_REF on one one-shot mesh of 65,536 elements or more rebuilds Dx, Dz in the
    kernels (after checking on the host that they equal the caller's arrays): traces and fields
    equal the array path and the CPU oracle bit for bit."""
    import os
    steps = 120
    w = pkg.workloads.homogeneous_square(n_cells=182, steps=steps, n_rec=183)
    s = pkg.host.build_setup(w)
    assert s.K >= 65536
    o = oracle.Oracle.from_setup(s)
    o.reset()
    rx, rz = o.run(0, steps, threads=os.cpu_count() or 1)
    out = []
    for arrays in ("1", "0"):
        monkeypatch.setenv("DG_REF_ARRAYS", arrays)
        with eng.Engine(eng.mesh_from_setup(s), "fp64_ref") as e:
            e.step(steps)
            out.append((e.fetch("trace_x"), e.fetch("trace_z"), e.fetch("Vz")))
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    assert np.array_equal(out[1][0], rx) and np.array_equal(out[1][1], rz)
    assert np.abs(rz).max() > 0
