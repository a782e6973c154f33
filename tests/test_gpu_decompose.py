"""A mesh split into parts on the GPU (domain decomposition through the C ABI).

All parts run as contexts on one device (`decompose.SplitRun` without a communicator: the halo
buffers are copied device to device; with `torch.distributed` the same buffers travel between
GPUs).  Owned triangles compute what the whole mesh computes, so every field and trace equals the
undivided run bit for bit, in every precision.
"""
import numpy as np
import pytest

from conftest import pkg

eng = pkg.engine
dec = pkg.decompose
pytestmark = pytest.mark.gpu
FIELDS = ("Vx", "Vz", "Txx", "Tzz", "Txz")


@pytest.fixture(scope="module")
def meshes():
    out = {}
    for shots in (1, 2, 3):
        w = pkg.workloads.small_square(n_cells=16, steps=160, shots=shots)
        s = pkg.host.build_setup(w, full=True)
        out[shots] = (s, eng.mesh_from_setup(s))
    return out


@pytest.mark.parametrize("precision,shots,P", [("fp64_ref", 1, 3), ("fp64", 2, 2), ("fp64", 3, 4),
                                               ("fp32", 1, 3), ("fp32", 2, 2), ("fp32_kahan", 3, 3)])
def test_split_mesh_equals_whole_mesh(meshes, precision, shots, P):
    s, mesh = meshes[shots]
    steps = 150
    with eng.Engine(mesh, precision, wavefront=-1) as whole:
        whole.step(steps)
        want = {(f, m): whole.fetch(f, 0, m).reshape(-1, 6) for f in FIELDS for m in range(shots)}
        want_tr = {(c, m): whole.fetch(c, 0, m) for c in ("trace_x", "trace_z") for m in range(shots)}
    with dec.SplitRun(mesh, P, precision) as run:
        run.step(steps)
        for (f, m), v in want.items():
            assert np.array_equal(run.fetch(f, m), v), (f, m)
        for (c, m), v in want_tr.items():
            assert np.array_equal(run.traces(c, m), v), (c, m)
    assert np.abs(want[("Vz", 0)]).max() > 0


def test_half_steps_must_alternate_and_need_the_two_launch_step(meshes):
    s, mesh = meshes[2]
    with eng.Engine(mesh, "fp64", wavefront=-1) as e:
        with pytest.raises(eng.DGError) as ei:
            e.half_step(1)
        assert ei.value.code == -6
        e.half_step(0)
        with pytest.raises(eng.DGError) as ei:
            e.step(1)
        assert ei.value.code == -6
        e.half_step(1)
        assert e.steps_done == 1
        with pytest.raises(eng.DGError) as ei:
            e.halo_pack(0, 0)
        assert ei.value.code == -6
    m16 = dict(mesh)
    m16["source"] = np.repeat(np.asarray(mesh["source"]).reshape(-1, 2)[:1], 16, axis=0)
    m16["fun"] = np.repeat(np.asarray(mesh["fun"]).reshape(-1, 6)[:1], 16, axis=0)
    with eng.Engine(m16, "fp32") as e:
        assert e.stats()["kernel_family"] in (5, 6)
        with pytest.raises(eng.DGError) as ei:
            e.half_step(0)
        assert ei.value.code == -7
