"""A mesh split into parts on the GPU (domain decomposition through the C ABI).

All parts run as contexts on one device (`decompose.SplitRun` without a communicator: the halo
buffers are copied device to device on a transfer stream; with `torch.distributed` the same
buffers travel between GPUs).  Owned triangles compute what the whole mesh computes, so every
field and trace equals the undivided run bit for bit, in every precision, with the half steps
whole or in two parts around the transfers (`dg_gpu_half_step_part`), in the part's own
numbering (boundary, interior, ghosts) or the engine's Hilbert numbering.
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
    for shots in (1, 2, 3, 16):
        w = pkg.workloads.small_square(n_cells=16, steps=160, shots=shots)
        s = pkg.host.build_setup(w, full=True)
        out[shots] = (s, eng.mesh_from_setup(s))
    return out


CASES = [("fp64_ref", 1, 3), ("fp64", 2, 2), ("fp64", 3, 4), ("fp32", 1, 3), ("fp32", 2, 2),
         ("fp32_kahan", 3, 3), ("fp32", 16, 3), ("fp32", 3, 1)]


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("precision,shots,P", CASES)
def test_split_mesh_equals_whole_mesh(meshes, precision, shots, P, overlap):
    _split_equals_whole(meshes, precision, shots, P, overlap=overlap)


@pytest.mark.parametrize("precision,shots,P,kw", [("fp32", 1, 4, {"reorder": True}),
                                                  ("fp64", 3, 3, {"reorder": True}),
                                                  ("fp32", 3, 3, {"block_threads": 256}),
                                                  ("fp32", 1, 5, {"block_threads": 128})])
def test_split_parts_in_any_numbering_and_block_size(meshes, precision, shots, P, kw):
    """The parts of a half step are block windows over the engine's numbering: with the engine's
    own Hilbert order the boundary triangles are scattered (the boundary window then covers most
    blocks) and the result is still exact; likewise for other block sizes."""
    _split_equals_whole(meshes, precision, shots, P, overlap=True, **kw)


def _split_equals_whole(meshes, precision, shots, P, overlap, **kw):
    s, mesh = meshes[shots]
    steps = 150
    with eng.Engine(mesh, precision, wavefront=-1) as whole:
        whole.step(steps)
        want = {(f, m): whole.fetch(f, 0, m).reshape(-1, 6) for f in FIELDS for m in range(shots)}
        want_tr = {(c, m): whole.fetch(c, 0, m) for c in ("trace_x", "trace_z") for m in range(shots)}
    with dec.SplitRun(mesh, P, precision, overlap=overlap, **kw) as run:
        run.step(steps // 2)
        run.step(steps - steps // 2)
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


def test_half_step_parts_state(meshes):
    """A half step in parts: each part once, both parts before the other half, halo lists first."""
    s, mesh = meshes[2]
    B, I = eng.PART_BOUNDARY, eng.PART_INTERIOR
    with eng.Engine(mesh, "fp32", wavefront=-1) as e:
        with pytest.raises(eng.DGError) as ei:
            e.half_step_part(0, B)
        assert ei.value.code == -6                     # no halo lists
        e.halo_lists([], [])
        e.half_step_part(0, I)
        for bad in ((0, I), (1, B), (1, I)):
            with pytest.raises(eng.DGError) as ei:
                e.half_step_part(*bad)
            assert ei.value.code == -6
        for call in (lambda: e.half_step(0), lambda: e.half_step(1), lambda: e.step(1)):
            with pytest.raises(eng.DGError) as ei:
                call()
            assert ei.value.code == -6
        e.half_step_part(0, B)
        with pytest.raises(eng.DGError) as ei:
            e.half_step_part(0, I)                     # velocity half again
        assert ei.value.code == -6
        e.half_step_part(1, B)
        e.half_step_part(1, I)
        assert e.steps_done == 1
        e.half_step_part(0, eng.PART_ALL)
        e.half_step(1)
        e.step(3)
        assert e.steps_done == 5
        with pytest.raises(eng.DGError) as ei:
            e.half_step_part(0, 3)
        assert ei.value.code == -1


@pytest.mark.parametrize("overlap", [True, False])
def test_split_reference_path_with_rebuilt_operators(overlap):
    """Parts of 65,536 elements or more take the reference path with Dx, Dz rebuilt in the
    kernels; in half-step windows too they equal the undivided run bit for bit."""
    w = pkg.workloads.homogeneous_square(n_cells=265, steps=60, n_rec=266)
    s = pkg.host.build_setup(w, full=True)
    mesh = eng.mesh_from_setup(s)
    with eng.Engine(mesh, "fp64_ref", wavefront=-1) as whole:
        whole.step(50)
        want = [whole.fetch(f).reshape(-1, 6) for f in ("Vz", "Txx")] + [whole.fetch("trace_z")]
    with dec.SplitRun(mesh, 2, "fp64_ref", overlap=overlap) as run:
        assert min(p.own.size for p in run.parts) >= 65536
        run.step(50)
        got = [run.fetch(f) for f in ("Vz", "Txx")] + [run.traces("trace_z")]
    for a, b in zip(want, got):
        assert np.array_equal(a, b)
    assert np.abs(want[0]).max() > 0    # the field (the wave reaches no receiver in 50 steps)
