"""The FP32 batch of meshes in one persistent cooperative launch (`k_step_mx_p`, family 8)
against two launches per step (`k_velocity_mx` / `k_stress_mx`, family 4).

Every work block runs the same body in both forms and a grid barrier separates the halves, so
fields and traces are equal bit for bit: stepped in one call or in chunks, timed, with
snapshots, and after the autotuner chose between the two.  The meshes differ in shot count (the
one-element-pair, one-(element, shot), element-major and plane-major packed bodies) and in step
count (a mesh past its last step does nothing).
"""
import numpy as np
import pytest

from conftest import pkg

eng = pkg.engine
pytestmark = pytest.mark.gpu
FIELDS = ("Vx", "Vz", "Txx", "Tzz", "Txz")
SPEC = ((12, 150, 1), (16, 120, 2), (10, 90, 3), (14, 150, 16), (9, 150, 6))


@pytest.fixture(scope="module")
def meshes():
    out = []
    for n_cells, steps, shots in SPEC:
        w = pkg.workloads.small_square(n_cells=n_cells, steps=steps, shots=shots)
        out.append(eng.mesh_from_setup(pkg.host.build_setup(w, full=False), with_ref_ops=False))
    return out


def _run(meshes, monkeypatch, precision, persistent, chunks=(150,), timed=False, **kw):
    monkeypatch.setenv("DG_MX_PERSISTENT", "1" if persistent else "0")
    with eng.Engine(meshes, precision, **kw) as e:
        fam = e.stats()["kernel_family"]
        for c in chunks:
            (e.step_timed if timed else e.step)(c)
        assert e.steps_done == sum(chunks)
        fields = [e.fetch(f, k, m) for k, (_, _, S) in enumerate(SPEC) for m in range(S) for f in FIELDS]
        traces = [e.fetch_traces(0, steps, mesh=k) for k, (_, steps, _) in enumerate(SPEC)]
    return fam, fields, traces


def _same(a, b):
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)
    for (x0, z0), (x1, z1) in zip(a[2], b[2]):
        assert np.array_equal(x0, x1) and np.array_equal(z0, z1)


@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
def test_persistent_batch_equals_two_launches(meshes, monkeypatch, precision):
    two = _run(meshes, monkeypatch, precision, False)
    one = _run(meshes, monkeypatch, precision, True)
    assert two[0] == 4 and one[0] == 8
    assert np.abs(one[2][0][1]).max() > 0
    _same(two, one)


def test_persistent_batch_in_chunks_timed_and_block_sizes(meshes, monkeypatch):
    ref = _run(meshes, monkeypatch, "fp32", False)
    _same(ref, _run(meshes, monkeypatch, "fp32", True, chunks=(1, 7, 42, 100)))
    _same(ref, _run(meshes, monkeypatch, "fp32", True, chunks=(3, 147), timed=True))
    for b in (128, 256):
        _same(ref, _run(meshes, monkeypatch, "fp32", True, block_threads=b))


def test_persistent_batch_snapshots_and_autotune(meshes, monkeypatch):
    ref = _run(meshes, monkeypatch, "fp32", False)
    monkeypatch.setenv("DG_MX_PERSISTENT", "1")
    seen = []
    with eng.Engine(meshes, "fp32") as e:
        e.step_snapshots(150, 50, lambda step, vx, vz: seen.append((step, vx.copy())), mesh=3, shot=5)
        assert [s for s, _ in seen] == [50, 100, 150]
        assert np.array_equal(seen[-1][1].ravel(), ref[1][(1 + 2 + 3) * 5 + 5 * 5])
    tuned = _run(meshes, monkeypatch, "fp32", True, autotune=True)
    assert tuned[0] in (4, 8)
    _same(ref, tuned)


def test_persistent_batch_barrier_limit_reports_timeout(meshes, monkeypatch):
    """A grid barrier whose wait runs out (the test hook makes it wait for one block more than
    the grid holds) ends the launch with DG_ERR_TIMEOUT; after a reset the context steps exactly
    as a fresh one."""
    ref = _run(meshes, monkeypatch, "fp32", False)
    monkeypatch.setenv("DG_MX_PERSISTENT", "1")
    with eng.Engine(meshes, "fp32") as e:
        e.step(5)
        e.debug_stall_wave(0)
        with pytest.raises(eng.DGError) as ei:
            e.step(3)
        assert ei.value.code == -10
        e.debug_stall_wave(-1)
        e.reset()
        e.step(150)
        fields = [e.fetch(f, k, m) for k, (_, _, S) in enumerate(SPEC) for m in range(S) for f in FIELDS]
    for x, y in zip(ref[1], fields):
        assert np.array_equal(x, y)


def test_all_meshes_trace_fetch_and_wavelet(meshes):
    """DG_ALL_MESHES: one call fetches every mesh's traces (blocks in mesh order) and one call
    sets every mesh's wavelet samples; both equal the per-mesh calls."""
    rng = np.random.default_rng(4)
    n = 80
    new = rng.normal(size=(len(SPEC), n))
    out = []
    for together in (False, True):
        with eng.Engine(meshes, "fp32") as e:
            if together:
                e.set_wavelet(0, new.ravel(), mesh=eng.ALL_MESHES)
            else:
                for k in range(len(SPEC)):
                    e.set_wavelet(0, new[k], mesh=k)
            e.step(120)
            per = [e.fetch_traces(0, n, mesh=k) for k in range(len(SPEC))]
            ax, az = e.fetch_traces(0, n, mesh=eng.ALL_MESHES)
            assert np.array_equal(ax, np.concatenate([p[0].ravel() for p in per]))
            assert np.array_equal(az, np.concatenate([p[1].ravel() for p in per]))
            out.append(az)
    assert np.array_equal(out[0], out[1]) and np.abs(out[0]).max() > 0


@pytest.mark.parametrize("precision,wave", [("fp32", -1), ("fp32", 0), ("fp64", -1)])
def test_async_steps_equal_synchronous_steps(meshes, precision, wave):
    """dg_gpu_step_async + dg_gpu_synchronize give the steps of dg_gpu_step; fetches after
    enqueued steps wait for them by themselves."""
    out = []
    for use_async in (False, True):
        with eng.Engine(meshes[3], precision, wavefront=wave) as e:   # 16 shots: wavefront when on
            if use_async:
                e.step_async(40)
                e.step_async(60)
                e.synchronize()
                e.step_async(50)
            else:
                e.step(150)
            out.append([e.fetch("Vz", 0, s) for s in (0, 15)] + [e.fetch("trace_z", 0, 15)])
            assert e.steps_done == 150
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision,wave", [("fp32", -1), ("fp32", 0), ("fp64", -1)])
def test_overlapped_chunks_equal_synchronous_chunks(meshes, precision, wave):
    """The end-to-end loop with overlap: the next chunk's wavelet uploaded while the current chunk
    steps (samples no enqueued step reads), its steps enqueued, then the previous chunk's traces
    fetched while they run, gives the traces and fields of the synchronous loop bit for bit."""
    chunk, n_chunks = 30, 5
    rng = np.random.default_rng(7)
    wav = rng.standard_normal(chunk * n_chunks) * 1e-2
    out = []
    for overlap in (False, True):
        with eng.Engine(meshes[3], precision, wavefront=wave) as e:   # 16 shots
            got = [None] * n_chunks
            for c in range(n_chunks):
                e.set_wavelet(c * chunk, wav[c * chunk:(c + 1) * chunk])
                if overlap:
                    e.step_async(chunk)
                    if c > 0:
                        got[c - 1] = e.fetch_traces((c - 1) * chunk, chunk)
                else:
                    e.step(chunk)
                    got[c] = e.fetch_traces(c * chunk, chunk)
            if overlap:
                got[-1] = e.fetch_traces((n_chunks - 1) * chunk, chunk)
                e.synchronize()
            out.append([np.concatenate([g[i] for g in got], axis=1) for i in (0, 1)] +
                       [e.fetch("Vz", 0, s) for s in (0, 15)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    assert np.abs(out[0][1]).max() > 0


@pytest.mark.parametrize("persistent", [True, False])
def test_overlapped_chunks_every_mesh(meshes, monkeypatch, persistent):
    """The same overlapped loop over the whole batch (one wavelet upload and one trace fetch for
    every mesh, DG_ALL_MESHES), in the persistent cooperative launch and in two launches a step:
    a fetch's gather on the copy stream runs beside the next chunk's grid."""
    monkeypatch.setenv("DG_MX_PERSISTENT", "1" if persistent else "0")
    chunk, n_chunks = 30, 3
    rng = np.random.default_rng(11)
    wav = rng.standard_normal((len(SPEC), chunk * n_chunks)) * 1e-2
    out = []
    for overlap in (False, True):
        with eng.Engine(meshes, "fp32") as e:
            got = [None] * n_chunks
            for c in range(n_chunks):
                e.set_wavelet(c * chunk, wav[:, c * chunk:(c + 1) * chunk].ravel(), mesh=eng.ALL_MESHES)
                if overlap:
                    e.step_async(chunk)
                    if c > 0:
                        got[c - 1] = e.fetch_traces((c - 1) * chunk, chunk, mesh=eng.ALL_MESHES)
                else:
                    e.step(chunk)
                    got[c] = e.fetch_traces(c * chunk, chunk, mesh=eng.ALL_MESHES)
            if overlap:
                got[-1] = e.fetch_traces((n_chunks - 1) * chunk, chunk, mesh=eng.ALL_MESHES)
                e.synchronize()
            out.append([g[i] for g in got for i in (0, 1)] + [e.fetch("Vz", k, 0) for k in range(len(SPEC))])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_wavelet_update_after_enqueued_steps(meshes, precision):
    """Samples that enqueued steps read are replaced only after those steps (the copy follows
    them); a fetch of a window that no single step call ends at waits for all enqueued work."""
    new = np.full(40, 5e-3)
    out = []
    for use_async in (False, True):
        with eng.Engine(meshes[3], precision) as e:
            if use_async:
                e.step_async(25)
                e.step_async(15)
                e.set_wavelet(20, new)         # steps 20..39 are in flight: they keep the old samples
                e.step_async(40)
                tr = e.fetch_traces(10, 50)   # ends inside the second 40-step call
                e.synchronize()
            else:
                e.step(40)
                e.set_wavelet(20, new)
                e.step(40)
                tr = e.fetch_traces(10, 50)
            out.append(list(tr) + [e.fetch("Vz", 0, 3)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fetch_every_shot_at_once(meshes, precision):
    """DG_ALL_SHOTS: one call returns a field of every shot of a mesh, equal to the per-shot calls."""
    with eng.Engine(meshes[3], precision) as e:     # 16 shots
        e.step(60)
        for f in ("Vx", "Txz"):
            every = e.fetch(f, 0, eng.ALL_SHOTS)
            assert every.shape == (16, e.info[0]["K"] * 6)
            for s in range(16):
                assert np.array_equal(every[s], e.fetch(f, 0, s))
        assert np.abs(every).max() > 0
