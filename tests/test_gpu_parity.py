"""GPU engine against the reference (golden fixtures) and the CPU oracle, through the C ABI.

Tolerances (relative L2 over all samples):
  DG_FP64_REF   bit-identical to the reference's OpenMP code (values compared with ==)
  DG_FP64       <= 1e-10   (geometric-factor form, FMA)
  DG_FP32       <= 1e-4    trace error against FP64
  DG_FP32_KAHAN <= 1e-4    and no worse than plain FP32 on the final fields
"""
import numpy as np
import pytest

from conftest import Golden, golden_names, pkg, rel_l2

import oracle

eng = pkg.engine
pytestmark = pytest.mark.gpu

FIELDS = ("Vx", "Vz", "Txx", "Tzz", "Txz")


def _engine(g: Golden, precision, **kw):
    a = g.setup_arrays()
    return eng.Engine(eng.mesh_from_setup(a), precision, **kw)


def _run_and_collect(e: eng.Engine, g: Golden, shot: int):
    snaps = {}
    for t0 in range(0, g.steps, g.snap_every):
        e.step(g.snap_every)
        t1 = t0 + g.snap_every
        snaps[t1] = (e.fetch("Vx", 0, shot), e.fetch("Vz", 0, shot))
    return snaps


@pytest.mark.parametrize("name", golden_names())
def test_fp64_ref_bit_identical_to_reference(name):
    g = Golden(name)
    with _engine(g, "fp64_ref") as e:
        for t0 in range(0, g.steps, g.snap_every):
            e.step(g.snap_every)
            t1 = t0 + g.snap_every
            for m in range(g.shots):
                assert np.array_equal(e.fetch("Vx", 0, m), g.z["shot%d_Vx%d" % (m, t1)]), (m, t1)
                assert np.array_equal(e.fetch("Vz", 0, m), g.z["shot%d_Vz%d" % (m, t1)]), (m, t1)
        for m in range(g.shots):
            assert np.array_equal(e.fetch("trace_x", 0, m), g.z["shot%d_rec_x" % m])
            assert np.array_equal(e.fetch("trace_z", 0, m), g.z["shot%d_rec_z" % m])
            for f in FIELDS:
                assert np.array_equal(e.fetch(f, 0, m), g.z["shot%d_final_%s" % (m, f)]), f


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-4), ("fp32_kahan", 1e-4)])
def test_compact_paths_against_reference(name, precision, tol):
    g = Golden(name)
    with _engine(g, precision) as e:
        e.step(g.steps)
        for m in range(g.shots):
            tx = e.fetch("trace_x", 0, m)
            tz = e.fetch("trace_z", 0, m)
            err = rel_l2(np.concatenate([tx, tz]), np.concatenate([g.z["shot%d_rec_x" % m], g.z["shot%d_rec_z" % m]]))
            assert err <= tol, (precision, m, err)
            for f in FIELDS:
                assert rel_l2(e.fetch(f, 0, m), g.z["shot%d_final_%s" % (m, f)]) <= 10 * tol, f


def test_kahan_not_worse_than_fp32():
    g = Golden("square_K288")
    errs = {}
    for p in ("fp32", "fp32_kahan"):
        with _engine(g, p) as e:
            e.step(g.steps)
            errs[p] = sum(rel_l2(e.fetch(f), g.z["shot0_final_%s" % f]) for f in FIELDS)
    assert errs["fp32_kahan"] <= errs["fp32"] * 1.05, errs


@pytest.mark.parametrize("precision", ["fp64_ref", "fp64", "fp32"])
def test_reordering_does_not_change_results(precision):
    g = Golden("slope_coupled")
    out = []
    for reorder in (False, True):
        with _engine(g, precision, reorder=reorder) as e:
            e.step(g.steps)
            out.append([e.fetch(f) for f in FIELDS] + [e.fetch("trace_x")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_block_sizes_and_graphs_agree():
    g = Golden("square_3shots")
    ref = None
    for block, graph in ((64, -1), (128, 7), (256, 0)):
        with _engine(g, "fp64", block_threads=block, graph_steps=graph) as e:
            e.step(g.steps)
            got = [e.fetch(f, 0, m) for m in range(g.shots) for f in FIELDS]
        if ref is None:
            ref = got
        else:
            for a, b in zip(ref, got):
                assert np.array_equal(a, b)


def test_multi_mesh_batch_matches_single_runs():
    gs = [Golden(n) for n in golden_names()]
    meshes = [eng.mesh_from_setup(g.setup_arrays()) for g in gs]
    with eng.Engine(meshes, "fp64") as e:
        e.step(max(g.steps for g in gs))
        batch = [[e.fetch(f, k, m) for m in range(g.shots) for f in FIELDS] for k, g in enumerate(gs)]
        traces = [[e.fetch("trace_x", k, m) for m in range(g.shots)] for k, g in enumerate(gs)]
    for k, g in enumerate(gs):
        with _engine(g, "fp64") as e:
            e.step(g.steps)
            single = [e.fetch(f, 0, m) for m in range(g.shots) for f in FIELDS]
            for m in range(g.shots):
                assert np.array_equal(traces[k][m], e.fetch("trace_x", 0, m))
        for a, b in zip(batch[k], single):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
def test_fp32_multi_mesh_batch_matches_single_runs(precision):
    """One launch over meshes of 1, 1 and 3 shots (the 3 padded to 4) equals separate runs."""
    gs = [Golden(n) for n in golden_names()]
    meshes = [eng.mesh_from_setup(g.setup_arrays()) for g in gs]
    with eng.Engine(meshes, precision) as e:
        assert e.stats()["kernel_family"] == 4
        e.step(max(g.steps for g in gs))
        batch = [[e.fetch(f, k, m) for m in range(g.shots) for f in FIELDS] for k, g in enumerate(gs)]
        tr = [e.fetch_traces(0, g.steps, mesh=k) for k, g in enumerate(gs)]
    for k, g in enumerate(gs):
        assert tr[k][0].shape == (g.shots, g.steps, g.z["rec"].shape[0])
        with _engine(g, precision) as e:
            e.step(g.steps)
            single = [e.fetch(f, 0, m) for m in range(g.shots) for f in FIELDS]
            for m in range(g.shots):
                assert np.array_equal(tr[k][0][m], e.fetch("trace_x", 0, m))
                ref = np.concatenate([g.z["shot%d_rec_x" % m], g.z["shot%d_rec_z" % m]])
                assert rel_l2(np.concatenate([tr[k][0][m], tr[k][1][m]]), ref) <= 1e-4
        for a, b in zip(batch[k], single):
            assert np.array_equal(a, b)


def test_checkpoint_restore_continues_identically():
    """Fields fetched at step 80 and loaded into a second context continue bit-identically."""
    g = Golden("square_K288")
    with _engine(g, "fp64_ref") as a, _engine(g, "fp64_ref") as b:
        a.step(80)
        state = [a.fetch(f) for f in FIELDS]
        a.step(g.steps - 80)
        final = [a.fetch(f) for f in FIELDS]
        # b runs its first 80 steps without a source (state stays zero), then takes the checkpoint
        b.set_wavelet(0, np.zeros(80))
        b.step(80)
        assert not np.any(b.fetch("Vz"))
        for f, v in zip(FIELDS, state):
            b.load(f, v)
        b.step(g.steps - 80)
        for x, y in zip(final, [b.fetch(f) for f in FIELDS]):
            assert np.array_equal(x, y)
        b.reset()
        assert b.steps_done == 0 and not np.any(b.fetch("Vx"))


def test_host_wavelet_update_equals_table():
    g = Golden("square_K288")
    a = g.setup_arrays()
    with _engine(g, "fp64") as e1, _engine(g, "fp64") as e2:
        e1.step(g.steps)
        for t0 in range(0, g.steps, 50):
            e2.set_wavelet(t0, a["wavelet"][t0:t0 + 50])
            e2.step(50)
        assert np.array_equal(e1.fetch("trace_z"), e2.fetch("trace_z"))


def test_linearity_power_of_two():
    """Doubling the source doubles every value: exactly in FP64; in FP32 up to the rounding of
    values that underflow ahead of the wave front (relative L2 1e-6)."""
    g = Golden("slope_coupled")
    a = g.setup_arrays()
    for p in ("fp64_ref", "fp64", "fp32"):
        m1 = eng.mesh_from_setup(a)
        m2 = eng.mesh_from_setup(a, wavelet=2.0 * a["wavelet"])
        with eng.Engine(m1, p) as e1, eng.Engine(m2, p) as e2:
            e1.step(g.steps)
            e2.step(g.steps)
            for what in ("trace_x", "Txz"):
                x, y = 2.0 * e1.fetch(what), e2.fetch(what)
                if p == "fp32":
                    assert rel_l2(x, y) <= 1e-6
                else:
                    assert np.array_equal(x, y)


def test_energy_fp32_tracks_fp64():
    g = Golden("slope_coupled")
    en = {}
    for p in ("fp64", "fp32", "fp32_kahan"):
        with _engine(g, p) as e:
            vals = []
            for _ in range(g.steps // 25):
                e.step(25)
                vals.append(e.fetch("energy"))
            en[p] = np.array(vals)
    assert np.all(en["fp64"] >= 0) and en["fp64"].max() > 0
    for p in ("fp32", "fp32_kahan"):
        drift = np.max(np.abs(en[p] - en["fp64"])) / en["fp64"].max()
        assert drift < 1e-4, (p, drift)


def test_errors_are_reported_not_raised_on_device():
    g = Golden("square_K288")
    with _engine(g, "fp64", watchdog_every=10) as e:
        with pytest.raises(eng.DGError) as ei:
            e.step(g.steps + 1)
        assert ei.value.code == -6  # DG_ERR_STATE: past the wavelet table, nothing ran
        assert e.steps_done == 0
        e.step(10)
        bad = e.fetch("Vx")
        bad[7] = np.nan
        e.load("Vx", bad)
        with pytest.raises(eng.DGError) as ei:
            e.step(10)
        assert ei.value.code == -5  # DG_ERR_NONFINITE from the watchdog


def test_invalid_maps_rejected_on_host():
    g = Golden("square_K288")
    a = g.setup_arrays()
    m = eng.mesh_from_setup(a)
    m["Neighbor"] = m["Neighbor"].copy()
    m["Neighbor"].ravel()[5] = 10 ** 6
    with pytest.raises(eng.DGError) as ei:
        eng.Engine(m, "fp64")
    assert ei.value.code == -4
    m = eng.mesh_from_setup(a)
    t = m["Triangle"].copy().reshape(-1, 3)
    t[3, [1, 2]] = t[3, [2, 1]]
    m["Triangle"] = t
    with pytest.raises(eng.DGError) as ei:
        eng.Engine(m, "fp64")
    assert ei.value.code == -9


def _repeat_shots(a, S, pattern=(0, 1, 2)):
    """Mesh dict with S shots cycling through the fixture's shots."""
    m = eng.mesh_from_setup(a)
    idx = [pattern[i % len(pattern)] for i in range(S)]
    m["source"] = np.ascontiguousarray(a["source"].reshape(-1, 2)[idx])
    m["fun"] = np.ascontiguousarray(a["fun"].reshape(-1, 6)[idx])
    return m, idx


@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
@pytest.mark.parametrize("S", [2, 4, 64])
def test_two_shot_kernels_against_reference(precision, S):
    """Packed FP32x2 kernels (element-major layout) against the reference's traces."""
    g = Golden("square_3shots")
    m, idx = _repeat_shots(g.setup_arrays(), S)
    with eng.Engine(m, precision, variant=2) as e:
        e.step(g.steps)
        for s in (0, 1, S - 1):
            ref = np.concatenate([g.z["shot%d_rec_x" % idx[s]], g.z["shot%d_rec_z" % idx[s]]])
            got = np.concatenate([e.fetch("trace_x", 0, s), e.fetch("trace_z", 0, s)])
            assert rel_l2(got, ref) <= 1e-4, (s, rel_l2(got, ref))
            assert rel_l2(e.fetch("Txz", 0, s), g.z["shot%d_final_Txz" % idx[s]]) <= 1e-3


@pytest.mark.parametrize("persistent", ["0", "1"])
@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
@pytest.mark.parametrize("S,block,margin", [(8, 64, None), (2, 256, 0), (64, 128, 0), (128, 256, None),
                                            (16, 64, 3), (15, 64, None), (1, 64, None), (1, 128, 0)])
def test_wavefront_step_equals_two_pass_step(precision, S, block, margin, persistent, monkeypatch):
    """One launch per step (k_step_wave / k_step_wave_p, RCM order) gives the same bits as the
    two launches, for warps covering 64 elements (one shot, two elements per thread), many
    elements (2 shots), one element (64) and half an element (128), an odd shot count padded
    with a silent shot (15 -> 16), with no lag margin (every stress update waits on velocity
    updates still in flight), one block per ticket and resident blocks looping over the
    tickets."""
    monkeypatch.setenv("DG_WAVE_PERSISTENT", persistent)
    if margin is not None:
        monkeypatch.setenv("DG_WAVE_MARGIN", str(margin))
    g = Golden("square_3shots")
    m, _ = _repeat_shots(g.setup_arrays(), S)
    out = []
    for wf in (-1, 1):
        # the two-launch side on the same packed bodies (two shots would otherwise take the
        # one-(element, shot)-per-thread kernels, whose rounding differs)
        with eng.Engine(m, precision, wavefront=wf, block_threads=block, variant=2) as e:
            assert e.stats()["kernel_family"] == ((6 if persistent == "1" else 5) if wf == 1 else (2 if S > 1 else 3))
            e.step(g.steps)
            out.append([e.fetch(f, 0, s) for s in (0, S // 2, S - 1) for f in FIELDS] +
                       [e.fetch("trace_x", 0, s) for s in range(S)] + [e.fetch("trace_z", 0, S - 1)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_wavefront_wait_limit_reports_timeout_and_context_recovers():
    """A stress update made to wait on a flag that nothing publishes gives up after its limit:
    the step returns DG_ERR_TIMEOUT instead of hanging, and after a reset the same context steps
    exactly like a fresh one."""
    g = Golden("square_3shots")
    m, _ = _repeat_shots(g.setup_arrays(), 8)
    with eng.Engine(m, "fp32", wavefront=1, block_threads=64) as fresh:
        fresh.step(20)
        want = [fresh.fetch(f, 0, s) for s in (0, 7) for f in FIELDS] + [fresh.fetch("trace_z", 0, 7)]
    with eng.Engine(m, "fp32", wavefront=1, block_threads=64) as e:
        e.step(2)
        e.debug_stall_wave(5)
        with pytest.raises(eng.DGError) as ei:
            e.step(3)
        assert ei.value.code == -10
        e.debug_stall_wave(-1)
        e.reset()
        e.step(20)
        got = [e.fetch(f, 0, s) for s in (0, 7) for f in FIELDS] + [e.fetch("trace_z", 0, 7)]
    for a, b in zip(want, got):
        assert np.array_equal(a, b)
    with eng.Engine(m, "fp32", wavefront=-1) as e:
        with pytest.raises(eng.DGError) as ei:
            e.debug_stall_wave(0)
        assert ei.value.code == -7


@pytest.mark.parametrize("precision,S", [("fp64", 3), ("fp32", 16)])
def test_snapshots_while_stepping_equal_step_then_fetch(precision, S):
    """dg_gpu_step_snapshots hands over the same Vx/Vz as stepping `every` steps and fetching,
    at the same steps, twice in a row (the rings are reused), and leaves the state where
    dg_gpu_step would."""
    g = Golden("square_3shots")
    m, _ = _repeat_shots(g.setup_arrays(), S)
    every, n = 15, 60  # 120 of the fixture's 150 steps
    got = []
    with eng.Engine(m, precision) as a, eng.Engine(m, precision) as b:
        for _ in range(2):
            a.step_snapshots(n, every, lambda step, vx, vz: got.append((step, vx, vz)), shot=S - 1)
        want = []
        for _ in range(2 * n // every):
            b.step(every)
            want.append((b.steps_done, b.fetch("Vx", 0, S - 1).reshape(-1, 6), b.fetch("Vz", 0, S - 1).reshape(-1, 6)))
        assert a.steps_done == b.steps_done == 2 * n
        assert np.array_equal(a.fetch("Txz", 0, 0), b.fetch("Txz", 0, 0))
    assert [x[0] for x in got] == [x[0] for x in want] == list(range(every, 2 * n + 1, every))
    for (_, vx, vz), (_, wx, wz) in zip(got, want):
        assert np.array_equal(vx, wx) and np.array_equal(vz, wz)
    assert np.any(got[-1][1])


@pytest.mark.parametrize("precision,S", [("fp32", 16), ("fp32_kahan", 16), ("fp64", 3)])
def test_autotuned_schedule_gives_the_same_bits_and_is_cached(precision, S, tmp_path):
    """The autotuner (block size; for the wavefront step also one block per ticket or resident
    blocks, and the lag margin) changes speed only; a second context reads its choice back."""
    g = Golden("square_3shots")
    m, _ = _repeat_shots(g.setup_arrays(), S)
    cache = str(tmp_path / "tune.txt")
    out, stats = [], []
    for kw in ({}, {"autotune": True, "tune_cache": cache}, {"autotune": True, "tune_cache": cache}):
        with eng.Engine(m, precision, **kw) as e:
            stats.append(e.stats())
            e.step(g.steps)
            out.append([e.fetch(f, 0, s) for s in (0, S - 1) for f in FIELDS] + [e.fetch("trace_z", 0, S - 1)])
    for got in out[1:]:
        for a, b in zip(out[0], got):
            assert np.array_equal(a, b)
    assert len(open(cache).read().splitlines()) == 1
    assert stats[1]["block_threads"] == stats[2]["block_threads"]
    assert stats[1]["kernel_family"] == stats[2]["kernel_family"]


@pytest.mark.parametrize("precision,S", [("fp32", 4), ("fp32", 6), ("fp32_kahan", 5), ("fp32", 16)])
def test_plane_major_and_element_major_packed_kernels_give_the_same_bits(precision, S):
    """The packed two-shot bodies on plane-major state (family 7) and on element-major state
    (family 2) do the same arithmetic: fields and traces agree bit for bit."""
    g = Golden("slope_coupled")
    m, _ = _repeat_shots(g.setup_arrays(), S, pattern=(0,))
    out = []
    for variant, fam in ((2, 2), (3, 7)):
        with eng.Engine(m, precision, variant=variant, wavefront=-1) as e:
            assert e.stats()["kernel_family"] == fam
            e.step(g.steps)
            out.append([e.fetch(f, 0, s) for s in (0, S - 1) for f in FIELDS] + [e.fetch("trace_z", 0, S - 1)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_two_shot_and_one_shot_kernels_agree():
    g = Golden("slope_coupled")
    m, _ = _repeat_shots(g.setup_arrays(), 4, pattern=(0,))
    out = []
    for variant in (1, 2):
        with eng.Engine(m, "fp32", variant=variant) as e:
            e.step(g.steps)
            out.append([e.fetch(f, 0, s) for s in range(4) for f in FIELDS] + [e.fetch("trace_z", 0, 3)])
    for a, b in zip(*out):
        assert rel_l2(a, b) <= 2e-5


@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
def test_two_element_kernels_agree_with_one_element(precision):
    """One shot: packed kernels (two elements per thread) against one element per thread."""
    g = Golden("slope_coupled")  # K = 296: the last pair straddles the padding
    out = []
    for variant in (1, 2):
        with _engine(g, precision, variant=variant) as e:
            e.step(g.steps)
            out.append([e.fetch(f) for f in FIELDS] + [e.fetch("trace_x"), e.fetch("trace_z")])
    for a, b in zip(*out):
        assert rel_l2(a, b) <= 2e-5


def test_two_shot_checkpoint_restore():
    g = Golden("square_K288")
    m, _ = _repeat_shots(g.setup_arrays(), 2, pattern=(0,))
    with eng.Engine(m, "fp32", variant=2) as a, eng.Engine(m, "fp32", variant=2) as b:
        a.step(80)
        state = [[a.fetch(f, 0, s) for f in FIELDS] for s in range(2)]
        a.step(g.steps - 80)
        b.set_wavelet(0, np.zeros(80))
        b.step(80)
        for s in range(2):
            for f, v in zip(FIELDS, state[s]):
                b.load(f, v, 0, s)
        b.step(g.steps - 80)
        for s in range(2):
            for f in FIELDS:
                assert np.array_equal(a.fetch(f, 0, s), b.fetch(f, 0, s))
            assert np.array_equal(a.fetch("trace_x", 0, s)[80:], b.fetch("trace_x", 0, s)[80:])


def test_poly_model_against_oracle():
    """A model meshed from a planar straight-line graph (two regions, acoustic over elastic)."""
    from test_poly_mesh_cpu import L_SHAPE
    w = pkg.workloads.poly_model(L_SHAPE, {1: (4000.0, 2300.0, 2500.0), 2: (1500.0, 0.0, 1000.0)},
                                 src=[(1500.0, 500.0)], rec=[(x, 2400.0) for x in (100.0, 800.0, 1600.0)],
                                 h=120.0, fp=8.0, steps=400)
    s = pkg.host.build_setup(w, full=True)
    o = oracle.Oracle.from_setup(s)
    rx, rz = o.run(0, w.steps, threads=0)
    with eng.Engine(eng.mesh_from_setup(s), "fp64_ref") as e:
        e.step(w.steps)
        assert np.array_equal(e.fetch("trace_z"), rz)
        assert np.array_equal(e.fetch("Txz"), o.fields[4])
    with eng.Engine(eng.mesh_from_setup(s), "fp64") as e:
        e.step(w.steps)
        assert rel_l2(np.concatenate([e.fetch("trace_x").ravel(), e.fetch("trace_z").ravel()]),
                      np.concatenate([rx.ravel(), rz.ravel()])) <= 1e-10
    assert np.abs(rz).max() > 0


@pytest.mark.parametrize("precision", ["fp32", "fp32_kahan"])
def test_whole_run_in_one_graph(precision):
    """graph_steps equal to the run's steps puts the whole run in one captured graph (the 64-shot
    configuration's "4,000 steps as one CUDA graph"): the same bits as the default 100-step graphs,
    on the wavefront step (16 shots)."""
    g = Golden("square_3shots")
    m, _ = _repeat_shots(g.setup_arrays(), 16)
    out = []
    for gs in (0, g.steps):
        with eng.Engine(m, precision, graph_steps=gs) as e:
            assert e.stats()["kernel_family"] == 6
            assert e.stats()["graph_steps"] == (gs or min(100, g.steps))
            e.step(g.steps)
            out.append([e.fetch(f, 0, s) for s in (0, 15) for f in FIELDS] + [e.fetch("trace_z", 0, 15)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
