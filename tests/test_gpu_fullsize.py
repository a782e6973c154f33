"""Full-size GPU checks of the benchmark configurations, against the CPU oracle.

* 20,000-element square, 2,000 steps: reference-operator path bit-identical to the CPU oracle,
  FP64 within 1e-10, FP32 and FP32-Kahan within 1e-4 (traces).
* coupled acoustic-elastic slope (~400k elements): bit-identical reference-operator path over the
  first 100 steps; FP64 within 1e-10 and FP32 within 1e-4 of the oracle over all 6,000 steps
  (traces and final fields); FP32 / FP32-Kahan within 1e-4 of FP64; energy drift.
* 2M-element random medium: FP64 within 1e-10 and FP32 / FP32-Kahan within 1e-4 of the oracle
  after 1,000 steps (every field: no wave reaches a receiver that early); over 10,000 steps
  FP32-Kahan and FP32 against FP64 (traces, energy).
* 200k elements x 64 shots: one shot of the batch against the oracle over 1,000 steps (FP64
  within 1e-10, FP32 within 1e-4); FP32 against FP64; a shot of the batch equals the same shot
  run alone (FP64, bit for bit); doubling the wavelet doubles the traces.
* uneven meshes with their own dt and step counts in one context: three meshes over their whole
  1.5 s runs against the oracle; twelve against FP64; each mesh stops at its own last step.

The long oracle runs flush subnormal values to zero (Oracle.run(flush_subnormals=True)): values
below 2^-1022 ahead of the wave front otherwise slow the host several times, and they are far
below every tolerance used with it.  Bit-exact comparisons never use that mode.
"""
import numpy as np
import pytest

from conftest import pkg, rel_l2

import oracle

eng = pkg.engine
W = pkg.workloads
pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _traces(e, mesh=0, shot=0):
    return np.concatenate([e.fetch("trace_x", mesh, shot).ravel(), e.fetch("trace_z", mesh, shot).ravel()])


def _energy_series(e, steps, every):
    out = []
    for _ in range(steps // every):
        e.step(every)
        out.append(e.fetch("energy"))
    return np.array(out)


def test_square_2000_steps_against_oracle():
    w = W.homogeneous_square(steps=2000)
    s = pkg.host.build_setup(w)
    o = oracle.Oracle.from_setup(s)
    rx, rz = o.run(0, w.steps, threads=0)
    ref = np.concatenate([rx.ravel(), rz.ravel()])
    fields = [f.copy() for f in o.fields]
    for p, tol in (("fp64_ref", 0.0), ("fp64", 1e-10), ("fp32", 1e-4), ("fp32_kahan", 1e-4)):
        with eng.Engine(eng.mesh_from_setup(s), p) as e:
            e.step(w.steps)
            got = _traces(e)
            if tol == 0.0:
                assert np.array_equal(got, ref)
                for k, f in enumerate(("Vx", "Vz", "Txx", "Tzz", "Txz")):
                    assert np.array_equal(e.fetch(f), fields[k])
            else:
                assert rel_l2(got, ref) <= tol, (p, rel_l2(got, ref))


@pytest.fixture(scope="module")
def slope():
    w = W.coupled_slope(steps=6000)
    return w, pkg.host.build_setup(w, full=True, n_steps=6000)


def test_slope_fp64_against_oracle(slope):
    w, s = slope
    o = oracle.Oracle.from_setup(s)
    rx, rz = o.run(0, 100, threads=0)
    with eng.Engine(eng.mesh_from_setup(s), "fp64") as e:
        e.step(100)
        assert rel_l2(_traces(e), np.concatenate([rx.ravel(), rz.ravel()])) <= 1e-10
    with eng.Engine(eng.mesh_from_setup(s), "fp64_ref") as e:
        e.step(100)
        assert np.array_equal(e.fetch("trace_z"), rz)


FIELDS = ("Vx", "Vz", "Txx", "Tzz", "Txz")


def test_slope_all_steps_against_oracle(slope):
    """The coupled slope over its whole 6,000-step run, against the oracle: FP64 within 1e-10 and
    FP32 within 1e-4, on every trace sample and on the five final fields."""
    w, s = slope
    o = oracle.Oracle.from_setup(s)
    rx, rz = o.run(0, w.steps, threads=0, flush_subnormals=True)
    ref = np.concatenate([rx.ravel(), rz.ravel()])
    assert np.abs(ref).max() > 1e-12  # the wave has arrived (a precursor alone is far smaller)
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    for p, tol in (("fp64", 1e-10), ("fp32", 1e-4)):
        with eng.Engine(m, p) as e:
            e.step(w.steps)
            assert rel_l2(_traces(e), ref) <= tol, (p, rel_l2(_traces(e), ref))
            for k, f in enumerate(FIELDS):
                assert rel_l2(e.fetch(f), o.fields[k]) <= tol, (p, f, rel_l2(e.fetch(f), o.fields[k]))


def test_slope_fp32_full_run(slope):
    w, s = slope
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    res = {}
    for p in ("fp64", "fp32", "fp32_kahan"):
        with eng.Engine(m, p) as e:
            en = _energy_series(e, w.steps, 500)
            res[p] = (_traces(e), en)
    t64, e64 = res["fp64"]
    assert np.all(np.isfinite(t64)) and np.abs(t64).max() > 0
    for p in ("fp32", "fp32_kahan"):
        assert rel_l2(res[p][0], t64) <= 1e-4, (p, rel_l2(res[p][0], t64))
        assert np.max(np.abs(res[p][1] - e64)) / e64.max() <= 1e-4


def test_random_medium_against_oracle():
    """The 2M-element random medium after 1,000 steps against the oracle, every field: FP64 within
    1e-10, FP32 and FP32-Kahan within 1e-4."""
    steps = 1000
    w = W.random_medium(steps=steps)
    s = pkg.host.build_setup(w, full=True, n_steps=steps)
    o = oracle.Oracle.from_setup(s)
    o.run(0, steps, threads=0, record=False, flush_subnormals=True)
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    for p, tol in (("fp64", 1e-10), ("fp32", 1e-4), ("fp32_kahan", 1e-4)):
        with eng.Engine(m, p) as e:
            e.step(steps)
            for k, f in enumerate(FIELDS):
                assert np.abs(o.fields[k]).max() > 0
                assert rel_l2(e.fetch(f), o.fields[k]) <= tol, (p, f, rel_l2(e.fetch(f), o.fields[k]))


def test_random_medium_kahan_and_fp32_against_fp64():
    w = W.random_medium(steps=10000)
    s = pkg.host.build_setup(w, full=False)
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    res = {}
    for p in ("fp64", "fp32_kahan", "fp32"):
        with eng.Engine(m, p) as e:
            en = _energy_series(e, w.steps, 2000)
            res[p] = (_traces(e), en)
    t64, e64 = res["fp64"]
    err = {p: rel_l2(res[p][0], t64) for p in ("fp32", "fp32_kahan")}
    assert err["fp32_kahan"] <= 1e-4 and err["fp32"] <= 1e-4, err
    assert err["fp32_kahan"] <= err["fp32"] * 1.05, err
    for p in ("fp32", "fp32_kahan"):
        assert np.max(np.abs(res[p][1] - e64)) / e64.max() <= 1e-4


def test_multishot_batch_properties():
    w = W.layered_multishot(steps=1000)
    s = pkg.host.build_setup(w, full=True)
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    # one shot of the batch against the oracle's run of that shot alone
    o = oracle.Oracle.from_setup(s)
    rx, rz = o.run(17, w.steps, threads=0, flush_subnormals=True)
    ref17 = np.concatenate([rx.ravel(), rz.ravel()])
    assert np.abs(ref17).max() > 1e-12
    with eng.Engine(m, "fp32") as e32, eng.Engine(m, "fp64") as e64:
        e32.step(w.steps)
        e64.step(w.steps)
        assert rel_l2(_traces(e64, 0, 17), ref17) <= 1e-10, rel_l2(_traces(e64, 0, 17), ref17)
        assert rel_l2(_traces(e32, 0, 17), ref17) <= 1e-4, rel_l2(_traces(e32, 0, 17), ref17)
        for k, f in enumerate(FIELDS):
            assert rel_l2(e64.fetch(f, 0, 17), o.fields[k]) <= 1e-10, f
            assert rel_l2(e32.fetch(f, 0, 17), o.fields[k]) <= 1e-4, f
        for shot in (0, 17, 63):
            assert rel_l2(_traces(e32, 0, shot), _traces(e64, 0, shot)) <= 1e-4
        batch_shot = _traces(e64, 0, 17)
        batch_field = e64.fetch("Txz", 0, 17)
    one = dict(m)
    one["source"] = m["source"][17:18].copy()
    one["fun"] = m["fun"][17:18].copy()
    with eng.Engine(one, "fp64") as e1:
        e1.step(w.steps)
        assert np.array_equal(_traces(e1), batch_shot)
        assert np.array_equal(e1.fetch("Txz"), batch_field)
    # doubling the source doubles every value up to the rounding of values that underflow ahead
    # of the wave front (their relative error is carried along as the front grows; on this mesh
    # the precursor reaches the FP64 subnormal range too), measured in relative L2
    m2 = dict(m)
    m2["wavelet"] = 2.0 * m["wavelet"]
    for p, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
        with eng.Engine(m, p) as a, eng.Engine(m2, p) as b:
            a.step(300)
            b.step(300)
            for shot in (0, 40):
                ta, tb = 2.0 * _traces(a, 0, shot), _traces(b, 0, shot)
                assert rel_l2(ta, tb) <= tol, (p, rel_l2(ta, tb))


def test_uneven_batch_each_mesh_against_fp64_and_own_step_count():
    ws, _ = W.uneven_batch()
    ws = ws[:12]
    setups, meshes = [], []
    for k, w in enumerate(ws):
        s = pkg.host.build_setup(w, full=False, n_steps=1)
        # 0.15 s of physical time (the Ricker delay is ~0.1 s): 500-1300 steps per mesh
        n = int(np.ceil(0.15 / s.dt))
        w.steps = n
        s = pkg.host.build_setup(w, full=False, n_steps=n)
        setups.append(s)
        meshes.append(eng.mesh_from_setup(s, with_ref_ops=False))
    longest = max(s.n_steps for s in setups)
    res = {}
    for p in ("fp64", "fp32"):
        with eng.Engine(meshes, p) as e:
            e.step(longest)
            res[p] = [[_traces(e, k, m) for m in range(ws[k].shots)] for k in range(len(ws))]
            for k in (0, len(ws) - 1):
                assert e.fetch("trace_x", k, 0).shape[0] == setups[k].n_steps
    for k, w in enumerate(ws):
        for m in range(w.shots):
            assert rel_l2(res["fp32"][k][m], res["fp64"][k][m]) <= 1e-4, (k, m)
    # a mesh that stopped early holds its state: stepping further is refused past the longest table
    with eng.Engine(meshes[:2], "fp64") as e:
        e.step(max(setups[0].n_steps, setups[1].n_steps))
        with pytest.raises(eng.DGError):
            e.step(1)


def test_uneven_meshes_whole_runs_against_oracle():
    """Three meshes of the uneven batch (6,050, 8,192 and 11,250 triangles; 7, 8 and 6 shots), each
    over its own whole run of 1.5 s of physical time (986, 1,585 and 1,396 steps of its own dt), in
    one context: the first and last shot of each mesh against the oracle, FP64 within 1e-10 and
    FP32 within 1e-4, traces and final fields; every mesh stops at its own last step."""
    ws_all, _ = W.uneven_batch()
    pick = [25, 21, 40]
    ws, setups = [], []
    for k in pick:
        w = ws_all[k]
        s = pkg.host.build_setup(w, full=False, n_steps=1)
        w.steps = int(np.ceil(1.5 / s.dt))
        setups.append(pkg.host.build_setup(w, full=True, n_steps=w.steps))
        ws.append(w)
    assert [s.K for s in setups] == [6050, 8192, 11250]
    meshes = [eng.mesh_from_setup(s, with_ref_ops=False) for s in setups]
    ref = {}
    for k, (w, s) in enumerate(zip(ws, setups)):
        for m in (0, w.shots - 1):
            o = oracle.Oracle.from_setup(s)
            rx, rz = o.run(m, w.steps, threads=0, flush_subnormals=True)
            ref[k, m] = (np.concatenate([rx.ravel(), rz.ravel()]), [f.copy() for f in o.fields])
            assert np.abs(ref[k, m][0]).max() > 1e-12  # the wave has reached the receivers
    longest = max(w.steps for w in ws)
    for p, tol in (("fp64", 1e-10), ("fp32", 1e-4)):
        with eng.Engine(meshes, p) as e:
            e.step(longest)
            for (k, m), (tr, fields) in ref.items():
                assert e.fetch("trace_x", k, m).shape[0] == ws[k].steps
                assert rel_l2(_traces(e, k, m), tr) <= tol, (p, k, m, rel_l2(_traces(e, k, m), tr))
                for q, f in enumerate(FIELDS):
                    assert rel_l2(e.fetch(f, k, m), fields[q]) <= tol, (p, k, m, f)
