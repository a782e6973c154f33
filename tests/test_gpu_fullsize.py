"""Full-size GPU checks of the benchmark configurations.

* 20,000-element square, 2,000 steps: reference-operator path bit-identical to the CPU oracle,
  FP64 within 1e-10, FP32 and FP32-Kahan within 1e-4 (traces).
* coupled acoustic-elastic slope (~400k elements): FP64 within 1e-10 of the oracle over the
  first 100 steps; FP32 / FP32-Kahan within 1e-4 of FP64 over all 6,000 steps; energy drift.
* 2M-element random medium, 10,000 steps: FP32-Kahan and FP32 against FP64 (traces, energy).
* 200k elements x 64 shots: FP32 against FP64 over 1,000 steps; a shot of the batch equals the
  same shot run alone (FP64, bit for bit); doubling the wavelet doubles the traces exactly.
* 48 uneven meshes with their own dt and step counts in one context: each mesh against FP64,
  and each mesh stops at its own last step.
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
    s = pkg.host.build_setup(w, full=False)
    m = eng.mesh_from_setup(s, with_ref_ops=False)
    with eng.Engine(m, "fp32") as e32, eng.Engine(m, "fp64") as e64:
        e32.step(w.steps)
        e64.step(w.steps)
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
