"""dg_gpu_energy_noalloc: the energy entry point that allocates no device memory.

It is meant for callers that cannot call cudaMalloc — for example an energy monitor running
inside another program's time loop, where that program owns all device memory through its own
pool and an allocation would synchronise the device and stall the solver.  The test plays such a
caller: it owns the input and output buffers and checks the result against the context's own
energy (dg_gpu_fetch with DG_ENERGY) on two calls in a row with different wavefields, so a
stale partial sum left in the shared static scratch by the first call would show in the second.
This file is collected last so a failure here stops a -x run only after every other test ran.
"""
import numpy as np
import pytest

from conftest import Golden, pkg

eng = pkg.engine
pytestmark = pytest.mark.gpu

TOL = 1e-10  # the FP64 tolerance of the parity tests


def test_energy_noalloc_matches_context_energy_on_two_calls():
    import torch

    g = Golden("slope_coupled")
    a = g.setup_arrays()
    dev = torch.device("cuda", 0)
    jac = torch.tensor(np.ascontiguousarray(a["Jacobi"]), dtype=torch.float64, device=dev)
    A = torch.tensor(np.ascontiguousarray(a["A"]), dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    with eng.Engine(eng.mesh_from_setup(a), "fp64") as e:
        results = []
        for steps in (100, 40):  # two calls in a row, on the wavefields at step 100 and 140
            e.step(steps)
            expected = e.fetch("energy")
            fields = [torch.tensor(e.fetch(f), dtype=torch.float64, device=dev)
                      for f in ("Vx", "Vz", "Txx", "Tzz", "Txz")]
            eng.energy_noalloc(0, g.K, fields, jac, A, g.ops["inverV"], out)
            got = float(out.cpu()[0])
            assert expected > 0
            assert abs(got - expected) <= TOL * expected, (steps, got, expected)
            results.append(got)
        assert results[0] != results[1]
    # sizes beyond the static scratch are refused before anything runs
    with pytest.raises(eng.DGError) as ei:
        eng.energy_noalloc(0, 4194305, fields, jac, A, g.ops["inverV"], out)
    assert ei.value.code == -1
