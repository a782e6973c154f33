import glob
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")

pkg = importlib.import_module("discontinuous-galerkin-method_b200")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: larger CPU or GPU cases")


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


class Golden:
    """A golden fixture: reference set-up arrays and outputs, plus the workload it came from."""

    def __init__(self, name):
        self.name = name
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.z = {k: z[k] for k in z.files}
        g = self.z
        self.K = int(g["setup_sizes"][0])
        self.P = int(g["setup_sizes"][1])
        self.dt, self.t0 = (float(v) for v in g["setup_dt_t0"])
        self.steps = int(g["steps"])
        self.shots = int(g["src"].shape[0])
        self.snap_every = int(g["snap_every"])
        ops = g["setup_ops_Vr_Vs_inverV_V_Fekete"]
        S = g["setup_S"].reshape(3, 6, 3)
        self.ops = {"Vr": ops[0:36].reshape(6, 6), "Vs": ops[36:72].reshape(6, 6), "inverV": ops[72:108].reshape(6, 6),
                    "V": ops[108:144].reshape(6, 6), "FeketeNew": ops[144:156].reshape(6, 2),
                    "S1": S[0].copy(), "S2": S[1].copy(), "S3": S[2].copy()}

    def workload(self):
        mg = pkg.meshgen
        mesh = mg.Mesh(self.z["points_raw"], self.z["tris"], self.z["neigh"], self.z["attr"], self.z["markers"])
        return pkg.workloads.Workload(self.name, mesh, self.z["vp"], self.z["vs"], self.z["rho"], float(self.z["fp"]),
                                      tuple(self.z["sponge"]), self.z["src"], self.z["rec"], self.steps)

    def setup_arrays(self):
        """Reference set-up arrays keyed like the host library's output, plus the wavelet table."""
        g = self.z
        a = {n[len("setup_"):]: g[n] for n in g if n.startswith("setup_")}
        a["Point"] = a["Point"].reshape(-1, 2)
        a["Triangle"] = a["Triangle"].reshape(-1, 3)
        w = pkg.host
        a["wavelet"] = np.array([w.lib().dgh_ricker(t, self.dt, self.t0, float(g["fp"]), 3.1415)
                                 for t in range(self.steps)])
        a["dt"] = self.dt
        a["ops"] = self.ops
        return a


@pytest.fixture(params=golden_names())
def golden(request):
    return Golden(request.param)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
