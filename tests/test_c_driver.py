"""The C ABI driven from C, as the reference's time loop would drive it.

CPU: the driver (tests/c_driver/dg_driver.c) compiles as C99 against include/dg_gpu.h with
-Wall -Werror and links against libdg_gpu.so.  GPU: it runs on set-up arrays written by Python
and its traces, final field and snapshots equal the Python binding's bit for bit; the same steps
taken again as half steps in parts (dg_gpu_half_step_part) give the same field.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, pkg

SRC = os.path.join(ROOT, "tests", "c_driver", "dg_driver.c")


def _build(tmp_path):
    cc = shutil.which("gcc") or "gcc"
    so = pkg.build.gpu_library()
    exe = str(tmp_path / "dg_driver")
    subprocess.run([cc, "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                    "-o", exe, "-L", os.path.dirname(so), "-ldg_gpu", "-Wl,-rpath," + os.path.dirname(so)],
                   check=True)
    return exe


def test_c_driver_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


def _write_inputs(d, s, mesh):
    os.makedirs(d, exist_ok=True)
    ints = {"Triangle", "ibe", "Neighbor", "Node_Neighbor", "Edge_flag", "source", "receiver"}
    for n in ("Point", "Triangle", "Vr", "Vs", "inverV", "V", "S", "ibe", "Neighbor", "Node_Neighbor", "Edge_flag",
              "A", "B", "Dx", "Dz", "Q", "absorb_fun", "source", "fun", "receiver", "wavelet"):
        np.ascontiguousarray(mesh[n], dtype=np.int64 if n in ints else np.float64).tofile(os.path.join(d, n + ".bin"))
    with open(os.path.join(d, "sizes.txt"), "w") as f:
        f.write("%d %d %d %d %d %.17g\n" % (s.K, s.n_points, s.n_shots, s.n_rec, s.n_steps, mesh["dt"]))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 2])
def test_c_driver_equals_python_binding(tmp_path, precision):
    exe = _build(tmp_path)
    w = pkg.workloads.small_square(n_cells=12, steps=120, shots=2)
    s = pkg.host.build_setup(w, full=True)
    mesh = pkg.engine.mesh_from_setup(s)
    _write_inputs(str(tmp_path / "in"), s, mesh)
    os.makedirs(tmp_path / "out")
    r = subprocess.run([exe, str(tmp_path / "in"), str(precision), "100", "20", str(tmp_path / "out")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    K, R = s.K, s.n_rec
    got = {n: np.fromfile(tmp_path / "out" / (n + ".bin"))
           for n in ("trace_x", "trace_z", "Txz", "snapshots", "Txz_parts")}
    assert np.array_equal(got["Txz_parts"], got["Txz"])    # the same steps as half steps in parts
    snaps = []
    with pkg.engine.Engine(mesh, precision) as e:
        for _ in range(5):
            e.step(20)
            snaps += [e.fetch("Vx", 0, 0), e.fetch("Vz", 0, 0)]
        assert np.array_equal(got["trace_x"], e.fetch("trace_x", 0, 0).ravel())
        assert np.array_equal(got["trace_z"], e.fetch("trace_z", 0, 0).ravel())
        assert np.array_equal(got["Txz"], e.fetch("Txz", 0, 0).ravel())
    assert np.array_equal(got["snapshots"], np.concatenate([v.ravel() for v in snaps]))
    assert got["trace_z"].size == 100 * R and np.abs(got["trace_z"]).max() > 0 and K > 0
