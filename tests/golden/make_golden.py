"""Generate the golden fixtures from the reference's own C code.

Run in a container that has the reference tree (default $DG_REFERENCE_ROOT, else /root/reference) and the compiled
harness (``make -C oracle ref``)::

    python tests/golden/make_golden.py [--ref /root/reference]

For each small workload it writes the mesh in the converted Triangle format, runs
oracle/_ref (the reference's fun_save_to_file.c / fun_DG.c / OpenMP_Function.c, unmodified,
built with -O2 -ffp-contract=off) with the operator text files shipped in the reference
(input_files/precomputed_matrix), and stores, compressed, in ``<name>.npz``:

* the generator's raw mesh (``points_raw``, 0-based ``tris``, ``neigh``) and the medium,
  sources, receivers, Ricker frequency and sponge geometry;
* every array the reference's host set-up produced (``setup_*``), as dumped by the harness;
* the receiver traces, Vx/Vz snapshots every 50 steps and the five final fields per shot.

The fixtures pin the CPU oracle (oracle/dg_oracle.c) and the host set-up library
(csrc/dg_host.c) bit for bit; the GPU tests then compare the engine against the oracle.
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

pkg = importlib.import_module("discontinuous-galerkin-method_b200")
import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
SNAP = 50

CASES = {
    "square_K288": lambda w: w.small_square(n_cells=12, steps=200, shots=1),
    "slope_coupled": lambda w: w.small_slope(steps=150),
    "square_3shots": lambda w: w.small_square(n_cells=10, steps=150, shots=3),
}

INT_ARRAYS = {"Neighbor", "Edge", "Edge_flag", "Node_Neighbor", "ibe", "source", "receiver", "Triangle",
              "neighbor_in", "attribute", "absorbing_triangle", "sizes"}


def make(name, w, ref_root):
    matrix_dir = os.path.join(ref_root, "input_files", "precomputed_matrix")
    with tempfile.TemporaryDirectory() as out:
        refrun.run(w, out, snap_every=SNAP, matrix_dir=matrix_dir, threads=2)
        K = w.K
        d = {"points_raw": w.mesh.points, "tris": w.mesh.tris, "neigh": w.mesh.neigh, "attr": w.mesh.attr,
             "markers": w.mesh.markers, "vp": w.vp, "vs": w.vs, "rho": w.rho, "src": w.src, "rec": w.rec,
             "fp": np.float64(w.fp), "sponge": np.asarray(w.sponge, dtype=np.float64), "steps": np.int64(w.steps),
             "snap_every": np.int64(SNAP)}
        for n in ["sizes", "dt_t0", "Point", "Triangle", "neighbor_in", "attribute", "Neighbor", "Edge", "Edge_flag",
                  "Node_Neighbor", "ibe", "Jacobi", "Jacobi_Edge", "normal1", "normal2", "normal3", "A", "B", "Q",
                  "Dx", "Dz", "S", "absorb_fun", "absorbing_triangle", "source", "fun", "receiver",
                  "ops_Vr_Vs_inverV_V_Fekete"]:
            d["setup_" + n] = refrun.load(out, n, np.int64 if n in INT_ARRAYS else np.float64)
        for m in range(w.shots):
            d["shot%d_rec_x" % m] = refrun.load(out, "shot%d_rec_x" % m).reshape(w.steps, -1)
            d["shot%d_rec_z" % m] = refrun.load(out, "shot%d_rec_z" % m).reshape(w.steps, -1)
            for t in range(SNAP, w.steps + 1, SNAP):
                for f in ("Vx", "Vz"):
                    d["shot%d_%s%d" % (m, f, t)] = refrun.load(out, "shot%d_%s%d" % (m, f, t))
            for f in ("Vx", "Vz", "Txx", "Tzz", "Txz"):
                d["shot%d_final_%s" % (m, f)] = refrun.load(out, "shot%d_final_%s" % (m, f))
        assert d["setup_sizes"][0] == K
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes; K =", K, "shots =", w.shots)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DG_REFERENCE_ROOT", "/root/reference"))
    args = ap.parse_args()
    for name, fn in CASES.items():
        w = fn(pkg.workloads)
        if not refrun.available(w):
            raise SystemExit("oracle/_ref binary missing for %s: run make -C oracle ref" % name)
        make(name, w, args.ref)


if __name__ == "__main__":
    main()
