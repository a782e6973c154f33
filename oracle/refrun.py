"""Run the reference's own C code (oracle/_ref, built by oracle/Makefile) on a workload.

TEST INFRASTRUCTURE ONLY: used by the fixture generator, the parity tests and the benchmark's
CPU-baseline leg; never by the product path.  The binary reads the mesh in the converted
Triangle text format and the ten operator text files exactly as DG_leap_Frog_OpenMP.c does,
so a workload is first written to disk.
"""
from __future__ import annotations

import importlib
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_pkg = importlib.import_module("discontinuous-galerkin-method_b200")
meshgen = _pkg.meshgen
operators = _pkg.operators


def binary_for(w) -> str:
    bx, bz, mw, mh = (int(round(v)) for v in w.sponge)
    return os.path.join(REF_DIR, "dgref_F%d_X%d_Z%d_W%d_H%d" % (int(round(w.fp)), bx, bz, mw, mh))


def available(w) -> bool:
    return os.access(binary_for(w), os.X_OK)


def write_inputs(w, d: str, matrix_dir: str | None = None) -> dict:
    """Mesh files, operator files, materials, receivers and the harness config under ``d``."""
    os.makedirs(d, exist_ok=True)
    prefix = os.path.join(d, "mesh")
    meshgen.write_converted(w.mesh, prefix)
    if matrix_dir is None:
        matrix_dir = os.path.join(d, "matrix")
        operators.write_text_files(matrix_dir)
    w.materials().tofile(os.path.join(d, "mat.bin"))
    np.ascontiguousarray(w.rec, dtype=np.float64).tofile(os.path.join(d, "rec.bin"))
    return {"prefix": prefix, "matrix_dir": matrix_dir}


def run(w, out_dir: str, *, steps: int | None = None, snap_every: int = 0, threads: int = 0,
        shots_to_run: int | None = None, dump_setup: int = 1, matrix_dir: str | None = None,
        work_dir: str | None = None, timeout: float | None = None) -> dict:
    """Run the reference harness; returns {"timing": {...}, "out": out_dir}."""
    if w.shots > 64:
        raise ValueError("the harness takes at most 64 shots")
    tmp = None
    if work_dir is None:
        tmp = tempfile.TemporaryDirectory(prefix="dgref_")
        work_dir = tmp.name
    try:
        paths = write_inputs(w, work_dir, matrix_dir)
        os.makedirs(out_dir, exist_ok=True)
        cfg = os.path.join(work_dir, "cfg.txt")
        with open(cfg, "w") as f:
            f.write("steps %d\nsnap_every %d\nn_src %d\n" % (steps if steps is not None else w.steps,
                                                          snap_every, w.shots))
            for x, z in w.src:
                f.write("src %.17g %.17g\n" % (x, z))
            f.write("n_rec %d\nrec_file %s\nmat_file %s\n" % (w.rec.shape[0], os.path.join(work_dir, "rec.bin"),
                                                              os.path.join(work_dir, "mat.bin")))
            f.write("dump_setup %d\nthreads %d\nquiet 1\n" % (dump_setup, threads))
            if shots_to_run is not None:
                f.write("shots_to_run %d\n" % shots_to_run)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        env.setdefault("OMP_PROC_BIND", "close")
        subprocess.run([binary_for(w), paths["prefix"], paths["matrix_dir"], cfg, out_dir], check=True,
                       env=env, timeout=timeout)
        timing = {}
        with open(os.path.join(out_dir, "timing.txt")) as f:
            for line in f:
                k, v = line.split()
                timing[k] = float(v)
        return {"timing": timing, "out": out_dir}
    finally:
        if tmp is not None:
            tmp.cleanup()


def load(out_dir: str, name: str, dtype=np.float64) -> np.ndarray:
    return np.fromfile(os.path.join(out_dir, name + ".bin"), dtype=dtype)
