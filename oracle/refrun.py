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


# instruction-set features of the x86-64-v3 level the throughput build is compiled for
_V3 = ("avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "movbe", "xsave", "abm")


def host_has_v3() -> bool:
    """True if this host's CPU reports every x86-64-v3 feature (Linux /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    have = set(line.split(":", 1)[1].split())
                    return all(x in have for x in _V3)
    except OSError:
        pass
    return False


def binary_for(w, fast: bool = False) -> str:
    """The parity build, or (fast) the throughput build of the same sources and settings."""
    bx, bz, mw, mh = (int(round(v)) for v in w.sponge)
    name = "dgref_%sF%d_X%d_Z%d_W%d_H%d" % ("fast_" if fast else "", int(round(w.fp)), bx, bz, mw, mh)
    return os.path.join(REF_DIR, name)


def available(w, fast: bool = False) -> bool:
    return os.access(binary_for(w, fast), os.X_OK) and (not fast or host_has_v3())


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
        work_dir: str | None = None, timeout: float | None = None, fast: bool = False) -> dict:
    """Run the reference harness (fast: the throughput build); returns {"timing": {...}, "out": out_dir}."""
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
        subprocess.run([binary_for(w, fast), paths["prefix"], paths["matrix_dir"], cfg, out_dir], check=True,
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
