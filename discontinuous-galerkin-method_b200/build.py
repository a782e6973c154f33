"""In-tree build of the native libraries (no JIT cache: the built .so files sit next to this file).

* ``libdg_host.so`` — host set-up (csrc/dg_host.c), gcc, ``-O2 -ffp-contract=off`` so its
  arrays equal the reference host code's; ``-fopenmp`` for its per-element loops.
* ``libdg_gpu.so``  — the sm_100a engine and its C ABI (csrc/dg_gpu.cu), nvcc
  ``-gencode arch=compute_100a,code=sm_100a``; the host side of ``dg_gpu_init`` uses OpenMP.
"""
from __future__ import annotations

import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

HOST_SO = os.path.join(PKG, "libdg_host.so")
GPU_SO = os.path.join(PKG, "libdg_gpu.so")

HOST_SRC = [os.path.join(CSRC, "dg_host.c")]
GPU_SRC = [os.path.join(CSRC, "dg_gpu.cu"), os.path.join(CSRC, "dg_noalloc.cu")]
GPU_DEPS = GPU_SRC + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
    [os.path.join(INCLUDE, "dg_gpu.h")]

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", "-shared", "--expt-relaxed-constexpr", "-Xptxas", "-v", "-lgomp"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _cc():
    # the environment may point CC at a wrapper; the system gcc is what the parity flags assume
    return shutil.which("gcc") or "gcc"


def host_library(force: bool = False) -> str:
    deps = HOST_SRC + [os.path.join(INCLUDE, "dg_host.h")]
    if force or _stale(HOST_SO, deps):
        tmp = HOST_SO + ".tmp%d" % os.getpid()
        subprocess.run([_cc(), "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-Wall",
                        "-I" + INCLUDE, "-o", tmp] + HOST_SRC + ["-lm"], check=True)
        os.replace(tmp, HOST_SO)
    return HOST_SO


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def gpu_library(force: bool = False, log: str | None = None) -> str:
    if force or _stale(GPU_SO, GPU_DEPS):
        tmp = GPU_SO + ".tmp%d" % os.getpid()
        cmd = [nvcc()] + NVCC_FLAGS + ["-I" + INCLUDE, "-I" + CSRC, "-o", tmp] + GPU_SRC
        r = subprocess.run(cmd, capture_output=True, text=True)
        if log:
            with open(log, "w") as f:
                f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
        os.replace(tmp, GPU_SO)
    return GPU_SO


def build_all(force: bool = False) -> dict:
    return {"host": host_library(force), "gpu": gpu_library(force)}
