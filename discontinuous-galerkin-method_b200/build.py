"""In-tree build of the native libraries (no JIT cache: the built .so files sit next to this file).

* ``libdg_host.so`` — host set-up (csrc/dg_host.c), gcc, ``-O2 -ffp-contract=off`` so its
  arrays equal the reference host code's; ``-fopenmp`` for its per-element loops.
* ``libdg_gpu.so``  — the sm_100a engine and its C ABI (csrc/dg_gpu.cu, dg_noalloc.cu) and the
  step kernels' instances (csrc/dg_k_*.cu), nvcc ``-gencode arch=compute_100a,code=sm_100a``;
  each translation unit is compiled on its own process, then all are linked; the host side of
  ``dg_gpu_init`` uses OpenMP.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

HOST_SO = os.path.join(PKG, "libdg_host.so")
GPU_SO = os.path.join(PKG, "libdg_gpu.so")

HOST_SRC = [os.path.join(CSRC, "dg_host.c")]
GPU_SRC = [os.path.join(CSRC, f) for f in ("dg_gpu.cu", "dg_noalloc.cu", "dg_k_generic.cu", "dg_k_x2_small.cu",
                                            "dg_k_x2_mid.cu", "dg_k_x2_large.cu", "dg_k_wave.cu", "dg_k_multi.cu")]
# translation units: (source, extra flags, object tag); dg_k_multi.cu is compiled once per part
GPU_UNITS = [(src, [], os.path.basename(src)) for src in GPU_SRC if not src.endswith("dg_k_multi.cu")] + \
    [(os.path.join(CSRC, "dg_k_multi.cu"), ["-DDG_MX_PART=%d" % k], "dg_k_multi%d" % k) for k in range(7)]
GPU_DEPS = GPU_SRC + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
    [os.path.join(INCLUDE, "dg_gpu.h")]

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", "--expt-relaxed-constexpr", "-Xptxas", "-v"]
LINK_FLAGS = ["-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fopenmp", "-lgomp"]


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
        tag = ".tmp%d" % os.getpid()
        objs = [os.path.join(PKG, "_obj", name + tag + ".o") for _, _, name in GPU_UNITS]
        os.makedirs(os.path.join(PKG, "_obj"), exist_ok=True)

        def compile_one(k):
            src, extra, _ = GPU_UNITS[k]
            cmd = [nvcc()] + NVCC_FLAGS + extra + ["-I" + INCLUDE, "-I" + CSRC, "-c", "-o", objs[k], src]
            return cmd, subprocess.run(cmd, capture_output=True, text=True)

        try:
            # the slow units (the batch parts) first
            order = sorted(range(len(GPU_UNITS)), key=lambda k: not GPU_UNITS[k][2].startswith("dg_k_multi"))
            with ThreadPoolExecutor(max_workers=max(1, min(len(GPU_UNITS), os.cpu_count() or 1))) as ex:
                results = list(ex.map(compile_one, order))
            text = "".join(" ".join(cmd) + "\n" + r.stdout + r.stderr for cmd, r in results)
            bad = [r for _, r in results if r.returncode != 0]
            if not bad:
                tmp = GPU_SO + tag
                cmd = [nvcc()] + LINK_FLAGS + ["-o", tmp] + objs
                r = subprocess.run(cmd, capture_output=True, text=True)
                text += " ".join(cmd) + "\n" + r.stdout + r.stderr
                if r.returncode != 0:
                    bad = [r]
            if log:
                with open(log, "w") as f:
                    f.write(text)
            if bad:
                raise RuntimeError("nvcc failed:\n" + bad[0].stderr[-4000:])
            os.replace(tmp, GPU_SO)
        finally:
            for o in objs:
                if os.path.exists(o):
                    os.remove(o)
    return GPU_SO


def build_all(force: bool = False) -> dict:
    return {"host": host_library(force), "gpu": gpu_library(force)}
