"""ctypes binding of the CPU oracle (oracle/dg_oracle.c) — TEST INFRASTRUCTURE ONLY.

Imported by the tests and by the benchmark's CPU-baseline leg; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")
_LIB = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "dg_oracle.c")
    if force or not os.path.exists(SO) or os.path.getmtime(src) > os.path.getmtime(SO):
        cc = shutil.which("gcc") or "gcc"
        tmp = SO + ".tmp%d" % os.getpid()
        subprocess.run([cc, "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        "-o", tmp, src, "-lm"], check=True)
        os.replace(tmp, SO)
    return SO


class _Problem(C.Structure):
    _fields_ = [("K", C.c_long), ("A", C.c_void_p), ("B", C.c_void_p), ("Dx", C.c_void_p), ("Dz", C.c_void_p),
                ("Q", C.c_void_p), ("S", C.c_void_p), ("ibe", C.c_void_p), ("Node_Neighbor", C.c_void_p),
                ("Neighbor", C.c_void_p), ("Edge_flag", C.c_void_p), ("absorb_fun", C.c_void_p),
                ("source", C.c_void_p), ("fun", C.c_void_p), ("n_rec", C.c_long), ("receiver", C.c_void_p),
                ("dt", C.c_double), ("wavelet", C.c_void_p), ("n_steps", C.c_long)]


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        _LIB.dgo_run.restype = C.c_int
        _LIB.dgo_run.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_long] + [C.c_void_p] * 7 + [C.c_int]
        _LIB.dgo_max_threads.restype = C.c_int
        _LIB.dgo_half.restype = C.c_int
        _LIB.dgo_half.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_int] + [C.c_void_p] * 7
        _LIB.dgo_set_flush_subnormals.argtypes = [C.c_int]
        _LIB.dgo_set_flush_subnormals.restype = None
    return _LIB


class Oracle:
    """Time loop on the reference arrays (a host ``Setup`` or a golden fixture dict)."""

    _NAMES = ["A", "B", "Dx", "Dz", "Q", "S", "ibe", "Node_Neighbor", "Neighbor", "Edge_flag", "absorb_fun",
              "source", "fun", "receiver", "wavelet"]
    _INTS = {"ibe", "Node_Neighbor", "Neighbor", "Edge_flag", "source", "receiver"}

    def __init__(self, arrays: dict, dt: float, K: int):
        self.K = int(K)
        self.keep = {}
        for n in self._NAMES:
            a = np.ascontiguousarray(arrays[n], dtype=np.int64 if n in self._INTS else np.float64)
            self.keep[n] = a
        self.n_rec = self.keep["receiver"].size // 2
        self.n_steps = self.keep["wavelet"].size
        self.prob = _Problem(K=self.K, n_rec=self.n_rec, dt=float(dt), n_steps=self.n_steps,
                             **{n: self.keep[n].ctypes.data for n in self._NAMES})
        self.fields = None

    @classmethod
    def from_setup(cls, s):
        return cls(s.arrays, s.dt, s.K)

    def reset(self):
        self.fields = [np.zeros(self.K * 6) for _ in range(5)]
        self.t = 0

    def run(self, shot: int, steps: int, threads: int = 0, record: bool = True, flush_subnormals: bool = False):
        """`steps` steps of `shot`; with flush_subnormals the loops flush subnormal values to zero
        (for long runs compared at a relative tolerance only: values below 2^-1022 become 0)."""
        if self.fields is None:
            self.reset()
        rx = np.zeros((steps, self.n_rec)) if record else None
        rz = np.zeros((steps, self.n_rec)) if record else None
        f = self.fields
        lib().dgo_set_flush_subnormals(1 if flush_subnormals else 0)
        try:
            rc = lib().dgo_run(C.byref(self.prob), shot, self.t, steps, *(a.ctypes.data for a in f),
                               None if rx is None else rx.ctypes.data, None if rz is None else rz.ctypes.data,
                               threads)
        finally:
            lib().dgo_set_flush_subnormals(0)
        if rc != 0:
            raise RuntimeError("oracle run failed (%d)" % rc)
        self.t += steps
        return rx, rz

    def half(self, shot: int, t: int, half: int, rec_x=None, rec_z=None):
        """One half of step t (0: sponge, source, velocity; 1: stress and record into the n_rec
        arrays rec_x/rec_z), for the split-mesh test."""
        if self.fields is None:
            self.reset()
        rc = lib().dgo_half(C.byref(self.prob), shot, t, half, *(a.ctypes.data for a in self.fields),
                            None if rec_x is None else rec_x.ctypes.data, None if rec_z is None else rec_z.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle half step failed (%d)" % rc)
