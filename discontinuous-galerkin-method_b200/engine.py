"""ctypes binding of the sm_100a engine (csrc/dg_gpu.cu, include/dg_gpu.h).

``Engine`` mirrors the reference's per-step call sequence (DG_leap_Frog_OpenMP.c:418-437):
``step(n)`` advances every mesh n steps (sponge, source, velocity, stress, record),
``fetch`` returns fields/traces in the reference's element-major layout.  There is no CPU
fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build as _build

FP64_REF, FP64, FP32, FP32_KAHAN = 0, 1, 2, 3
PRECISIONS = {"fp64_ref": FP64_REF, "fp64": FP64, "fp32": FP32, "fp32_kahan": FP32_KAHAN}
VX, VZ, TXX, TZZ, TXZ, TRACE_X, TRACE_Z, ENERGY = range(8)
FIELDS = {"Vx": VX, "Vz": VZ, "Txx": TXX, "Tzz": TZZ, "Txz": TXZ}

ERRORS = {0: "DG_OK", -1: "DG_ERR_ARG", -2: "DG_ERR_CUDA", -3: "DG_ERR_NOMEM", -4: "DG_ERR_MESH",
          -5: "DG_ERR_NONFINITE", -6: "DG_ERR_STATE", -7: "DG_ERR_UNSUPPORTED", -8: "DG_ERR_NODEVICE",
          -9: "DG_ERR_ORIENTATION", -10: "DG_ERR_TIMEOUT"}

def _ptr(a):
    """Address of a host buffer: a numpy array or anything with data_ptr() (e.g. pinned memory)."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"] or a.dtype != np.float64:
        raise ValueError("need a C-contiguous float64 buffer")
    return a.ctypes.data


# exported symbols of include/dg_gpu.h (checked by the CPU tests)
EXPORTS = ["dg_gpu_default_opts", "dg_gpu_init", "dg_gpu_step", "dg_gpu_step_async", "dg_gpu_synchronize", "dg_gpu_step_timed", "dg_gpu_step_profiled",
           "dg_gpu_fetch_traces", "dg_gpu_fetch", "dg_gpu_load",
           "dg_gpu_reset", "dg_gpu_set_wavelet", "dg_gpu_flush_l2", "dg_gpu_stats_get", "dg_gpu_steps_done",
           "dg_gpu_free", "dg_gpu_strerror", "dg_gpu_last_error", "dg_gpu_energy_noalloc",
           "dg_gpu_debug_stall_wave", "dg_gpu_step_snapshots", "dg_gpu_half_step", "dg_gpu_half_step_part",
           "dg_gpu_halo_lists", "dg_gpu_halo_pack", "dg_gpu_halo_pack_async", "dg_gpu_halo_unpack",
           "dg_gpu_context_stream"]
# parts of a half step (dg_gpu_half_step_part)
PART_ALL, PART_BOUNDARY, PART_INTERIOR = 0, 1, 2
# every mesh of the context at once (dg_gpu_fetch_traces, dg_gpu_set_wavelet), every shot of a
# mesh at once (dg_gpu_fetch of a field)
ALL_MESHES = -1
ALL_SHOTS = -1


def energy_noalloc(device: int, K: int, fields, jacobi, A, inverV: np.ndarray, out, stream=None) -> None:
    """dg_gpu_energy_noalloc through the C ABI.

    ``fields`` (Vx, Vz, Txx, Tzz, Txz), ``jacobi``, ``A`` and ``out`` are device buffers the
    caller owns (anything with ``data_ptr()``); ``inverV`` is a host array.  Nothing is allocated.
    """
    iv = np.ascontiguousarray(inverV, dtype=np.float64)
    ptrs = [f.data_ptr() for f in fields] + [jacobi.data_ptr(), A.data_ptr(), iv.ctypes.data, out.data_ptr()]
    _check(lib().dg_gpu_energy_noalloc(int(device), int(K), *ptrs, stream), "dg_gpu_energy_noalloc")


class DGError(RuntimeError):
    def __init__(self, code, where, detail=""):
        self.code = code
        super().__init__("%s failed: %s (%d) %s" % (where, ERRORS.get(code, "?"), code, detail))


class _Mesh(C.Structure):
    _fields_ = [("K", C.c_long), ("Np", C.c_int), ("Nfp", C.c_int), ("n_points", C.c_long),
                ("Point", C.c_void_p), ("Triangle", C.c_void_p), ("Vr", C.c_void_p), ("Vs", C.c_void_p),
                ("inverV", C.c_void_p), ("V", C.c_void_p), ("S", C.c_void_p), ("ibe", C.c_void_p),
                ("Neighbor", C.c_void_p), ("Node_Neighbor", C.c_void_p), ("Edge_flag", C.c_void_p),
                ("A", C.c_void_p), ("B", C.c_void_p), ("Dx", C.c_void_p), ("Dz", C.c_void_p), ("Q", C.c_void_p),
                ("absorb_fun", C.c_void_p), ("n_shots", C.c_int), ("source", C.c_void_p), ("fun", C.c_void_p),
                ("n_rec", C.c_int), ("receiver", C.c_void_p), ("dt", C.c_double), ("n_steps", C.c_long),
                ("wavelet", C.c_void_p)]


class _Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("reorder", C.c_int), ("block_threads", C.c_int),
                ("graph_steps", C.c_int), ("autotune", C.c_int), ("watchdog_every", C.c_int),
                ("tune_cache", C.c_char_p), ("variant", C.c_int), ("wavefront", C.c_int)]


class _Stats(C.Structure):
    _fields_ = [("ms_velocity", C.c_double), ("ms_stress", C.c_double), ("launches", C.c_long),
                ("steps_done", C.c_long), ("block_threads", C.c_int), ("graph_steps", C.c_int),
                ("bytes_per_step", C.c_double), ("dof_per_step", C.c_double), ("kernel_family", C.c_int)]

KERNEL_FAMILIES = {0: "reference operators (k_velocity_ref/k_stress_ref)",
                   1: "one (element, shot) per thread (k_velocity/k_stress)",
                   2: "two shots per thread, packed FP32x2 (k_velocity_x2/k_stress_x2)",
                   3: "two elements per thread, packed FP32x2 (k_velocity_x2e/k_stress_x2e)",
                   4: "batch of meshes, each block on its mesh's packed body (k_velocity_mx/k_stress_mx)",
                   5: "wavefront step: one launch per step, two shots per thread, L2-resident lag (k_step_wave)",
                   6: "wavefront step on resident blocks looping over tickets: one launch per step, two shots "
                      "per thread, L2-resident lag (k_step_wave_p)",
                   7: "two shots per thread, packed FP32x2, plane-major layout (k_velocity_x2/k_stress_x2)",
                   8: "batch of meshes in one persistent cooperative launch, grid barrier between the halves "
                      "(k_step_mx_p)"}
KERNEL_NAMES = {0: ("k_velocity_ref", "k_stress_ref"), 1: ("k_velocity", "k_stress"),
                2: ("k_velocity_x2", "k_stress_x2"), 3: ("k_velocity_x2e", "k_stress_x2e"),
                4: ("k_velocity_mx", "k_stress_mx"), 5: ("k_step_wave", None),
                6: ("k_step_wave_p", None), 7: ("k_velocity_x2", "k_stress_x2"), 8: ("k_step_mx_p", None)}


_LIB = None

# void (*)(void *user, long step, const double *vx, const double *vz)
SNAPSHOT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_long, C.POINTER(C.c_double), C.POINTER(C.c_double))


def lib(path: str | None = None):
    global _LIB
    if _LIB is None:
        so = path or _build.gpu_library()
        L = C.CDLL(so)
        L.dg_gpu_default_opts.argtypes = [C.c_void_p]
        L.dg_gpu_init.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.dg_gpu_step.argtypes = [C.c_void_p, C.c_long]
        L.dg_gpu_step_async.argtypes = [C.c_void_p, C.c_long]
        L.dg_gpu_synchronize.argtypes = [C.c_void_p]
        L.dg_gpu_step_timed.argtypes = [C.c_void_p, C.c_long]
        L.dg_gpu_step_profiled.argtypes = [C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dg_gpu_step_profiled.restype = C.c_int
        L.dg_gpu_fetch_traces.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_void_p, C.c_void_p]
        L.dg_gpu_fetch_traces.restype = C.c_int
        L.dg_gpu_energy_noalloc.argtypes = [C.c_int, C.c_long] + [C.c_void_p] * 10
        L.dg_gpu_energy_noalloc.restype = C.c_int
        L.dg_gpu_fetch.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.dg_gpu_load.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.dg_gpu_reset.argtypes = [C.c_void_p]
        L.dg_gpu_set_wavelet.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_void_p]
        L.dg_gpu_flush_l2.argtypes = [C.c_void_p]
        L.dg_gpu_debug_stall_wave.argtypes = [C.c_void_p, C.c_int]
        L.dg_gpu_step_snapshots.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_int, C.c_int, SNAPSHOT_FN,
                                            C.c_void_p]
        L.dg_gpu_step_snapshots.restype = C.c_int
        L.dg_gpu_half_step.argtypes = [C.c_void_p, C.c_int]
        L.dg_gpu_half_step_part.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.dg_gpu_halo_lists.argtypes = [C.c_void_p, C.c_int, C.c_long, C.c_void_p, C.c_long, C.c_void_p]
        L.dg_gpu_halo_pack.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.dg_gpu_halo_pack_async.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.dg_gpu_context_stream.argtypes = [C.c_void_p]
        L.dg_gpu_context_stream.restype = C.c_void_p
        L.dg_gpu_halo_unpack.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        for n in ("dg_gpu_half_step", "dg_gpu_half_step_part", "dg_gpu_halo_lists", "dg_gpu_halo_pack",
                  "dg_gpu_halo_pack_async", "dg_gpu_halo_unpack"):
            getattr(L, n).restype = C.c_int
        L.dg_gpu_stats_get.argtypes = [C.c_void_p, C.c_void_p]
        L.dg_gpu_steps_done.argtypes = [C.c_void_p]
        L.dg_gpu_steps_done.restype = C.c_long
        L.dg_gpu_free.argtypes = [C.c_void_p]
        L.dg_gpu_strerror.restype = C.c_char_p
        L.dg_gpu_strerror.argtypes = [C.c_int]
        L.dg_gpu_last_error.restype = C.c_char_p
        for n in ("dg_gpu_init", "dg_gpu_step", "dg_gpu_step_async", "dg_gpu_synchronize", "dg_gpu_step_timed",
                  "dg_gpu_fetch", "dg_gpu_load", "dg_gpu_reset", "dg_gpu_set_wavelet", "dg_gpu_flush_l2",
                  "dg_gpu_stats_get", "dg_gpu_free"):
            getattr(L, n).restype = C.c_int
        _LIB = L
    return _LIB


def _check(rc, where):
    if rc != 0:
        raise DGError(rc, where, lib().dg_gpu_last_error().decode(errors="replace"))


_INTS = {"ibe", "Neighbor", "Node_Neighbor", "Edge_flag", "source", "receiver", "Triangle"}


def mesh_from_setup(setup, *, wavelet=None, with_ref_ops: bool = True) -> dict:
    """Collect the arrays of a host ``Setup`` (or a golden fixture) that dg_gpu_init takes."""
    a = setup.arrays if hasattr(setup, "arrays") else setup
    get = (lambda n: a[n]) if isinstance(a, dict) else (lambda n: getattr(a, n))
    d = {"Point": setup.Point if hasattr(setup, "Point") else get("Point"),
         "Triangle": setup.Triangle if hasattr(setup, "Triangle") else get("Triangle")}
    ops = setup.ops if hasattr(setup, "ops") else get("ops")
    d.update({"Vr": ops["Vr"], "Vs": ops["Vs"], "inverV": ops["inverV"], "V": ops["V"]})
    for n in ("S", "ibe", "Neighbor", "Node_Neighbor", "Edge_flag", "A", "B", "absorb_fun", "source", "fun",
              "receiver"):
        d[n] = get(n)
    if with_ref_ops:
        for n in ("Dx", "Dz", "Q"):
            try:
                d[n] = get(n)
            except (KeyError, AttributeError):
                pass
    d["wavelet"] = get("wavelet") if wavelet is None else wavelet
    d["dt"] = float(setup.dt if hasattr(setup, "dt") else get("dt"))
    return d


class Engine:
    """One device context over one or more meshes (all meshes step together)."""

    def __init__(self, meshes, precision="fp64", *, device=0, reorder=True, block_threads=0, graph_steps=0,
                 autotune=False, watchdog_every=0, tune_cache=None, variant=0, wavefront=0):
        if isinstance(meshes, dict):
            meshes = [meshes]
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.precision = prec
        self.device = int(device)
        self._keep = []
        arr = (_Mesh * len(meshes))()
        self.info = []
        for k, m in enumerate(meshes):
            conv = {}
            for n, v in m.items():
                if isinstance(v, np.ndarray):
                    v = np.ascontiguousarray(v, dtype=np.int64 if n in _INTS else np.float64)
                    self._keep.append(v)
                conv[n] = v
            K = conv["Triangle"].size // 3
            S = conv["fun"].size // 6
            R = conv["receiver"].size // 2
            T = conv["wavelet"].size
            ptr = lambda n: conv[n].ctypes.data if n in conv and conv[n] is not None else None  # noqa: E731
            arr[k] = _Mesh(K=K, Np=6, Nfp=3, n_points=conv["Point"].size // 2, Point=ptr("Point"),
                           Triangle=ptr("Triangle"), Vr=ptr("Vr"), Vs=ptr("Vs"), inverV=ptr("inverV"), V=ptr("V"),
                           S=ptr("S"), ibe=ptr("ibe"), Neighbor=ptr("Neighbor"), Node_Neighbor=ptr("Node_Neighbor"),
                           Edge_flag=ptr("Edge_flag"), A=ptr("A"), B=ptr("B"), Dx=ptr("Dx"), Dz=ptr("Dz"),
                           Q=ptr("Q"), absorb_fun=ptr("absorb_fun"), n_shots=S, source=ptr("source"),
                           fun=ptr("fun"), n_rec=R, receiver=ptr("receiver"), dt=float(conv["dt"]), n_steps=T,
                           wavelet=ptr("wavelet"))
            self.info.append({"K": K, "S": S, "R": R, "T": T})
        opts = _Opts()
        lib().dg_gpu_default_opts(C.byref(opts))
        opts.precision = prec
        opts.device = device
        opts.reorder = 1 if reorder else 0
        opts.block_threads = block_threads
        opts.graph_steps = graph_steps
        opts.autotune = 1 if autotune else 0
        opts.watchdog_every = watchdog_every
        opts.tune_cache = tune_cache.encode() if tune_cache else None
        opts.variant = int(variant)
        opts.wavefront = int(wavefront)
        self._ctx = C.c_void_p()
        _check(lib().dg_gpu_init(C.byref(self._ctx), arr, len(meshes), C.byref(opts)), "dg_gpu_init")
        self._keep = []

    # -- the reference's loop body ---------------------------------------------------------
    def step(self, n: int = 1):
        _check(lib().dg_gpu_step(self._ctx, int(n)), "dg_gpu_step")

    def step_async(self, n: int = 1):
        """Enqueue n steps and return; `synchronize` waits for them (fetches wait by themselves)."""
        _check(lib().dg_gpu_step_async(self._ctx, int(n)), "dg_gpu_step_async")

    def synchronize(self):
        _check(lib().dg_gpu_synchronize(self._ctx), "dg_gpu_synchronize")

    def step_timed(self, n: int = 1):
        _check(lib().dg_gpu_step_timed(self._ctx, int(n)), "dg_gpu_step_timed")
        return self.stats()

    def step_profiled(self, n: int, flush_l2: bool = False):
        """n steps with CUDA events around every launch; returns (ms_vel[n], ms_str[n], ms_total)."""
        mv = np.zeros(max(int(n), 1), dtype=np.float32)
        ms = np.zeros(max(int(n), 1), dtype=np.float32)
        tot = C.c_double(0.0)
        _check(lib().dg_gpu_step_profiled(self._ctx, int(n), 1 if flush_l2 else 0, mv.ctypes.data, ms.ctypes.data,
                                          C.byref(tot)), "dg_gpu_step_profiled")
        return mv[:n], ms[:n], tot.value

    def step_snapshots(self, n: int, every: int, fn, mesh: int = 0, shot: int = 0):
        """Advance n steps; after every `every` steps call fn(step, vx, vz) with copies of the
        mesh/shot's Vx and Vz ([K][Np] doubles) while the device keeps stepping."""
        K = self.info[mesh]["K"]

        def cb(_user, step, vx, vz):
            fn(int(step), np.ctypeslib.as_array(vx, shape=(K, 6)).copy(),
               np.ctypeslib.as_array(vz, shape=(K, 6)).copy())

        cfn = SNAPSHOT_FN(cb)
        _check(lib().dg_gpu_step_snapshots(self._ctx, int(n), int(every), mesh, shot, cfn, None),
               "dg_gpu_step_snapshots")

    # ---- one part of a split mesh (decompose.SplitRun drives these) ----
    def half_step(self, half: int):
        _check(lib().dg_gpu_half_step(self._ctx, int(half)), "dg_gpu_half_step")

    def half_step_part(self, half: int, part: int):
        """One part of a half step: PART_BOUNDARY (elements with a ghost neighbour) or
        PART_INTERIOR (the other non-ghost elements); the half ends with its second part."""
        _check(lib().dg_gpu_half_step_part(self._ctx, int(half), int(part)), "dg_gpu_half_step_part")

    def halo_lists(self, send, recv, mesh: int = 0):
        s = np.ascontiguousarray(send, dtype=np.int64)
        r = np.ascontiguousarray(recv, dtype=np.int64)
        _check(lib().dg_gpu_halo_lists(self._ctx, mesh, s.size, s.ctypes.data if s.size else None, r.size,
                                       r.ctypes.data if r.size else None), "dg_gpu_halo_lists")

    def halo_pack(self, what: int, dev_ptr: int, mesh: int = 0, wait: bool = True):
        """Pack the send list into a device buffer; `wait=False` only enqueues it on the context
        stream (order the transfer after `stream()` with an event)."""
        if wait:
            _check(lib().dg_gpu_halo_pack(self._ctx, mesh, int(what), C.c_void_p(dev_ptr)), "dg_gpu_halo_pack")
        else:
            _check(lib().dg_gpu_halo_pack_async(self._ctx, mesh, int(what), C.c_void_p(dev_ptr)),
                   "dg_gpu_halo_pack_async")

    def stream(self):
        """The context's CUDA stream as a `torch.cuda.ExternalStream`."""
        import torch
        return torch.cuda.ExternalStream(lib().dg_gpu_context_stream(self._ctx), device=self.device)

    def halo_unpack(self, what: int, dev_ptr: int, mesh: int = 0):
        _check(lib().dg_gpu_halo_unpack(self._ctx, mesh, int(what), C.c_void_p(dev_ptr)), "dg_gpu_halo_unpack")

    def fetch_traces(self, t0: int, n: int, mesh: int = 0, out_x=None, out_z=None):
        """Traces of steps [t0, t0+n) of all shots, shape (shots, n, n_rec) each; mesh =
        ALL_MESHES: every mesh's block one after the other, flat (sum of shots * n * n_rec)."""
        if mesh == ALL_MESHES:
            shape = (sum(inf["S"] * inf["R"] for inf in self.info) * int(n),)
        else:
            inf = self.info[mesh]
            shape = (inf["S"], int(n), inf["R"])
        ox = np.empty(shape) if out_x is None else out_x
        oz = np.empty(shape) if out_z is None else out_z
        _check(lib().dg_gpu_fetch_traces(self._ctx, mesh, int(t0), int(n), _ptr(ox), _ptr(oz)), "dg_gpu_fetch_traces")
        return ox, oz

    @property
    def steps_done(self) -> int:
        return int(lib().dg_gpu_steps_done(self._ctx))

    def fetch(self, what, mesh: int = 0, shot: int = 0) -> np.ndarray:
        if isinstance(what, str):
            what = FIELDS.get(what, {"trace_x": TRACE_X, "trace_z": TRACE_Z, "energy": ENERGY}.get(what, -99))
        inf = self.info[mesh]
        if what in (VX, VZ, TXX, TZZ, TXZ) and shot == ALL_SHOTS:
            out = np.empty((inf["S"], inf["K"] * 6))
        elif what in (VX, VZ, TXX, TZZ, TXZ):
            out = np.empty(inf["K"] * 6)
        elif what in (TRACE_X, TRACE_Z):
            out = np.empty((min(self.steps_done, inf["T"]), inf["R"]))
        elif what == ENERGY:
            out = np.empty(1)
        else:
            out = np.empty(1)
        if out.size == 0:
            return out
        _check(lib().dg_gpu_fetch(self._ctx, what, mesh, shot, out.ctypes.data), "dg_gpu_fetch")
        return out[0] if what == ENERGY else out

    def load(self, what, values: np.ndarray, mesh: int = 0, shot: int = 0):
        if isinstance(what, str):
            what = FIELDS[what]
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(lib().dg_gpu_load(self._ctx, what, mesh, shot, v.ctypes.data), "dg_gpu_load")

    def reset(self):
        _check(lib().dg_gpu_reset(self._ctx), "dg_gpu_reset")

    def set_wavelet(self, t0: int, w, mesh: int = 0):
        """Wavelet samples from step t0 on; mesh = ALL_MESHES: w holds the same number of samples
        for each mesh, one mesh after the other."""
        if not hasattr(w, "data_ptr"):
            w = np.ascontiguousarray(w, dtype=np.float64)
        n = w.numel() if hasattr(w, "numel") else w.size
        if mesh == ALL_MESHES:
            n //= len(self.info)
        _check(lib().dg_gpu_set_wavelet(self._ctx, mesh, int(t0), n, _ptr(w)), "dg_gpu_set_wavelet")

    def flush_l2(self):
        _check(lib().dg_gpu_flush_l2(self._ctx), "dg_gpu_flush_l2")

    def debug_stall_wave(self, unit: int):
        """Test hook: the stress update of warp unit `unit` of the wavefront step waits on a flag
        that is never published (unit < 0 undoes it); the next step reports DG_ERR_TIMEOUT."""
        _check(lib().dg_gpu_debug_stall_wave(self._ctx, int(unit)), "dg_gpu_debug_stall_wave")

    def stats(self) -> dict:
        s = _Stats()
        _check(lib().dg_gpu_stats_get(self._ctx, C.byref(s)), "dg_gpu_stats_get")
        return {n: getattr(s, n) for n, _ in _Stats._fields_}

    def close(self):
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            lib().dg_gpu_free(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
