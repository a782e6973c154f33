"""ctypes binding of the C host set-up library (csrc/dg_host.c, include/dg_host.h).

``build_setup`` turns a :class:`workloads.Workload` (or a mesh read from the converted text
files) into every array the reference's host code hands the time loop: the 1-based index maps,
the per-element operator arrays, the sponge, sources, receivers, ``dt`` and the wavelet table.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import build as _build
from . import operators

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build.host_library()
        _LIB = C.CDLL(path)
        _LIB.dgh_build.argtypes = [C.c_void_p, C.c_void_p]
        _LIB.dgh_build.restype = C.c_int
        _LIB.dgh_strerror.restype = C.c_char_p
        _LIB.dgh_strerror.argtypes = [C.c_int]
        _LIB.dgh_read_matrix.restype = C.c_long
        _LIB.dgh_read_matrix.argtypes = [C.c_char_p, C.c_void_p, C.c_long, C.c_long]
        _LIB.dgh_read_int_matrix.restype = C.c_long
        _LIB.dgh_read_int_matrix.argtypes = [C.c_char_p, C.c_void_p, C.c_long, C.c_long]
        _LIB.dgh_read_mesh.restype = C.c_int
        _LIB.dgh_read_mesh.argtypes = [C.c_char_p, C.c_void_p]
        _LIB.dgh_free_mesh.argtypes = [C.c_void_p]
        _LIB.dgh_quantize_e7.argtypes = [C.c_void_p, C.c_long]
        _LIB.dgh_ricker.restype = C.c_double
        _LIB.dgh_ricker.argtypes = [C.c_long, C.c_double, C.c_double, C.c_double, C.c_double]
        _LIB.dgh_write_matrix.restype = C.c_int
        _LIB.dgh_write_matrix.argtypes = [C.c_char_p, C.c_void_p, C.c_long, C.c_long]
        _LIB.dgh_write_binary.restype = C.c_int
        _LIB.dgh_write_binary.argtypes = [C.c_char_p, C.c_void_p, C.c_long]
        _LIB.dgh_write_record.restype = C.c_int
        _LIB.dgh_write_record.argtypes = [C.c_char_p, C.c_void_p, C.c_long]
        _LIB.dgh_parse_e7.restype = C.c_double
        _LIB.dgh_parse_e7.argtypes = [C.c_char_p, C.c_long]
    return _LIB


class HostError(RuntimeError):
    pass


def _check(rc):
    if rc < 0:
        raise HostError("dg_host: %s (%d)" % (lib().dgh_strerror(int(rc)).decode(), rc))
    return rc


def _p(a):
    return None if a is None else a.ctypes.data


class _SetupIn(C.Structure):
    _fields_ = [("K", C.c_long), ("n_points", C.c_long), ("Point", C.c_void_p), ("Triangle", C.c_void_p),
                ("neighbor", C.c_void_p), ("vp", C.c_void_p), ("vs", C.c_void_p), ("rho", C.c_void_p),
                ("V", C.c_void_p), ("Vr", C.c_void_p), ("Vs", C.c_void_p), ("inverV", C.c_void_p),
                ("S1", C.c_void_p), ("S2", C.c_void_p), ("S3", C.c_void_p), ("Fekete", C.c_void_p),
                ("fp", C.c_double), ("pi", C.c_double), ("beta", C.c_double), ("bound_x", C.c_double),
                ("bound_z", C.c_double), ("model_w", C.c_double), ("model_h", C.c_double),
                ("n_shots", C.c_long), ("src_pos", C.c_void_p), ("n_rec", C.c_long), ("rec_pos", C.c_void_p),
                ("n_steps", C.c_long)]


_OUT_ARRAYS = ["A", "B", "Jacobi", "Jacobi_Edge", "normal1", "normal2", "normal3", "Q", "Dx", "Dz", "S", "ibe",
               "Neighbor", "Edge", "Edge_flag", "Node_Neighbor", "absorb_fun", "source", "fun", "receiver",
               "wavelet", "Vp_used"]


class _SetupOut(C.Structure):
    _fields_ = [("dt", C.c_double), ("t0", C.c_double), ("absorb_count", C.c_long), ("absorb_filled", C.c_long)] + \
               [(n, C.c_void_p) for n in _OUT_ARRAYS]


class _Mesh(C.Structure):
    _fields_ = [("K", C.c_long), ("n_points", C.c_long), ("Point", C.c_void_p), ("Triangle", C.c_void_p),
                ("neighbor", C.c_void_p), ("attribute", C.c_void_p)]


@dataclasses.dataclass
class Setup:
    """The arrays the reference's host code produces for the time loop (1-based int64 maps)."""
    K: int
    n_points: int
    Point: np.ndarray
    Triangle: np.ndarray
    dt: float
    t0: float
    absorb_count: int
    absorb_filled: int
    arrays: dict
    ops: dict
    n_shots: int
    n_rec: int
    n_steps: int

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)


def read_text_operators(matrix_dir: str) -> dict:
    """Read the ten operator text files with the reference parser (ReadDouble)."""
    out = {}
    for name, shape in operators.SHAPES.items():
        a = np.zeros(shape, dtype=np.float64)
        _check(lib().dgh_read_matrix(os.path.join(matrix_dir, name + ".txt").encode(), a.ctypes.data, *shape))
        out[name] = a
    return out


def text_operators() -> dict:
    """The P2 operators as the reference pipeline sees them: restated, printed at 8 significant
    digits and parsed back by the reference parser."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        operators.write_text_files(d)
        return read_text_operators(d)


def read_mesh(prefix: str):
    m = _Mesh()
    _check(lib().dgh_read_mesh(prefix.encode(), C.byref(m)))
    try:
        K, P = m.K, m.n_points
        pts = np.ctypeslib.as_array(C.cast(m.Point, C.POINTER(C.c_double)), shape=(P * 2,)).copy().reshape(P, 2)
        tri = np.ctypeslib.as_array(C.cast(m.Triangle, C.POINTER(C.c_long)), shape=(K * 3,)).copy().reshape(K, 3)
        nb = np.ctypeslib.as_array(C.cast(m.neighbor, C.POINTER(C.c_long)), shape=(K * 3,)).copy().reshape(K, 3)
        at = np.ctypeslib.as_array(C.cast(m.attribute, C.POINTER(C.c_long)), shape=(K,)).copy()
    finally:
        lib().dgh_free_mesh(C.byref(m))
    return pts, tri, nb, at


def quantize_e7(x: np.ndarray) -> np.ndarray:
    """Values after the ``%16.7e`` text round trip of the reference pipeline."""
    y = np.ascontiguousarray(x, dtype=np.float64).copy()
    lib().dgh_quantize_e7(y.ctypes.data, y.size)
    return y


def build_setup(w, *, ops: dict | None = None, mesh_arrays=None, full: bool = True, n_steps: int | None = None,
                quantize: bool = True) -> Setup:
    """Run the host set-up for workload ``w``.

    ``mesh_arrays`` = (Point, Triangle 1-based, neighbor 1-based/-1) overrides the in-memory mesh
    (e.g. as read back from the text files).  Without it the in-memory mesh coordinates are
    ``quantize``d through the text format, so the result equals the file-based pipeline.
    ``full`` also produces Dx/Dz/Q/normals (only the bit-exact reference-operator path needs
    them; at 2M elements they take 1.6 GB of host memory).
    """
    ops = text_operators() if ops is None else ops
    if mesh_arrays is None:
        pts = quantize_e7(w.mesh.points) if quantize else np.ascontiguousarray(w.mesh.points, dtype=np.float64)
        tri = np.ascontiguousarray(w.mesh.tris + 1, dtype=np.int64)
        nb = np.where(w.mesh.neigh >= 0, w.mesh.neigh + 1, -1).astype(np.int64)
    else:
        pts, tri, nb = (np.ascontiguousarray(a) for a in mesh_arrays[:3])
        pts = pts.astype(np.float64)
        tri = tri.astype(np.int64)
        nb = nb.astype(np.int64)
    K = tri.shape[0]
    P = pts.shape[0]
    S = w.shots
    R = w.rec.shape[0]
    T = int(w.steps if n_steps is None else n_steps)
    vp = np.ascontiguousarray(w.vp, dtype=np.float64)
    vs = np.ascontiguousarray(w.vs, dtype=np.float64)
    rho = np.ascontiguousarray(w.rho, dtype=np.float64)
    src = np.ascontiguousarray(w.src, dtype=np.float64)
    rec = np.ascontiguousarray(w.rec, dtype=np.float64)
    opc = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in ops.items()}
    si = _SetupIn(K=K, n_points=P, Point=_p(pts), Triangle=_p(tri), neighbor=_p(nb), vp=_p(vp), vs=_p(vs),
                  rho=_p(rho), V=_p(opc["V"]), Vr=_p(opc["Vr"]), Vs=_p(opc["Vs"]), inverV=_p(opc["inverV"]),
                  S1=_p(opc["S1"]), S2=_p(opc["S2"]), S3=_p(opc["S3"]), Fekete=_p(opc["FeketeNew"]),
                  fp=float(w.fp), pi=float(w.pi), beta=float(w.beta), bound_x=float(w.sponge[0]),
                  bound_z=float(w.sponge[1]), model_w=float(w.sponge[2]), model_h=float(w.sponge[3]),
                  n_shots=S, src_pos=_p(src), n_rec=R, rec_pos=_p(rec), n_steps=T)
    shapes = {"A": (K, 5), "B": (K, 5), "Jacobi": (K,), "Jacobi_Edge": (K, 3), "normal1": (K, 2),
              "normal2": (K, 2), "normal3": (K, 2), "Q": (K, 3, 5, 2), "Dx": (K, 6, 6), "Dz": (K, 6, 6),
              "S": (3, 6, 3), "ibe": (3, 3), "Neighbor": (K, 3), "Edge": (K, 3), "Edge_flag": (K, 3),
              "Node_Neighbor": (K, 3, 3), "absorb_fun": (K, 6), "source": (S, 2), "fun": (S, 6),
              "receiver": (R, 2), "wavelet": (T,), "Vp_used": (K,)}
    ints = {"ibe", "Neighbor", "Edge", "Edge_flag", "Node_Neighbor", "source", "receiver"}
    skip = set() if full else {"Q", "Dx", "Dz", "normal1", "normal2", "normal3", "Jacobi_Edge"}
    arrays = {}
    so = _SetupOut()
    for name in _OUT_ARRAYS:
        if name in skip:
            continue
        a = np.zeros(shapes[name], dtype=np.int64 if name in ints else np.float64)
        arrays[name] = a
        setattr(so, name, a.ctypes.data if a.size else None)
    _check(lib().dgh_build(C.byref(si), C.byref(so)))
    return Setup(K=K, n_points=P, Point=pts, Triangle=tri, dt=so.dt, t0=so.t0, absorb_count=so.absorb_count,
                 absorb_filled=so.absorb_filled, arrays=arrays, ops=opc, n_shots=S, n_rec=R, n_steps=T)
