"""The C-ABI libraries load and export every function their headers declare (no GPU needed)."""
import ctypes
import os
import re

from conftest import ROOT, pkg

DECL = re.compile(r"^[A-Za-z_][\w \t\*]*?\b((?:dg_gpu|dgh)_\w+)\s*\(", re.M)


def declared(header):
    with open(os.path.join(ROOT, "include", header)) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(DECL.findall(text)))


def test_gpu_library_exports_header():
    lib = ctypes.CDLL(pkg.build.gpu_library())
    names = declared("dg_gpu.h")
    assert "dg_gpu_init" in names and "dg_gpu_step" in names and "dg_gpu_fetch" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.engine.EXPORTS) <= set(names)


def test_host_library_exports_header():
    lib = ctypes.CDLL(pkg.build.host_library())
    names = declared("dg_host.h")
    assert "dgh_build" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_error_strings_without_device():
    lib = pkg.engine.lib()
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8, -9):
        assert lib.dg_gpu_strerror(code)


def test_binding_constants_equal_header():
    """Every #define of dg_gpu.h the Python binding restates has the header's value."""
    with open(os.path.join(ROOT, "include", "dg_gpu.h")) as f:
        defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define (DG_\w+) \(?(-?\d+)L?\)?", f.read(), re.M)}
    e = pkg.engine
    same = {"DG_FP64_REF": e.FP64_REF, "DG_FP64": e.FP64, "DG_FP32": e.FP32, "DG_FP32_KAHAN": e.FP32_KAHAN,
            "DG_VX": e.VX, "DG_VZ": e.VZ, "DG_TXX": e.TXX, "DG_TZZ": e.TZZ, "DG_TXZ": e.TXZ,
            "DG_TRACE_X": e.TRACE_X, "DG_TRACE_Z": e.TRACE_Z, "DG_ENERGY": e.ENERGY,
            "DG_ALL_MESHES": e.ALL_MESHES, "DG_ALL_SHOTS": e.ALL_SHOTS, "DG_PART_ALL": e.PART_ALL,
            "DG_PART_BOUNDARY": e.PART_BOUNDARY, "DG_PART_INTERIOR": e.PART_INTERIOR}
    for name, value in same.items():
        assert defs[name] == value, name
    for code, name in e.ERRORS.items():
        assert defs[name] == code, name
