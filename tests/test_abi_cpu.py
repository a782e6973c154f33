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
