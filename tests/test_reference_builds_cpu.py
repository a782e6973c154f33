"""The two builds of the reference's own C code in oracle/_ref: the parity build (-O2) that pins
the golden fixtures, and the throughput build (-O3, x86-64-v3) that the CPU baseline times.
Floating-point contraction is off in both and GCC reorders no floating-point operation without
-ffast-math, so the throughput build writes the same bytes."""
import os
import sys

import pytest

from conftest import pkg

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import refrun  # noqa: E402


def test_throughput_build_writes_the_parity_builds_bytes(tmp_path):
    w = pkg.workloads.small_square(n_cells=12, steps=60, shots=2)
    if not (refrun.available(w) and refrun.available(w, fast=True)):
        pytest.skip("reference builds not present (oracle/_ref is built where the reference sources are)")
    a = refrun.run(w, str(tmp_path / "parity"), steps=60, snap_every=20, threads=2)
    b = refrun.run(w, str(tmp_path / "fast"), steps=60, snap_every=20, threads=2, fast=True)
    names = sorted(n for n in os.listdir(a["out"]) if n.endswith(".bin"))
    assert names and names == sorted(n for n in os.listdir(b["out"]) if n.endswith(".bin"))
    for n in names:
        with open(os.path.join(a["out"], n), "rb") as f, open(os.path.join(b["out"], n), "rb") as g:
            assert f.read() == g.read(), n
