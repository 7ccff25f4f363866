"""CPU test of the C++ facade's host-only logic: tests/facade_host_check.cpp
is compiled against the facade library and run; it makes no device call."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "biofvm-b_b200" / "lib"


def test_facade_mesh_resize_compare_and_nonuniform_refusal(tmp_path):
    if not (LIB / "libbiofvm_b200_host.so").exists():
        pytest.fail("facade library missing: build it with `python biofvm-b_b200/build.py`")
    exe = tmp_path / "facade_host_check"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-ffp-contract=off", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'biofvm-b_b200' / 'host'}", "-o", str(exe), str(ROOT / "tests" / "facade_host_check.cpp"),
                    f"-L{LIB}", "-lbiofvm_b200_host", "-lbiofvm_b200", f"-Wl,-rpath,{LIB}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
    assert "uniform Cartesian meshes" in r.stdout  # the solver's refusal was printed
