"""CPU test of the C++ facade's host-only logic: tests/facade_host_check.cpp
is compiled against the facade library and run; it makes no device call. Its
print_result text dump is compared byte for byte with the reference's own
(oracle/_ref) where that library is built."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "biofvm-b_b200" / "lib"


def test_facade_mesh_resize_compare_nonuniform_refusal_and_print_result(tmp_path):
    if not (LIB / "libbiofvm_b200_host.so").exists():
        pytest.fail("facade library missing: build it with `python biofvm-b_b200/build.py`")
    exe = tmp_path / "facade_host_check"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-ffp-contract=off", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'biofvm-b_b200' / 'host'}", "-o", str(exe), str(ROOT / "tests" / "facade_host_check.cpp"),
                    f"-L{LIB}", "-lbiofvm_b200_host", "-lbiofvm_b200", f"-Wl,-rpath,{LIB}"], check=True)
    dump = tmp_path / "densities.txt"
    r = subprocess.run([str(exe), str(dump)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
    assert "uniform Cartesian meshes" in r.stdout  # the solver's refusal was printed
    lines = dump.read_text().splitlines()
    assert len(lines) == 60 and lines[0] == "0 0 0 : 0 0.142857 "
    assert lines[-1] == "2 3 4 : 5.9 6.04286 "

    from oracle.oracle import REF_SO, RefEnv, RefLib
    if not REF_SO.exists():
        return
    # the reference's own print_voxels_densities, on the same field: the same bytes
    import numpy as np
    ref = RefEnv(RefLib(), (0.0, 0.0, 0.0, 60.0, 80.0, 100.0), 20.0, [1e3, 1e4], [0.1, 0.2])
    n = np.arange(60, dtype=float)[:, None]
    d = np.arange(2, dtype=float)[None, :]
    ref.set_field((n * 0.1 + d / 7.0).reshape(3, 4, 5, 2))
    ref_dump = tmp_path / "ref_densities.txt"
    ref.print_densities(ref_dump)
    assert ref_dump.read_bytes() == dump.read_bytes()
