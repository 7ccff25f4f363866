"""The B200 solver behind the reference's own plugin point, on the device.

`oracle/_ref/adapter_driver` is a reference build (the reference's objects,
compiled from its sources by `make -C oracle adapter`) with the adapter
`biofvm-b_b200/host/reference_adapter/BioFVM_b200_solver.cpp` linked in and
registered in `Microenvironment::diffusion_decay_solver`
(BioFVM_microenvironment.h:164), the pointer `simulate_diffusion_decay` calls
(BioFVM_microenvironment.cpp:1018-1029). It steps one Microenvironment
through the reference's LOD_3D and an identical one through the adapter and
prints "identical <steps>" when the two fields agree bit for bit.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
DRIVER = ROOT / "oracle" / "_ref" / "adapter_driver"


def run_driver(*args, timeout=600):
    assert DRIVER.exists(), f"{DRIVER} is missing: build it with `make -C oracle adapter`"
    out = subprocess.run([str(DRIVER), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "B200 solver:" not in out.stdout, out.stdout[-2000:]  # the adapter reported no error
    return out.stdout.strip().splitlines()[-1]


def test_adapter_identical_to_lod3d_small_grid():
    """12 x 10 x 8 voxels, 3 substrates, default faces (100.0) with substrate 1
    deactivated, 5 steps: cp.async tiles."""
    assert run_driver(5) == "identical 5"


def test_adapter_identical_to_lod3d_tma_grid_with_dt_change():
    """64 x 48 x 40 voxels, 3 substrates (every pitch suits the TMA tiles),
    default faces with substrate 1 deactivated; after the first step dt
    changes to 0.02, which both solvers ignore (their factors stay at the first
    call's, BioFVM_parallel.cpp:714, 913)."""
    assert run_driver("compare", 4, 1280, 960, 800, 3, 0.02) == "identical 4"


def test_adapter_identical_to_lod3d_unaligned_grid():
    """15 x 13 x 11 voxels, 5 substrates: no row pitch is a multiple of 16
    bytes (cp.async tiles), default faces, substrate 1 deactivated."""
    assert run_driver("compare", 3, 300, 260, 220, 5) == "identical 3"


def test_adapter_end_to_end_time_256cube_s8():
    """The drop-in's own end-to-end cost: a 256^3 x 8 reference Microenvironment
    (default Dirichlet faces) stepped through the adapter, each step copying
    the field in and out of its page-locked std::vector."""
    line = run_driver("time", 256, 8, 10, timeout=1200)
    assert line.startswith("ms_per_step ")
    ms = float(line.split()[1])
    print(f"\nadapter end to end, 256^3 x 8 FP64: {ms:.2f} ms per step "
          f"({256 ** 3 * 8 / (ms / 1e3):.3e} voxel*substrate updates/s)")
    assert ms > 0
