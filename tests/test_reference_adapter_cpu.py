"""The B200 solver adapter (biofvm-b_b200/host/reference_adapter/) inside a
reference build, made by `make -C oracle adapter`: it compiles against the
reference's own headers with the one friend declaration it documents, links
against the reference's objects and this library, and, where no CUDA device
is visible, fails loudly and leaves the reference's field untouched. (With a
device, the same driver prints "identical <steps>" when the adapter's steps
equal the reference LOD_3D's bit for bit.)"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from oracle.oracle import REF_SO

ROOT = Path(__file__).resolve().parents[1]
DRIVER = ROOT / "oracle" / "_ref" / "adapter_driver"


def test_adapter_builds_into_the_reference_and_fails_loudly_without_a_device():
    if not REF_SO.exists():
        pytest.skip("reference library not built here")
    r = subprocess.run(["make", "-C", str(ROOT / "oracle"), "adapter"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible; this test covers the path without one")
    out = subprocess.run([str(DRIVER), "3"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "B200 solver: bfb_create" in out.stdout
    assert out.stdout.strip().splitlines()[-1] == "unchanged"
