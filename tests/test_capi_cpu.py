"""CPU tests of the boundary: the CUDA library loads here (no GPU needed to
dlopen it) and exports exactly what include/biofvm_b200.h declares. No
compute call is made."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "biofvm_b200.h").read_text()
    return sorted(set(re.findall(r"BFB_API\s+[\w\s\*]+?\b(bfb_\w+)\s*\(", text)))


def test_header_and_binding_agree(bfb):
    assert header_symbols() == sorted(bfb.EXPORTS)


def test_library_loads_and_exports_every_symbol(bfb):
    L = bfb.load_library()
    for name in header_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(bfb.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (bfb_\w+)", out))
    assert set(header_symbols()) <= exported


def test_last_error_and_version_need_no_gpu(bfb):
    L = bfb.load_library()
    assert L.bfb_version() >= 100
    assert isinstance(L.bfb_last_error(), bytes)


def test_null_handle_is_rejected_without_gpu(bfb):
    L = bfb.load_library()
    assert L.bfb_destroy(None) == 0
    assert L.bfb_set_option(None, 1, 1) == -1
    assert b"null" in L.bfb_last_error()
    assert L.bfb_watchdog_selftest(None, 8) == -1
    assert L.bfb_host_register(None, 8) == -1
    assert L.bfb_host_unregister(None) == -1
    assert L.bfb_field_pitch(None, None) == -1


def test_create_validates_arguments_before_touching_a_device(bfb):
    """bfb_create / bfb_create_domain reject bad arguments with their own
    status, before any CUDA call (so the same codes come back with or without
    a GPU)."""
    import ctypes

    L = bfb.load_library()
    h = ctypes.c_void_p()

    def create(nx=4, ny=4, nz=4, S=1, dx=20.0, prec=0, out=True):
        return L.bfb_create(ctypes.byref(h) if out else None, nx, ny, nz, S, dx, prec, 0)

    assert create(out=False) == -1
    assert create(nx=0) == -2 and create(nz=-3) == -2 and create(S=0) == -2
    assert create(dx=0.0) == -1 and create(dx=-1.0) == -1
    assert create(dx=float("nan")) == -1 and create(dx=float("inf")) == -1
    assert create(prec=7) == -1
    assert create(nx=2048, ny=2048, nz=2048) == -2  # more than 2^31-1 voxels

    def domain(x1=80.0, y1=80.0, z1=80.0, dx=20.0):
        return L.bfb_create_domain(ctypes.byref(h), 0.0, x1, 0.0, y1, 0.0, z1, dx, 1, 0, 0)

    assert domain(dx=0.0) == -1 and domain(dx=float("nan")) == -1
    assert domain(x1=-40.0) == -2  # x1 < x0
    assert domain(y1=1e300) == -2  # beyond 2^31-1 voxels on an axis
    assert domain(z1=float("nan")) == -2 and domain(x1=float("inf")) == -2
    assert L.bfb_create_domain(None, 0.0, 80.0, 0.0, 80.0, 0.0, 80.0, 20.0, 1, 0, 0) == -1


def test_noalloc_checksum_validates_arguments_before_any_cuda_call(bfb):
    """bfb_checksum_noalloc's argument checks come first; the pointers below
    are never dereferenced because every call returns at a check."""
    import ctypes

    L = bfb.load_library()
    p = ctypes.c_void_p(256)  # a non-NULL value; never used
    assert L.bfb_checksum_noalloc(None, 0, 8, 1, p, None) == -1
    assert L.bfb_checksum_noalloc(p, 0, 8, 1, None, None) == -1
    assert L.bfb_checksum_noalloc(p, 5, 8, 1, p, None) == -1
    assert L.bfb_checksum_noalloc(p, 0, -1, 1, p, None) == -1
    assert L.bfb_checksum_noalloc(p, 0, 8, 0, p, None) == -1
    assert L.bfb_checksum_noalloc(p, 1, 8, 65, p, None) == -2
    assert b"64" in L.bfb_last_error()


def test_env_fails_loudly_without_a_gpu(bfb):
    """No CPU fallback: creating an env where no CUDA device is visible raises
    the library's CUDA error rather than computing anything on the host."""
    import pytest
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(bfb.BFBError) as ei:
        bfb.Env((4, 4, 4), 1)
    assert ei.value.code == -4
