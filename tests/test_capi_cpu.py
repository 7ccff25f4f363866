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
