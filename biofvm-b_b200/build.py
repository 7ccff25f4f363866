"""Build recipe of the product library (no torch involved).

    python biofvm-b_b200/build.py          # -> biofvm-b_b200/lib/libbiofvm_b200.so

Compiles the CUDA sources for sm_100a only, in-tree, with nvcc. FP64 parity
with the reference depends on two flags: --fmad=false (device code fuses only
where the source says __fma_rn) and -ffp-contract=off for host code (the
Thomas factors are computed on the host with explicit std::fma).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libbiofvm_b200.so"
SOURCES = ["bfb_capi.cu", "bfb_sweeps.cu", "bfb_tma.cu", "bfb_aux.cu", "bfb_batch.cu", "bfb_noalloc.cu", "bfb_adjoint.cu", "bfb_gradient.cu", "bfb_matlab.cu", "bfb_tmem.cu", "bfb_slab.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
         f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    deps = ([CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "biofvm_b200.h"] +
            list((PKG / "host").rglob("*.cpp")) + list((PKG / "host").glob("*.h")))
    newest = max(p.stat().st_mtime for p in deps)
    if LIB.exists() and LIB.stat().st_mtime >= newest and not force:
        return LIB
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    objs = [obj_dir / (Path(s).stem + ".o") for s in SOURCES]
    # one nvcc per translation unit, in parallel
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as pool:
        list(pool.map(lambda so: _run([NVCC, *ARCH, *FLAGS, *extra, "-c", CSRC / so[0], "-o", so[1]]),
                      zip(SOURCES, objs)))
    _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    build_host()
    return LIB


HOST_LIB = LIB_DIR / "libbiofvm_b200_host.so"
DEMO = LIB_DIR / "facade_demo"
CXX = "/usr/bin/g++"


def build_host() -> None:
    """The C++ facade (host/) over the C ABI, and its example driver."""
    inc = [f"-I{ROOT / 'include'}", f"-I{PKG / 'host'}"]
    flags = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall"]
    _run([CXX, *flags, *inc, "-shared", "-o", HOST_LIB, PKG / "host" / "BioFVM_B200.cpp", f"-L{LIB_DIR}",
          "-lbiofvm_b200", "-Wl,-rpath,$ORIGIN"])
    _run([CXX, *flags, *inc, "-o", DEMO, PKG / "host" / "examples" / "facade_demo.cpp", f"-L{LIB_DIR}",
          "-lbiofvm_b200_host", "-lbiofvm_b200", "-Wl,-rpath,$ORIGIN"])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
