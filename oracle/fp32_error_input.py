"""Writes the input of oracle/fp32_error.c for the benchmark's workload: the
seeded D, lambda and U[0,1) field of bench.py at an n^3 x 8 grid.

    python oracle/fp32_error_input.py <n> <steps> <out.bin>

Test infrastructure (the oracle).
"""
from __future__ import annotations

import importlib.util
import struct
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def main(n: int, steps: int, out: str) -> None:
    spec = importlib.util.spec_from_file_location("bench", ROOT / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.NX = b.NY = b.NZ = n
    D, lam, rng = b.coefficients()
    rho0 = b.initial_field(rng)
    with open(out, "wb") as f:
        f.write(struct.pack("5i", n, n, n, b.S, steps))
        f.write(np.asarray(D, np.float64).tobytes())
        f.write(np.asarray(lam, np.float64).tobytes())
        f.write(np.ascontiguousarray(rho0, np.float64).tobytes())


if __name__ == "__main__":
    main(int(sys.argv[1]), int(sys.argv[2]), sys.argv[3])
