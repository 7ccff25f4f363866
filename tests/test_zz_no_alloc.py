"""bfb_checksum_noalloc: per-substrate field sums without any device allocation.

Some callers cannot let a library allocate device memory: code that keeps
its device buffers in its own pool, or a host loop with other streams in
flight, which cudaMalloc/cudaFree would stall because they synchronize the
device. bfb_checksum_noalloc gives them the sums of bfb_checksum with its
scratch in a fixed array inside the library. This test calls it through the
C ABI on an env's device field and checks two calls in a row against
bfb_checksum. It sits in its own file, collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-12  # the tolerance the other checksum test uses


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_noalloc_checksum_matches_env_checksum_twice(bfb, precision):
    import torch

    rng = np.random.default_rng(77)
    shape, S = (40, 36, 28), 5
    env = bfb.Env(shape, S, precision=precision)
    env.set_field(rng.random((*shape, S)) * 3.0)
    want = env.checksum()  # the existing entry point (allocates its scratch)

    L = bfb.load_library()
    out = torch.zeros(S, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    V = shape[0] * shape[1] * shape[2]
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out.zero_()
        rc = L.bfb_checksum_noalloc(ctypes.c_void_p(env.field_device_ptr()), precision, V, S,
                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.bfb_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, want, rtol=RTOL, atol=0), (got, want)
    env.close()


def test_noalloc_checksum_rejects_too_many_substrates(bfb):
    import torch

    L = bfb.load_library()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.bfb_checksum_noalloc(ctypes.c_void_p(buf.data_ptr()), 0, 1, 65, ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == -2
    assert b"64" in L.bfb_last_error()
