"""bfb_checksum_noalloc: per-substrate field sums without any device allocation.

Some callers cannot let a library allocate device memory: code that keeps
its device buffers in its own pool, or a host loop with other streams in
flight, which cudaMalloc/cudaFree would stall because they synchronize the
device. bfb_checksum_noalloc gives them the sums of bfb_checksum with its
scratch in a fixed array inside the library. This test calls it through the
C ABI on an env's device field and checks two calls in a row against the
existing entry point bfb_checksum and against a float64 numpy sum of the
field as set. It sits in its own file, collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-12  # the tolerance the other checksum test uses


def _noalloc(bfb, env, precision, V, S):
    import torch

    L = bfb.load_library()
    out = torch.zeros(S, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.bfb_checksum_noalloc(ctypes.c_void_p(env.field_device_ptr()), precision, V, S,
                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.bfb_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


# (40, 36, 28) x 5: many voxels per reduction block; (5, 4, 3) x 64: fewer
# voxels than reduction blocks and the largest substrate count allowed
@pytest.mark.parametrize("shape,S", [((40, 36, 28), 5), ((5, 4, 3), 64)], ids=["40x36x28_S5", "5x4x3_S64"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_noalloc_checksum_matches_env_checksum_twice(bfb, precision, shape, S):
    rng = np.random.default_rng(77)
    rho = rng.random((*shape, S)) * 3.0
    env = bfb.Env(shape, S, precision=precision)
    env.set_field(rho)
    want = env.checksum()  # the existing entry point (allocates its scratch)
    as_set = rho if precision == 0 else rho.astype(np.float32).astype(np.float64)
    V = shape[0] * shape[1] * shape[2]
    want_np = as_set.reshape(V, S).sum(axis=0, dtype=np.float64)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        got = _noalloc(bfb, env, precision, V, S)
        assert np.allclose(got, want, rtol=RTOL, atol=0), (got, want)
        assert np.allclose(got, want_np, rtol=RTOL, atol=0), (got, want_np)
    env.close()


def test_noalloc_checksum_rejects_too_many_substrates(bfb):
    import torch

    L = bfb.load_library()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.bfb_checksum_noalloc(ctypes.c_void_p(buf.data_ptr()), 0, 1, 65, ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == -2
    assert b"64" in L.bfb_last_error()
