"""Gradient vectors (bfb_compute_gradients / bfb_get_gradients) against the
oracle's compute_all_gradient_vectors restatement, which is pinned bit for bit
to the reference library (tests/test_oracle.py)."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import log_uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _env(bfb, shape, S, prec, rng, steps=3):
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    env = bfb.Env(shape, S, dx=20.0, precision=prec)
    env.set_coefficients(D, lam)
    env.set_field(rng.random((*shape, S)) * 10)
    act = np.ones(S, np.uint8)
    env.set_dirichlet(act, values=rng.random((*shape, S)) * 5)
    env.simulate(0.01, steps)
    return env


# Shapes cover both kernels: rows of nz*S elements that are a whole number of
# 16-byte vectors take the vectorised kernel (its z neighbours as vectors when
# S is a multiple of the vector width, else per element), the rest the
# per-element kernel; (3, 2, 300) has more vectors per row than threads.
@pytest.mark.parametrize("shape,S", [((5, 4, 6), 2), ((2, 3, 2), 1), ((7, 5, 3), 3), ((3, 6, 1), 2),
                                     ((1, 4, 5), 2), ((4, 1, 3), 1), ((33, 17, 40), 5), ((64, 48, 80), 8),
                                     ((6, 5, 8), 1), ((9, 7, 5), 4), ((4, 3, 2), 6), ((3, 2, 300), 4)])
def test_gradients_fp64_bitexact(bfb, oracle, shape, S):
    rng = np.random.default_rng(sum(shape) * 10 + S)
    env = _env(bfb, shape, S, bfb.FP64, rng)
    field = env.get_field()
    assert np.array_equal(env.gradients(), oracle.gradients(field, 20.0))
    env.close()


def fp32_gradients(f, dx):
    """The reference's arithmetic in IEEE FP32 (numpy float32 operations)."""
    f = np.asarray(f, np.float32)
    h1, h2 = np.float32(dx), np.float32(dx * 2.0)
    out = np.zeros((*f.shape, 3), np.float32)
    for c in range(3):
        n = f.shape[c]
        if n == 1:
            continue
        a = np.moveaxis(f, c, 0)
        g = np.empty_like(a)
        g[0] = (a[1] - a[0]) / h1
        g[-1] = (a[-1] - a[-2]) / h1
        if n > 2:
            g[1:-1] = (a[2:] - a[:-2]) / h2
        out[..., c] = np.moveaxis(g, 0, c)
    return out


@pytest.mark.parametrize("shape,S", [((5, 4, 6), 2), ((33, 17, 40), 5), ((64, 48, 80), 8), ((2, 1, 3), 1),
                                     ((6, 5, 8), 1), ((9, 7, 5), 4), ((7, 5, 3), 3), ((4, 3, 2), 6),
                                     ((3, 2, 300), 4)])
def test_gradients_fp32_bitexact_with_fp32_arithmetic(bfb, shape, S):
    """FP32 envs compute in FP32; checked bit for bit against numpy float32."""
    rng = np.random.default_rng(3 + S)
    env = _env(bfb, shape, S, bfb.FP32, rng)
    field = env.get_field_raw()
    want = fp32_gradients(field, 20.0)
    dev = torch.empty(3 * field.size, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    env.compute_gradients_device(dev.data_ptr())
    env.synchronize()
    assert np.array_equal(dev.cpu().numpy().reshape(want.shape), want)
    assert np.array_equal(env.gradients(), want.astype(np.float64))
    env.close()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_gradients_unaligned_output_takes_the_element_kernel(bfb, prec):
    """An output pointer off a 16-byte boundary selects the per-element
    kernel; its values equal the vectorised kernel's bit for bit."""
    rng = np.random.default_rng(11)
    shape, S = (20, 12, 16), 4
    p = bfb.FP32 if prec == "fp32" else bfb.FP64
    dt = torch.float32 if prec == "fp32" else torch.float64
    env = _env(bfb, shape, S, p, rng)
    n = 3 * int(np.prod(shape)) * S
    aligned = torch.empty(n, dtype=dt, device="cuda")
    shifted = torch.empty(n + 1, dtype=dt, device="cuda")
    torch.cuda.synchronize()
    env.compute_gradients_device(aligned.data_ptr())
    env.compute_gradients_device(shifted.data_ptr() + shifted.element_size())  # 4 or 8 bytes off
    env.synchronize()
    assert np.array_equal(aligned.cpu().numpy(), shifted[1:].cpu().numpy())
    env.close()


def test_gradients_256cube_bandwidth(bfb):
    """The chemotaxis consumer at the bench size: one read of the field,
    three writes; timed with CUDA events on the env's stream and reported,
    not asserted against a roofline."""
    rng = np.random.default_rng(1)
    S = 8
    env = bfb.Env((256, 256, 256), S, precision=bfb.FP32)
    env.set_coefficients(log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S))
    stream = torch.cuda.Stream()
    env.set_stream(stream.cuda_stream)
    n = 256 ** 3 * S
    out = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(3):
        env.compute_gradients_device(out.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        env.compute_gradients_device(out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 10
    gbs = 4 * n * 4 / (ms / 1e3) / 1e9
    print(f"\ngradients 256^3 x 8 FP32: {ms:.3f} ms per call, {gbs:.0f} GB/s of algorithmic traffic (1 read + 3 writes)")
    assert ms > 0
    env.close()
