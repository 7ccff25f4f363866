"""The FP32 path pinned bit for bit to its CPU restatement.

The FP32 kernels are not a reference function: the reference has no FP32
solver. `orc_lod_steps_f32`, `orc_bulk_step_f32` and `orc_cells_step_f32`
(oracle/lod_oracle.c) restate them operation by operation -- the factor
tables rounded once from the reference's FP64 factors, the deviation-form
line solve with the reciprocal as hi + lo, the face values rounded to FP32,
the bulk update and the agents' update in binary32. Here the device's FP32
field must EQUAL that restatement after every case: Dirichlet faces on all
six faces, on the x faces only and with per-voxel values, fused bulk and
agents sharing voxels, the TMA, cp.async and long-line kernels, S from 1 to
33. The tolerance of the FP32 path against FP64 (<= 1e-5 relative L-inf
after each workload's step count) is then a property of the restatement,
which the CPU can evaluate at full size.
"""
from __future__ import annotations

import zlib

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import face_mask_all

pytestmark = pytest.mark.gpu
DT, DX = 0.01, 20.0


def fp32_env(bfb, rho, D, lam, tma):
    nx, ny, nz, S = rho.shape
    env = bfb.Env((nx, ny, nz), S, dx=DX, precision=bfb.FP32)
    env.set_option(bfb.OPT_USE_TMA, tma)
    env.set_coefficients(D, lam)
    env.set_field(rho)
    return env


def dirichlet_case(mode, rng, shape, S):
    """(activation, per-voxel values, face mask [6][S]) of a Dirichlet mode."""
    act = np.ones(S, np.uint8)
    if S > 1:
        act[1] = 0  # one inactive substrate in every mode
    if mode == "none":
        return None, None, None
    if mode == "all_faces_uniform":
        vals = np.broadcast_to(np.linspace(1.0, 38.0, S), (*shape, S)).copy()
        return act, vals, None
    if mode == "x_faces_only":
        vals = np.broadcast_to(np.full(S, 38.0), (*shape, S)).copy()
        mask = np.zeros((6, S), np.uint8)
        mask[0:2, :] = 1
        return act, vals, mask
    if mode == "per_voxel_values":
        return act, rng.random((*shape, S)) * 10.0, None
    raise ValueError(mode)


def run_both(bfb, oracle, rng, shape, S, tma, mode, steps=3):
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    act, vals, mask = dirichlet_case(mode, rng, shape, S)
    env = fp32_env(bfb, rho0, D, lam, tma)
    fm = None
    if act is not None:
        env.set_dirichlet(act, values=vals, face_mask=mask)
        fm = face_mask_all(act) if mask is None else (mask & act[None, :])
    env.simulate(DT, steps, bfb.STEP_DIFFUSION)
    got = env.get_field_raw()
    env.close()
    want = oracle.lod_steps_f32(rho0, DT, DX, D, lam, steps, vals, fm)
    return got, want


PIN_SHAPES = [((24, 20, 16), 1), ((24, 20, 16), 3), ((24, 20, 16), 8), ((15, 13, 11), 3), ((17, 9, 33), 5),
              ((6, 5, 7), 33), ((1, 4, 6), 2), ((2, 3, 1), 3), ((40, 3, 64), 7),
              ((100, 6, 8), 3), ((5, 130, 4), 2),  # lines of about 100 rows
              ((20, 9, 16), 5), ((10, 10, 10), 6), ((9, 7, 12), 7)]  # z rows of whole 16-byte vectors, S not 4 or 8


@pytest.mark.parametrize("mode", ["none", "all_faces_uniform", "x_faces_only", "per_voxel_values"])
@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
@pytest.mark.parametrize("shape,S", PIN_SHAPES, ids=[f"{a}x{b}x{c}_S{s}" for (a, b, c), s in PIN_SHAPES])
def test_fp32_bitexact_with_restatement(bfb, oracle, shape, S, tma, mode):
    rng = np.random.default_rng(zlib.crc32(repr((shape, S, mode)).encode()))
    got, want = run_both(bfb, oracle, rng, shape, S, tma, mode)
    assert got.dtype == np.float32 and want.dtype == np.float32
    assert np.array_equal(got, want), f"max |diff| {np.abs(got - want).max():.3e}"


@pytest.mark.parametrize("shape,S", [((1900, 3, 2), 2), ((2, 1900, 3), 1), ((2, 3, 1900), 2)],
                         ids=["x_long", "y_long", "z_long"])
def test_fp32_long_lines_bitexact(bfb, oracle, shape, S):
    """Lines too long for a shared-memory tile run the global-memory kernels."""
    rng = np.random.default_rng(11)
    got, want = run_both(bfb, oracle, rng, shape, S, 1, "per_voxel_values", steps=2)
    assert np.array_equal(got, want), f"max |diff| {np.abs(got - want).max():.3e}"


@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
@pytest.mark.parametrize("shape,S", [((16, 12, 8), 4), ((15, 13, 11), 3)], ids=["16x12x8_S4", "15x13x11_S3"])
def test_fp32_bulk_diffusion_agents_bitexact(bfb, oracle, shape, S, tma):
    """Bulk fused into the x-sweep load, Dirichlet faces, then agents (many per
    voxel), for three composite steps, against bulk -> LOD -> agents restated."""
    rng = np.random.default_rng(31)
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    Sr, Tt, Ur = rng.random((3, *shape, S)) * 4.0
    act = np.ones(S, np.uint8)
    act[1] = 0
    vals = rng.random((*shape, S)) * 5.0
    n = 400
    ext = np.array(shape) * DX
    pos = rng.uniform(0.0, 1.0, (n, 3)) * ext * 0.5 + ext * 0.25  # crowded centre: agents share voxels
    vol = np.full(n, 4.0 / 3.0 * np.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, n, S))
    active = (rng.random(n) > 0.1).astype(np.uint8)

    env = fp32_env(bfb, rho0, D, lam, tma)
    env.set_dirichlet(act, values=vals)
    env.set_bulk(Sr, Tt, Ur)
    env.set_agents(pos, vol, sec, upt, sat, DT, active=active)
    env.simulate(DT, 3, bfb.STEP_BULK | bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    got = env.get_field_raw()
    env.close()

    vox = oracle.bin_agents(pos, (0, 0, 0, *ext), DX, shape)
    vox = np.where(vox < 0, 0, vox)
    t1, t2 = oracle.agent_constants(DT, DX, vol, sec, upt, sat)
    want = rho0.astype(np.float32)
    for _ in range(3):
        want = oracle.bulk_step_f32(want, DT, Sr, Tt, Ur)
        want = oracle.lod_steps_f32(want, DT, DX, D, lam, 1, vals, face_mask_all(act))
        want = oracle.cells_step_f32(want, vox, t1, t2, active)
    assert np.array_equal(got, want), f"max |diff| {np.abs(got - want).max():.3e}"


def test_cube75_s1_fp32_on_the_device(bfb, oracle):
    """The 75^3 single-substrate workload in FP32 on the device: 75^3 x 1,
    D = 1e5, lambda = 0.1, dt = 0.01, 100 steps, Dirichlet 1.0 on all faces,
    U[0,1) field. The FP32 field equals the restatement bit for bit, and its
    error against the FP64 path (bit-exact with the reference) is printed and
    bounded by 1e-5 relative L-inf."""
    rng = np.random.default_rng(2024)
    rho0 = rng.random((75, 75, 75, 1))
    envs = {}
    for prec in (bfb.FP32, bfb.FP64):
        env = bfb.Env((75, 75, 75), 1, dx=DX, precision=prec)
        env.set_coefficients([1e5], [0.1])
        env.set_field(rho0)
        env.set_dirichlet_uniform([1], [1.0])
        env.simulate(DT, 100, bfb.STEP_DIFFUSION)
        envs[prec] = env
    linf, l2 = envs[bfb.FP32].compare(envs[bfb.FP64])
    got = envs[bfb.FP32].get_field_raw()
    for e in envs.values():
        e.close()
    want = oracle.lod_steps_f32(rho0, DT, DX, [1e5], [0.1], 100, np.ones_like(rho0), face_mask_all([1]))
    print(f"\n75^3 x 1, 100 steps, Dirichlet 1.0: FP32 vs FP64 on the device rel L-inf {linf:.3e}, rel L2 {l2:.3e}")
    assert np.array_equal(got, want)
    assert linf <= 1e-5
