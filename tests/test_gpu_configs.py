"""The named workloads at their full sizes.

FP64 is pinned bit-exact to the oracle at reduced sizes (test_gpu_parity.py
and the reduced 200^3-with-agents case here); at full size the FP64 GPU path
is the FP64 reference, and the FP32 path's relative L-inf / L2 error against
it is measured on the device and stated after each workload's step count.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import log_uniform

pytestmark = pytest.mark.gpu
FP32_TOL = 1e-5


def agents_in_ball(rng, n, centre, radius):
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    return np.asarray(centre) + u * (radius * rng.random((n, 1)) ** (1.0 / 3.0))


def agents_xface_inputs(rng, n_vox, n_agents, radius):
    S = 8
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((n_vox, n_vox, n_vox, S))
    L = n_vox * 20.0
    pos = agents_in_ball(rng, n_agents, (L / 2, L / 2, L / 2), radius)
    vol = np.full(n_agents, 4.0 / 3.0 * math.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, n_agents, S))
    fm = np.zeros((6, S), np.uint8)
    fm[0, 0] = fm[1, 0] = 1  # x-faces, substrate 0 only
    act = np.zeros(S, np.uint8)
    act[0] = 1
    vals = np.full(S, 38.0)
    return D, lam, rho0, pos, vol, sec, upt, sat, fm, act, vals


def build_env(bfb, prec, rho0, D, lam, agents, dt, dirichlet):
    nx = rho0.shape[0]
    env = bfb.Env((nx, nx, nx), rho0.shape[-1], dx=20.0, precision=prec)
    env.set_coefficients(D, lam)
    env.set_field(rho0)
    fm, act, vals = dirichlet
    env.set_dirichlet_uniform(act, vals, face_mask=fm)
    pos, vol, sec, upt, sat = agents
    env.set_agents(pos, vol, sec, upt, sat, dt)
    return env


def test_agents_xface_reduced_fp64_bitexact(bfb, oracle):
    """The 200^3 x 8 agents workload's recipe (x-face Dirichlet 38 on substrate 0, agents in a
    central ball, diffusion then cells) on 40^3 x 8 for 20 steps."""
    rng = np.random.default_rng(202)
    D, lam, rho0, pos, vol, sec, upt, sat, fm, act, vals = agents_xface_inputs(rng, 40, 4000, 100.0)
    dt = 0.01
    env = build_env(bfb, bfb.FP64, rho0, D, lam, (pos, vol, sec, upt, sat), dt, (fm, act, vals))
    env.simulate(dt, 20, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    got = env.get_field()
    box = (0.0, 0.0, 0.0, 800.0, 800.0, 800.0)
    vox = oracle.bin_agents(pos, box, 20.0, (40, 40, 40))
    vox = np.where(vox < 0, 0, vox)
    t1, t2 = oracle.agent_constants(dt, 20.0, vol, sec, upt, sat)
    dirv = np.broadcast_to(vals, rho0.shape)
    want = rho0
    for _ in range(20):
        want = oracle.lod_steps(want, dt, 20.0, D, lam, 1, dirv, fm * act[None, :])
        want = oracle.cells_step(want, vox, t1, t2)
    assert np.array_equal(got, want)


def test_agents_200cube_s8_fp32_vs_fp64(bfb):
    """The agents workload: 200^3 x 8, 100k agents in a 500 um ball, 500 steps."""
    rng = np.random.default_rng(2)
    D, lam, rho0, pos, vol, sec, upt, sat, fm, act, vals = agents_xface_inputs(rng, 200, 100_000, 500.0)
    dt = 0.01
    envs = {}
    for prec in (bfb.FP64, bfb.FP32):
        env = build_env(bfb, prec, rho0, D, lam, (pos, vol, sec, upt, sat), dt, (fm, act, vals))
        env.simulate(dt, 500, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
        env.synchronize()
        envs[prec] = env
    linf, l2 = envs[bfb.FP32].compare(envs[bfb.FP64])
    f32, f64 = envs[bfb.FP32].get_field(), envs[bfb.FP64].get_field()
    per = [float(np.abs(f32[..., d] - f64[..., d]).max() / np.abs(f64[..., d]).max()) for d in range(8)]
    print(f"\nagents workload (200^3 x 8, 100k agents, 500 steps): FP32 vs FP64 rel Linf {linf:.3e}, rel L2 {l2:.3e}; "
          f"per substrate rel Linf {['%.1e' % v for v in per]}")
    assert linf <= FP32_TOL


def blobs_field(torch, n, S, seed):
    """Sum of 16 seeded Gaussian blobs (sigma 50-200 um, amplitude 0-10) per
    substrate plus 1e-3 * U[0,1), on a grid of 20 um voxels."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    L = n * 20.0
    x = (torch.arange(n, device="cuda", dtype=torch.float64) + 0.5) * 20.0
    f = 1e-3 * torch.rand((n, n, n, S), generator=g, device="cuda", dtype=torch.float64)
    for d in range(S):
        for _ in range(16):
            c = torch.rand(3, generator=g, device="cuda", dtype=torch.float64) * L
            sig = 50.0 + 150.0 * torch.rand(1, generator=g, device="cuda", dtype=torch.float64)
            amp = 10.0 * torch.rand(1, generator=g, device="cuda", dtype=torch.float64)
            gx = torch.exp(-((x - c[0]) ** 2) / (2 * sig**2))
            gy = torch.exp(-((x - c[1]) ** 2) / (2 * sig**2))
            gz = torch.exp(-((x - c[2]) ** 2) / (2 * sig**2))
            f[..., d] += amp * gx[:, None, None] * gy[None, :, None] * gz[None, None, :]
    return f


def test_blobs_512cube_s4_fp32_vs_fp64_and_mass(bfb):
    """Gaussian blobs: 512^3 x 4 (4.3 GB FP64), D {1e3,1e4,1e5,1e5}, lambda
    {0.01,0.1,1,0.001}, 1000 steps, blobs + noise, no Dirichlet."""
    import torch

    n, S, dt, steps = 512, 4, 0.01, 1000
    D = np.array([1e3, 1e4, 1e5, 1e5])
    lam = np.array([0.01, 0.1, 1.0, 0.001])
    f0 = blobs_field(torch, n, S, 3)
    torch.cuda.synchronize()  # the env copies on its own stream: f0 must be complete first
    envs = {}
    for prec in (bfb.FP64, bfb.FP32):
        env = bfb.Env((n, n, n), S, dx=20.0, precision=prec)
        env.set_coefficients(D, lam)
        env.set_field_device(f0.data_ptr(), bfb.FP64)
        envs[prec] = env
    torch.cuda.synchronize()
    m0 = envs[bfb.FP64].checksum()
    del f0
    torch.cuda.empty_cache()
    for prec in (bfb.FP64, bfb.FP32):
        envs[prec].simulate(dt, steps, bfb.STEP_DIFFUSION)
        envs[prec].synchronize()
    linf, l2 = envs[bfb.FP32].compare(envs[bfb.FP64])
    exact = m0 * (1.0 + dt * lam / 3.0) ** (-3 * steps)  # no Dirichlet: 1^T A = (1 + c2) 1^T per sweep
    drift64 = np.abs(envs[bfb.FP64].checksum() / exact - 1.0)
    drift32 = np.abs(envs[bfb.FP32].checksum() / exact - 1.0)
    print(f"\nGaussian blobs (512^3 x 4, 1000 steps): FP32 vs FP64 rel Linf {linf:.3e}, rel L2 {l2:.3e}; "
          f"mass drift vs exact decay FP64 {['%.1e' % v for v in drift64]}, FP32 {['%.1e' % v for v in drift32]} "
          f"(remaining mass fraction {['%.1e' % v for v in exact / m0]})")
    assert linf <= FP32_TOL
    assert drift64.max() <= 1e-10
    assert drift32.max() <= 1e-4  # relative to each substrate's remaining mass (lambda = 1 keeps 4.5e-5 of it)
