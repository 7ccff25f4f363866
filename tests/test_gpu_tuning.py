"""Launch-shape tuning (bfb_set_tuning / bfb_get_tuning / bfb_autotune).

Every launch shape of the three sweeps -- TMA or cp.async tiles, 1/2/4 warps
per CTA, 2/4/8 row groups per TMA tile -- must compute the same numbers: FP64
bit for bit against the oracle (with Dirichlet faces, the fused bulk update
and agents), FP32 bit for bit against the default shape. The autotuner must
leave the field untouched and pick a valid shape.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import face_mask_all

pytestmark = pytest.mark.gpu

SHAPES = [((tma, warps, chunks),) * 3 for tma, warps, chunks in itertools.product((1, 0), (1, 2, 4), (2, 4, 8))]
SHAPES.append(((2, 1, 2),) * 3)  # FP64 x/y: the tensor-memory tiles (elsewhere as TMA tiles)


def _problem(rng, shape=(40, 36, 48), S=2, n_agents=800, dx=20.0, dt=0.01):
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    Sr, Tt, Ur = rng.random((3, *shape, S)) * 4.0
    vals = rng.random((*shape, S)) * 5
    act = np.array([1, 0] * S, np.uint8)[:S]
    L = np.array(shape) * dx
    pos = rng.random((n_agents, 3)) * L
    vol = np.full(n_agents, 4.0 / 3.0 * np.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10, (3, n_agents, S))
    return dict(shape=shape, S=S, D=D, lam=lam, rho0=rho0, bulk=(Sr, Tt, Ur), vals=vals, act=act, pos=pos,
                vol=vol, sec=sec, upt=upt, sat=sat, dx=dx, dt=dt)


def _env(bfb, P, prec, tuning=None):
    env = bfb.Env(P["shape"], P["S"], dx=P["dx"], precision=prec)
    if tuning is not None:
        env.set_tuning(tuning)
    env.set_coefficients(P["D"], P["lam"])
    env.set_field(P["rho0"])
    env.set_dirichlet(P["act"], values=P["vals"])
    env.set_bulk(*P["bulk"])
    env.set_agents(P["pos"], P["vol"], P["sec"], P["upt"], P["sat"], P["dt"])
    return env


STEPS = 3


def _oracle_run(oracle, P):
    dx, dt = P["dx"], P["dt"]
    bbox = (0.0, 0.0, 0.0, *(np.array(P["shape"]) * dx))
    vox = np.maximum(oracle.bin_agents(P["pos"], bbox, dx, P["shape"]), 0)
    t1, t2 = oracle.agent_constants(dt, dx, P["vol"], P["sec"], P["upt"], P["sat"])
    want = P["rho0"]
    for _ in range(STEPS):
        want = oracle.bulk_step(want, dt, *P["bulk"])
        want = oracle.lod_steps(want, dt, dx, P["D"], P["lam"], 1, P["vals"], face_mask_all(P["act"]))
        want = oracle.cells_step(want, vox, t1, t2)
    return want


def test_every_launch_shape_fp64_bitexact_fp32_identical(bfb, oracle):
    rng = np.random.default_rng(4242)
    P = _problem(rng)
    want = _oracle_run(oracle, P)
    flags = bfb.STEP_BULK | bfb.STEP_DIFFUSION | bfb.STEP_CELLS
    ref32 = None
    for shape in SHAPES:
        for prec in (bfb.FP64, bfb.FP32):
            env = _env(bfb, P, prec, shape)
            assert env.get_tuning() == list(shape)
            env.simulate(P["dt"], STEPS, flags)
            got = env.get_field_raw()
            env.close()
            if prec == bfb.FP64:
                assert np.array_equal(got, want), shape
            elif ref32 is None:
                ref32 = got
            else:
                assert np.array_equal(got, ref32), shape


def test_autotune_keeps_field_and_results(bfb, oracle):
    rng = np.random.default_rng(77)
    P = _problem(rng)
    want = _oracle_run(oracle, P)
    env = _env(bfb, P, bfb.FP64)
    before = env.get_field_raw()
    chosen, ms = env.autotune(P["dt"], trials=2)
    assert np.array_equal(env.get_field_raw(), before)  # tuning ran out of place
    assert env.get_tuning() == chosen
    for tma, warps, chunks in chosen:
        assert tma in (0, 1, 2) and 1 <= warps <= 4 and 1 <= chunks <= 16
    assert np.all(ms > 0)
    env.simulate(P["dt"], STEPS, bfb.STEP_BULK | bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    assert np.array_equal(env.get_field(), want)
    env.close()


def test_autotune_large_fp32(bfb):
    """The 256^3 x 8 workload: the tuned shape is at least as fast as the default."""
    rng = np.random.default_rng(5)
    S = 8
    env = bfb.Env((256, 256, 256), S, precision=bfb.FP32)
    env.set_coefficients(log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S))
    t_default = env.profile_steps(0.01, 5)[:3] / 5
    chosen, ms = env.autotune(0.01, trials=3)
    t_tuned = env.profile_steps(0.01, 5)[:3] / 5
    assert chosen != [] and len(chosen) == 3
    assert np.sum(t_tuned) <= 1.10 * np.sum(t_default), (chosen, t_tuned, t_default)
    env.close()


@pytest.mark.parametrize("bad", [
    [(3, 1, 4)] * 3,
    [(1, 0, 4)] * 3,
    [(1, 5, 4)] * 3,
    [(1, 1, 0)] * 3,
    [(1, 1, 17)] * 3,
])
def test_set_tuning_rejects_bad_shapes(bfb, bad):
    env = bfb.Env((8, 8, 8), 1, precision=bfb.FP64)
    with pytest.raises(bfb.BFBError):
        env.set_tuning(bad)
    assert env.get_tuning() == [(1, 1, 2)] * 3
    env.close()


# FP64 x/y sweeps with the lines' forward results in tensor memory: lines of
# 16 to 256 rows, whole and partial 16-row groups and 8-row blocks, head rows
# (factors that vary by row) and Dirichlet faces on either end; bit for bit
# with the oracle, with the fused bulk update and per-face Dirichlet masks
@pytest.mark.parametrize("shape,S", [((256, 10, 6), 3), ((6, 256, 10), 2), ((37, 45, 9), 3), ((250, 17, 4), 1),
                                     ((16, 16, 16), 2), ((100, 100, 8), 4), ((23, 200, 5), 5)])
def test_tensor_memory_tiles_fp64_bitexact(bfb, oracle, shape, S):
    rng = np.random.default_rng(sum(shape) * 31 + S)
    dt, dx = 0.01, 20.0
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    Sr, Tt, Ur = rng.random((3, *shape, S)) * 4.0
    vals = rng.random((*shape, S)) * 30
    act = (rng.random(S) < 0.8).astype(np.uint8)
    fm = (rng.random((6, S)) < 0.6).astype(np.uint8)
    env = bfb.Env(shape, S, dx=dx, precision=bfb.FP64)
    env.set_tuning([(2, 1, 2), (2, 1, 2), (1, 1, 2)])
    env.set_coefficients(D, lam)
    env.set_field(rho0)
    env.set_dirichlet(act, values=vals, face_mask=fm)
    env.set_bulk(Sr, Tt, Ur)
    env.simulate(dt, 3, bfb.STEP_BULK | bfb.STEP_DIFFUSION)
    want = rho0
    for _ in range(3):
        want = oracle.bulk_step(want, dt, Sr, Tt, Ur)
        want = oracle.lod_steps(want, dt, dx, D, lam, 1, vals, fm * act[None, :])
    assert np.array_equal(env.get_field(), want)
    # without the fused bulk update (the plain kernel instantiation)
    env.set_field(rho0)
    env.diffusion_step(dt, 2)
    want = oracle.lod_steps(rho0, dt, dx, D, lam, 2, vals, fm * act[None, :])
    assert np.array_equal(env.get_field(), want)
    env.close()
