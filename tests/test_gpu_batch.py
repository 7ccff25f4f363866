"""Batched ensembles over many uneven envs, in all three modes: one launch per
stage over every env's tiles (staged), one persistent launch per step, and
the envs' own kernels as branches of one graph."""
from __future__ import annotations

import math
import time

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import face_mask_all

pytestmark = pytest.mark.gpu
MODES = {"persistent": 0, "staged": 1, "graph": 2}  # BFB_BATCH_MODE_*


def make_instance(bfb, rng, edge_lo, edge_hi, n_agents_max, prec, dt):
    shape = tuple(int(v) for v in rng.integers(edge_lo, edge_hi + 1, 3))
    S = int(rng.integers(1, 7))
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    fm = np.zeros((6, S), np.uint8)
    fm[0, 0] = fm[1, 0] = 1  # 38.0 on the x-faces for substrate 0, as the 200^3 agents workload has
    act = np.zeros(S, np.uint8)
    act[0] = 1
    na = int(rng.integers(0, n_agents_max + 1))
    box = np.array(shape) * 20.0
    pos = rng.random((na, 3)) * box
    vol = np.full(na, 4.0 / 3.0 * math.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, na, S))
    spec = dict(shape=shape, S=S, D=D, lam=lam, rho0=rho0, fm=fm, act=act, pos=pos, vol=vol, sec=sec, upt=upt,
                sat=sat, box=(0, 0, 0, *box))
    return spec, build(bfb, spec, prec, dt)


def build(bfb, spec, prec, dt):
    env = bfb.Env(spec["shape"], spec["S"], dx=20.0, precision=prec)
    env.set_coefficients(spec["D"], spec["lam"])
    env.set_field(spec["rho0"])
    env.set_dirichlet_uniform(spec["act"], np.full(spec["S"], 38.0), face_mask=spec["fm"])
    if len(spec["pos"]):
        env.set_agents(spec["pos"], spec["vol"], spec["sec"], spec["upt"], spec["sat"], dt)
    return env


def oracle_run(oracle, spec, dt, steps):
    rho = spec["rho0"]
    vals = np.full_like(rho, 38.0)
    fm = spec["fm"] * spec["act"][None, :]
    if len(spec["pos"]):
        vox = oracle.bin_agents(spec["pos"], spec["box"], 20.0, spec["shape"])
        vox = np.where(vox < 0, 0, vox)
        t1, t2 = oracle.agent_constants(dt, 20.0, spec["vol"], spec["sec"], spec["upt"], spec["sat"])
    for _ in range(steps):
        rho = oracle.lod_steps(rho, dt, 20.0, spec["D"], spec["lam"], 1, vals, fm)
        if len(spec["pos"]):
            rho = oracle.cells_step(rho, vox, t1, t2)
    return rho


@pytest.mark.parametrize("mode", ["staged", "persistent", "graph"])
@pytest.mark.parametrize("warps", [1, 2])
def test_batch_small_fp64_bitexact(bfb, oracle, warps, mode):
    rng = np.random.default_rng(404)
    dt, steps = 0.01, 4
    specs, envs = zip(*[make_instance(bfb, rng, 2, 24, 300, bfb.FP64, dt) for _ in range(12)])
    batch = bfb.Batch(envs)
    batch.set_mode(MODES[mode])
    batch.set_warps(warps)
    batch.simulate(dt, steps, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    batch.synchronize()
    for spec, env in zip(specs, envs):
        assert np.array_equal(env.get_field(), oracle_run(oracle, spec, dt, steps)), spec["shape"]


def make_aligned_instance(bfb, rng, prec, dt, n_agents=400):
    """Shapes whose row pitches suit TMA on every axis (edges multiples of 8,
    S in {2, 4}), so every stage of the persistent kernel runs TMA tiles."""
    shape = tuple(int(v) * 8 for v in rng.integers(2, 7, 3))
    S = int(rng.choice([2, 4]))
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    fm = np.zeros((6, S), np.uint8)
    fm[:, 0] = [1, 1, 0, 1, 1, 0]
    act = np.zeros(S, np.uint8)
    act[0] = 1
    box = np.array(shape) * 20.0
    pos = rng.random((n_agents, 3)) * box
    vol = np.full(n_agents, 4.0 / 3.0 * math.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, n_agents, S))
    spec = dict(shape=shape, S=S, D=D, lam=lam, rho0=rho0, fm=fm, act=act, pos=pos, vol=vol, sec=sec, upt=upt,
                sat=sat, box=(0, 0, 0, *box))
    return spec, build(bfb, spec, prec, dt)


@pytest.mark.parametrize("mode,warps,tiles", [("persistent", 1, 1), ("persistent", 2, 3), ("persistent", 4, 8),
                                              ("persistent", 1, 64), ("staged", 1, 2), ("staged", 4, 2),
                                              ("graph", 1, 2)])
def test_batch_tma_items_fp64_bitexact(bfb, oracle, mode, warps, tiles):
    rng = np.random.default_rng(900 + warps * 10 + tiles)
    dt, steps = 0.01, 3
    specs, envs = zip(*[make_aligned_instance(bfb, rng, bfb.FP64, dt) for _ in range(6)])
    batch = bfb.Batch(envs)
    batch.set_mode(MODES[mode])
    assert batch.mode == MODES[mode]
    batch.set_warps(warps)
    batch.set_tiles_per_item(tiles)
    batch.simulate(dt, steps, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    batch.synchronize()
    for spec, env in zip(specs, envs):
        assert np.array_equal(env.get_field(), oracle_run(oracle, spec, dt, steps)), spec["shape"]


@pytest.mark.parametrize("mode", ["staged", "persistent", "graph"])
def test_batch_wide_substrates_fp64_bitexact(bfb, oracle, mode):
    """Envs with more than 32 substrates (a lane solves several z lines) next
    to ordinary ones in one batch."""
    rng = np.random.default_rng(77)
    dt, steps = 0.01, 3
    specs, envs = [], []
    for shape, S in (((6, 5, 7), 40), ((9, 4, 6), 33), ((8, 8, 8), 3)):
        D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
        fm = np.zeros((6, S), np.uint8)
        fm[0, 0] = fm[1, 0] = 1
        act = np.zeros(S, np.uint8)
        act[0] = 1
        spec = dict(shape=shape, S=S, D=D, lam=lam, rho0=rng.random((*shape, S)), fm=fm, act=act,
                    pos=np.zeros((0, 3)), vol=np.zeros(0), sec=None, upt=None, sat=None, box=None)
        specs.append(spec)
        envs.append(build(bfb, spec, bfb.FP64, dt))
    batch = bfb.Batch(envs)
    batch.set_mode(MODES[mode])
    batch.simulate(dt, steps, bfb.STEP_DIFFUSION)
    batch.synchronize()
    for spec, env in zip(specs, envs):
        assert np.array_equal(env.get_field(), oracle_run(oracle, spec, dt, steps)), (spec["shape"], spec["S"])


def test_batch_autotune_restores_fields(bfb, oracle):
    rng = np.random.default_rng(31)
    dt, steps = 0.01, 2
    specs, envs = zip(*[make_aligned_instance(bfb, rng, bfb.FP64, dt) for _ in range(5)])
    batch = bfb.Batch(envs)
    before = [e.get_field_raw() for e in envs]
    (w, t), ms = batch.autotune(dt, bfb.STEP_DIFFUSION | bfb.STEP_CELLS, trials=1)
    assert w in (1, 2, 4) and t in (1, 2, 4, 8) and ms > 0
    assert batch.mode in (bfb.BATCH_MODE_STAGED, bfb.BATCH_MODE_PERSISTENT, bfb.BATCH_MODE_GRAPH)
    for e, b0 in zip(envs, before):
        assert np.array_equal(e.get_field_raw(), b0)
    batch.simulate(dt, steps, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    batch.synchronize()
    for spec, env in zip(specs, envs):
        assert np.array_equal(env.get_field(), oracle_run(oracle, spec, dt, steps))


@pytest.mark.parametrize("mode", ["staged", "persistent", "graph"])
def test_batch_fp32_equals_per_instance_loop(bfb, mode):
    rng = np.random.default_rng(405)
    dt, steps = 0.01, 5
    made = [make_instance(bfb, rng, 3, 40, 800, bfb.FP32, dt) for _ in range(10)]
    specs = [m[0] for m in made]
    envs_b = [m[1] for m in made]
    envs_l = [build(bfb, sp, bfb.FP32, dt) for sp in specs]
    b = bfb.Batch(envs_b)
    b.set_mode(MODES[mode])
    b.simulate(dt, steps, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    b.synchronize()
    lp = bfb.Batch(envs_l)
    lp.simulate_loop(dt, steps, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    for eb, el in zip(envs_b, envs_l):
        assert np.array_equal(eb.get_field_raw(), el.get_field_raw())


def test_ensemble_256_batch_vs_loop_and_fp64_check(bfb):
    """Uneven ensemble: 256 envs, edges U{32..160} per axis, 1-6 substrates, 0-20k
    agents each, 200 steps in FP32; FP64 check on 8 sampled envs; the batch
    (staged launches, and one persistent launch per step) against the
    per-instance launch loop."""
    rng = np.random.default_rng(4)
    dt, steps = 0.01, 200
    made = [make_instance(bfb, rng, 32, 160, 20_000, bfb.FP32, dt) for _ in range(256)]
    specs = [m[0] for m in made]
    envs = [m[1] for m in made]
    vs = sum(int(np.prod(sp["shape"])) * sp["S"] for sp in specs)
    flags = bfb.STEP_DIFFUSION | bfb.STEP_CELLS
    batch = bfb.Batch(envs)

    def timed(n):
        batch.simulate(dt, 2, flags)  # warm-up (graph capture)
        batch.synchronize()
        t0 = time.perf_counter()
        batch.simulate(dt, n, flags)
        batch.synchronize()
        return (time.perf_counter() - t0) / n

    batch.set_mode(bfb.BATCH_MODE_PERSISTENT)
    batch.set_warps(1)
    batch.set_tiles_per_item(4)
    t_pers = timed(20)
    batch.set_mode(bfb.BATCH_MODE_STAGED)
    t_staged = timed(20)
    batch.set_mode(bfb.BATCH_MODE_GRAPH)
    t_graph = timed(20)
    tuned, _ = batch.autotune(dt, flags, trials=2)  # mode, warps per CTA and tiles per item
    mode = {v: k for k, v in MODES.items()}[batch.mode]
    t_batch = timed(steps - 66)  # 202 steps in all (4 x 2 warm + 3 x 20 + 134), as the FP64 check below
    # per-instance launch loop over fresh copies of the same envs
    loop_envs = [build(bfb, sp, bfb.FP32, dt) for sp in specs]
    loop = bfb.Batch(loop_envs)
    loop.simulate_loop(dt, 2, flags)
    t0 = time.perf_counter()
    loop.simulate_loop(dt, steps, flags)
    t_loop = (time.perf_counter() - t0) / steps
    # FP64 check on 8 sampled envs (same 202 steps)
    pick = rng.choice(len(specs), 8, replace=False)
    errs = []
    for q in pick:
        e64 = build(bfb, specs[q], bfb.FP64, dt)
        e64.simulate(dt, steps + 2, flags)
        e64.synchronize()
        errs.append(envs[q].compare(e64)[0])
        e64.close()
    print(f"\nuneven ensemble (256 envs, {vs / 1e6:.0f} M voxel*substrates, 200 steps): batch, autotuned "
          f"({mode}, warps, tiles per item = {tuned}) {t_batch * 1e3:.3f} ms/step ({vs / t_batch:.3e} vox*sub/s); "
          f"staged (1 warp) {t_staged * 1e3:.3f}, persistent (1 warp, 4 tiles) {t_pers * 1e3:.3f}, "
          f"graph {t_graph * 1e3:.3f}; "
          f"per-instance loop {t_loop * 1e3:.3f} ms/step ({vs / t_loop:.3e}); "
          f"FP32 vs FP64 rel Linf on 8 envs: max {max(errs):.2e}")
    assert max(errs) <= 1e-5
