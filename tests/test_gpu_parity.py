"""GPU parity tests: the CUDA path through the C ABI against the oracle.

FP64 is compared BIT FOR BIT with the oracle restatement (which is itself
bit-exact with the reference build, see test_oracle.py) and with the golden
fixtures the reference produced. The contract is <= 1e-12 relative L-inf per
step; exact equality is what the kernels deliver and what is asserted.
FP32 is compared with a stated relative L-inf tolerance.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import face_mask_all

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
FP32_TOL = 1e-5  # relative L-inf of the FP32 path vs the FP64 oracle


def golden(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make_env(bfb, rho, D, lam, prec, dx=20.0, tma=1):
    nx, ny, nz, S = rho.shape
    env = bfb.Env((nx, ny, nz), S, dx=dx, precision=prec)
    env.set_option(bfb.OPT_USE_TMA, tma)
    env.set_coefficients(D, lam)
    env.set_field(rho)
    return env


# ---------------------------------------------------------------------------
# golden fixtures made by the reference
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("via", ["diffusion_step", "simulate"])
def test_lod_15cube_golden(bfb, via):
    g = golden("lod_15cube_s1_dirichlet")
    env = make_env(bfb, g["rho0"], g["D"], g["lam"], bfb.FP64, float(g["dx"]))
    env.set_dirichlet_uniform([1], g["dir_value"])
    steps, dt = int(g["steps"]), float(g["dt"])
    if via == "simulate":
        env.simulate(dt, steps, bfb.STEP_DIFFUSION)
    else:
        env.diffusion_step(dt, steps)
    assert np.array_equal(env.get_field(), g["out"])


@pytest.mark.parametrize("name", ["multi_7x5x9_S3", "multi_1x4x6_S2", "multi_2x3x1_S2", "multi_17x3x33_S5"])
def test_multi_golden(bfb, name):
    g = golden(name)
    env = make_env(bfb, g["rho0"], g["D"], g["lam"], bfb.FP64, float(g["dx"]))
    env.set_dirichlet(g["activation"], values=g["dir_values"])
    env.diffusion_step(float(g["dt"]), int(g["steps"]))
    assert np.array_equal(env.get_field(), g["out"])


@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
def test_bulk_golden_standalone_and_fused(bfb, tma):
    g = golden("bulk_9x8x7_S3")
    dt = float(g["dt"])
    for fused in (False, True):
        env = make_env(bfb, g["rho0"], g["D"], g["lam"], bfb.FP64, float(g["dx"]), tma=tma)
        env.set_bulk(g["S_rate"], g["T_target"], g["U_rate"])
        if fused:
            env.simulate(dt, 3, bfb.STEP_BULK | bfb.STEP_DIFFUSION)
        else:
            for _ in range(3):
                env.bulk_step(dt)
                env.diffusion_step(dt, 1)
        assert np.array_equal(env.get_field(), g["out"]), f"fused={fused}"


@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
def test_bulk_fused_aligned_grid(bfb, oracle, rng, tma):
    """Bulk fused into the x-sweep load on a grid whose rows suit TMA."""
    shape, S = (16, 12, 8), 4
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    Sr, Tt, Ur = rng.random((3, *shape, S)) * 4.0
    vals = rng.random((*shape, S)) * 5
    act = np.array([1, 0, 1, 1], np.uint8)
    env = make_env(bfb, rho0, D, lam, bfb.FP64, tma=tma)
    env.set_dirichlet(act, values=vals)
    env.set_bulk(Sr, Tt, Ur)
    env.simulate(0.01, 3, bfb.STEP_BULK | bfb.STEP_DIFFUSION)
    want = rho0
    for _ in range(3):
        want = oracle.bulk_step(want, 0.01, Sr, Tt, Ur)
        want = oracle.lod_steps(want, 0.01, 20.0, D, lam, 1, vals, face_mask_all(act))
    assert np.array_equal(env.get_field(), want)


def test_agents_golden(bfb):
    g = golden("agents_12x10x9_S2")
    dt = float(g["dt"])
    env = make_env(bfb, g["rho0"], g["D"], g["lam"], bfb.FP64, float(g["dx"]))
    env.set_agents(g["pos"], g["vol"], g["sec"], g["upt"], g["sat"], dt)
    assert np.array_equal(env.agent_voxels(), g["voxels"])
    for _ in range(3):
        env.diffusion_step(dt, 1)
        env.cells_step(dt)
    assert np.array_equal(env.get_field(), g["out"])
    env2 = make_env(bfb, g["rho0"], g["D"], g["lam"], bfb.FP64, float(g["dx"]))
    env2.set_agents(g["pos"], g["vol"], g["sec"], g["upt"], g["sat"], dt)
    env2.simulate(dt, 3, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
    assert np.array_equal(env2.get_field(), g["out"])


# ---------------------------------------------------------------------------
# against the oracle restatement
# ---------------------------------------------------------------------------
def test_cube75_s1_full_size_fp64(bfb, oracle):
    """The 75^3 single-substrate workload exactly: 75^3 x 1, D=1e5, lambda=0.1, dt=0.01, 100 steps,
    Dirichlet 1.0 on all faces, U[0,1) field from a seed."""
    rng = np.random.default_rng(2024)
    rho0 = rng.random((75, 75, 75, 1))
    env = make_env(bfb, rho0, [1e5], [0.1], bfb.FP64)
    env.set_dirichlet_uniform([1], [1.0])
    env.simulate(0.01, 100, bfb.STEP_DIFFUSION)
    got = env.get_field()
    want = oracle.lod_steps(rho0, 0.01, 20.0, [1e5], [0.1], 100, np.ones_like(rho0), face_mask_all([1]))
    assert rel_linf(got, want) <= 1e-12
    assert np.array_equal(got, want)


SHAPES = [((1, 1, 1), 1), ((1, 4, 6), 2), ((2, 3, 1), 3), ((3, 2, 2), 1), ((5, 17, 3), 4), ((17, 5, 2), 6),
          ((8, 8, 8), 4), ((8, 8, 8), 8), ((7, 5, 9), 3), ((33, 31, 35), 5), ((64, 2, 3), 2), ((2, 64, 40), 1),
          ((40, 3, 64), 7), ((6, 5, 7), 40), ((3, 9, 4), 33),  # S > 32: lanes solve several z lines each
          ((100, 6, 8), 3), ((5, 130, 4), 2), ((97, 96, 4), 1),  # lines of about 100 rows
          ((256, 10, 6), 3), ((6, 256, 10), 2)]  # 256-row lines: FP64 tiles narrower than a warp


@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
@pytest.mark.parametrize("shape,S", SHAPES)
def test_random_shapes_fp64_bitexact(bfb, oracle, rng, shape, S, tma):
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    vals = rng.random((*shape, S)) * 30
    act = (rng.random(S) < 0.7).astype(np.uint8)
    fm = (rng.random((6, S)) < 0.6).astype(np.uint8)  # per-face mask (extension)
    env = make_env(bfb, rho0, D, lam, bfb.FP64, tma=tma)
    env.set_dirichlet(act, values=vals, face_mask=fm)
    env.diffusion_step(0.01, 3)
    want = oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 3, vals, fm * act[None, :])
    assert np.array_equal(env.get_field(), want)


@pytest.mark.parametrize("tma", [1, 0], ids=["tma", "cpasync"])
@pytest.mark.parametrize("shape,S", SHAPES)
def test_random_shapes_fp32(bfb, oracle, rng, shape, S, tma):
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    vals = rng.random((*shape, S)) * 30
    act = (rng.random(S) < 0.7).astype(np.uint8)
    env = make_env(bfb, rho0, D, lam, bfb.FP32, tma=tma)
    env.set_dirichlet(act, values=vals)
    env.diffusion_step(0.01, 5)
    want = oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 5, vals, face_mask_all(act))
    assert rel_linf(env.get_field(), want) <= FP32_TOL


@pytest.mark.parametrize("shape,S,prec", [((900, 3, 4), 2, 0), ((3, 2, 4000), 1, 0), ((1200, 2, 2), 1, 1),
                                          ((2, 3, 9000), 1, 1)])
def test_long_lines_use_fallback_kernels(bfb, oracle, rng, shape, S, prec):
    """Lines longer than shared memory holds run the two-pass fallback."""
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    env = make_env(bfb, rho0, D, lam, prec)
    env.set_dirichlet_uniform(np.ones(S), np.full(S, 2.0))
    env.diffusion_step(0.01, 2)
    want = oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 2, np.full_like(rho0, 2.0), face_mask_all(np.ones(S)))
    got = env.get_field()
    if prec == 0:
        assert np.array_equal(got, want)
    else:
        assert rel_linf(got, want) <= FP32_TOL


def test_factors_without_a_constant_tail(bfb, oracle, rng):
    """With a huge D (c1 = 2500) the Thomas factors still vary at the end of a
    96-row line, so no row uses the register copies of the tail factors; the
    head-table path alone must reproduce the reference."""
    shape, S = (96, 4, 4), 1
    D, lam = np.array([1e8]), np.array([0.1])
    rho0 = rng.random((*shape, S))
    env = make_env(bfb, rho0, D, lam, bfb.FP64)
    env.diffusion_step(0.01, 2)
    assert np.array_equal(env.get_field(), oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 2))


def test_agents_random_fp64_and_fp32(bfb, oracle, rng):
    shape, S = (20, 18, 16), 3
    dx, dt = 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S))
    n = 5000
    pos = rng.uniform(-10.0, 330.0, (n, 3))
    vol = np.full(n, 4.0 / 3.0 * np.pi * 125.0)
    sec, upt, sat = log_uniform(rng, 1e-2, 10, (3, n, S))
    active = (rng.random(n) < 0.9).astype(np.uint8)
    bbox = (0.0, 0.0, 0.0, shape[0] * dx, shape[1] * dx, shape[2] * dx)
    vox = oracle.bin_agents(pos, bbox, dx, shape)
    vox = np.where(vox < 0, 0, vox)
    t1, t2 = oracle.agent_constants(dt, dx, vol, sec, upt, sat)
    want = rho0
    for _ in range(4):
        want = oracle.lod_steps(want, dt, dx, D, lam, 1)
        want = oracle.cells_step(want, vox, t1, t2, active)
    for prec in (bfb.FP64, bfb.FP32):
        env = make_env(bfb, rho0, D, lam, prec, dx)
        env.set_agents(pos, vol, sec, upt, sat, dt, active=active)
        assert np.array_equal(env.agent_voxels(), vox)
        env.simulate(dt, 4, bfb.STEP_DIFFUSION | bfb.STEP_CELLS)
        got = env.get_field()
        if prec == bfb.FP64:
            assert np.array_equal(got, want)
        else:
            assert rel_linf(got, want) <= FP32_TOL


@pytest.mark.parametrize("shape,S", [((30, 20, 25), 3), ((7, 5, 3), 64), ((2, 3, 1), 1), ((40, 3, 64), 7),
                                     ((5, 4, 3), 33), ((64, 64, 64), 8)])
def test_checksum_matches_oracle(bfb, oracle, rng, shape, S):
    """One pass of per-substrate FP64 sums, against the oracle's voxel-order sum
    (fewer voxels than reduction blocks included)."""
    rho = rng.random((*shape, S))
    for prec in (bfb.FP64, bfb.FP32):
        env = make_env(bfb, rho, [1e3] * S, [0.1] * S, prec)
        want = oracle.checksum(rho if prec == bfb.FP64 else rho.astype(np.float32).astype(np.float64))
        got = env.checksum()
        assert np.allclose(got, want, rtol=1e-12, atol=0)
        env.close()


@pytest.mark.parametrize("shape,S", [((6, 5, 7), 3), ((4, 3, 9), 1), ((5, 4, 8), 2), ((3, 3, 5), 5)])
def test_field_rows_padded_to_16_bytes(bfb, rng, shape, S):
    """The device field's (i, j) rows are nz*S elements apart when that is a
    whole number of 16-byte vectors, else padded to the next one; the
    transfer calls still take and return the packed layout, bit for bit."""
    rho = rng.random((*shape, S))
    L = shape[2] * S
    for prec, eb in ((bfb.FP64, 8), (bfb.FP32, 4)):
        env = make_env(bfb, rho, [1e3] * S, [0.1] * S, prec)
        epv = 16 // eb
        assert env.field_pitch() == (L + epv - 1) // epv * epv
        want = rho if prec == bfb.FP64 else rho.astype(np.float32)
        assert np.array_equal(env.get_field_raw(), want)
        env.close()


def test_checksum_256cube_bandwidth(bfb):
    """The per-substrate mass checksum at the bench size reads the field once;
    timed with CUDA events on one stream (through the allocation-free entry
    point, which queues the same kernels without waiting) and reported."""
    import ctypes

    import torch

    S, n = 8, 256 ** 3
    L = bfb.load_library()
    out = torch.zeros(S, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    for prec, eb in ((bfb.FP32, 4), (bfb.FP64, 8)):
        env = bfb.Env((256, 256, 256), S, precision=prec)
        torch.cuda.synchronize()

        def call():
            rc = L.bfb_checksum_noalloc(ctypes.c_void_p(env.field_device_ptr()), prec, n, S,
                                        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, L.bfb_last_error()

        for _ in range(3):
            call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(10):
            call()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 10
        print(f"\nchecksum 256^3 x 8 {'FP32' if eb == 4 else 'FP64'}: {ms:.3f} ms per call, "
              f"{n * S * eb / (ms / 1e3) / 1e9:.0f} GB/s (one read of the field)")
        assert ms > 0
        env.close()


def test_graph_replay_equals_direct_launches(bfb, rng):
    rho0 = rng.random((24, 20, 16, 4))
    D, lam = log_uniform(rng, 1e2, 1e5, 4), log_uniform(rng, 1e-3, 1.0, 4)
    outs = []
    for graphs in (0, 1):
        env = make_env(bfb, rho0, D, lam, bfb.FP32)
        env.set_option(bfb.OPT_USE_GRAPHS, graphs)
        env.set_dirichlet_uniform([1, 0, 1, 0], [3.0, 0, 1.0, 0])
        env.simulate(0.01, 7, bfb.STEP_DIFFUSION)
        outs.append(env.get_field_raw())
    assert np.array_equal(outs[0], outs[1])


def test_step_host_equals_device_path(bfb, rng):
    import torch

    rho0 = rng.random((16, 12, 10, 2))
    D, lam = [1e4, 3e2], [0.1, 0.01]
    env = make_env(bfb, rho0, D, lam, bfb.FP64)
    env.diffusion_step(0.01, 2)
    want = env.get_field()
    env2 = bfb.Env((16, 12, 10), 2, precision=bfb.FP64)
    env2.set_coefficients(D, lam)
    host = torch.from_numpy(rho0.copy()).pin_memory()
    env2.step_host_ptr(host.data_ptr(), 0.01, 2)
    assert np.array_equal(host.numpy(), want)


def test_factors_frozen_at_first_dt_like_the_reference(bfb, oracle, rng):
    """BioFVM_parallel.cpp:714,913: factors from the first call's dt are kept."""
    rho0 = rng.random((6, 5, 4, 2))
    D, lam = [1e4, 1e3], [0.5, 0.05]
    env = make_env(bfb, rho0, D, lam, bfb.FP64)
    env.diffusion_step(0.01, 1)
    env.diffusion_step(0.02, 1)  # ignored dt change
    want = oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 2)
    assert np.array_equal(env.get_field(), want)
    env2 = make_env(bfb, rho0, D, lam, bfb.FP64)
    env2.set_option(bfb.OPT_FREEZE_FACTORS, 0)
    env2.diffusion_step(0.01, 1)
    env2.diffusion_step(0.02, 1)
    want2 = oracle.lod_steps(oracle.lod_steps(rho0, 0.01, 20.0, D, lam, 1), 0.02, 20.0, D, lam, 1)
    assert np.array_equal(env2.get_field(), want2)


def test_apply_dirichlet_matches_oracle(bfb, oracle, rng):
    rho0 = rng.random((7, 6, 5, 3))
    vals = rng.random((7, 6, 5, 3))
    act = np.array([1, 0, 1], np.uint8)
    env = make_env(bfb, rho0, [1.0] * 3, [0.0] * 3, bfb.FP64)
    env.set_dirichlet(act, values=vals)
    env.apply_dirichlet()
    assert np.array_equal(env.get_field(), oracle.dirichlet(rho0, vals, face_mask_all(act)))


def test_invalid_arguments_return_errors(bfb):
    with pytest.raises(bfb.BFBError) as e:
        bfb.Env((0, 4, 4), 1)
    assert e.value.code == -2
    env = bfb.Env((4, 4, 4), 1)
    with pytest.raises(bfb.BFBError):
        env.diffusion_step(-1.0, 1)
    with pytest.raises(bfb.BFBError):
        env.simulate(0.01, 1, 64)
    with pytest.raises(bfb.BFBError):
        env.set_option(99, 1)


# ---------------------------------------------------------------------------
# full-size properties (256^3 x 8, the benchmark workload)
# ---------------------------------------------------------------------------
def test_mass_balance_full_size(bfb, rng):
    """Without Dirichlet, 1^T A = (1 + c2) 1^T for every axis, so each LOD step
    scales the per-substrate mass by exactly (1 + dt*lambda/3)^-3."""
    S = 8
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((256, 256, 256, S), dtype=np.float32).astype(np.float64)
    for prec, tol in ((bfb.FP64, 1e-11), (bfb.FP32, 2e-6)):
        env = make_env(bfb, rho0, D, lam, prec)
        m0 = env.checksum()
        env.simulate(0.01, 10, bfb.STEP_DIFFUSION)
        m1 = env.checksum()
        c2 = 0.01 * lam / 3.0
        assert np.allclose(m1, m0 * (1 + c2) ** -30, rtol=tol, atol=0), (prec, m1 / m0, (1 + c2) ** -30)
        env.close()


def test_fp32_vs_fp64_full_size_1000_steps(bfb, rng):
    """The FP32 precision target: FP32 within 1e-5 relative L-inf of
    the FP64 path (itself bit-exact with the reference) after 1000 steps at
    256^3 x 8 (D, lambda log-uniform as in the 200^3 x 8 agents workload, U[0,1) field)."""
    S = 8
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((256, 256, 256, S))
    e64 = make_env(bfb, rho0, D, lam, bfb.FP64)
    e64.simulate(0.01, 1000, bfb.STEP_DIFFUSION)
    f64 = e64.get_field()
    e64.close()
    e32 = make_env(bfb, rho0, D, lam, bfb.FP32)
    e32.simulate(0.01, 1000, bfb.STEP_DIFFUSION)
    f32 = e32.get_field()
    e32.close()
    err = rel_linf(f32, f64)
    print(f"FP32 vs FP64 after 1000 steps at 256^3x8: rel Linf {err:.3e}, "
          f"rel L2 {np.linalg.norm(f32 - f64) / np.linalg.norm(f64):.3e}")
    assert err <= FP32_TOL
