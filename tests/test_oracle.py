"""CPU tests: the oracle restatement is pinned to the reference.

* against the committed golden fixtures (made by the reference library), bit-exact;
* against the live reference library when it is built here (oracle/_ref), bit-exact;
* the adjoint restatement against central finite differences.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import REF_SO, RefEnv, RefLib, face_mask_all

GOLD = Path(__file__).resolve().parent / "golden"


def golden(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def test_lod_15cube_golden_bitexact(oracle):
    g = golden("lod_15cube_s1_dirichlet")
    S = 1
    vals = np.broadcast_to(np.asarray(g["dir_value"], float), g["rho0"].shape)
    out = oracle.lod_steps(g["rho0"], float(g["dt"]), float(g["dx"]), g["D"], g["lam"], int(g["steps"]),
                           vals, face_mask_all(g["activation"]))
    assert np.array_equal(out, g["out"])
    # the reference's AVX2 solver gives the same bits (both fuse the axpy)
    assert np.array_equal(g["out_avx"], g["out"])
    assert S == g["rho0"].shape[-1]


@pytest.mark.parametrize("name", ["multi_7x5x9_S3", "multi_1x4x6_S2", "multi_2x3x1_S2", "multi_17x3x33_S5"])
def test_multi_golden_bitexact(oracle, name):
    g = golden(name)
    out = oracle.lod_steps(g["rho0"], float(g["dt"]), float(g["dx"]), g["D"], g["lam"], int(g["steps"]),
                           g["dir_values"], face_mask_all(g["activation"]))
    assert np.array_equal(out, g["out"])


def test_bulk_golden_bitexact(oracle):
    g = golden("bulk_9x8x7_S3")
    rho = g["rho0"]
    S = rho.shape[-1]
    for _ in range(3):
        rho = oracle.bulk_step(rho, float(g["dt"]), g["S_rate"], g["T_target"], g["U_rate"])
        rho = oracle.lod_steps(rho, float(g["dt"]), float(g["dx"]), g["D"], g["lam"], 1, None,
                               np.zeros((6, S), np.uint8))
    assert np.array_equal(rho, g["out"])


def test_agents_golden_bitexact(oracle):
    g = golden("agents_12x10x9_S2")
    rho = g["rho0"]
    S = rho.shape[-1]
    dt, dx = float(g["dt"]), float(g["dx"])
    vox = oracle.bin_agents(g["pos"], g["bbox"], dx, rho.shape[:3])
    # rejected positions keep a new agent's voxel 0
    assert np.array_equal(np.where(vox < 0, 0, vox), g["voxels"])
    assert (vox < 0).sum() == 2
    t1, t2 = oracle.agent_constants(dt, dx, g["vol"], g["sec"], g["upt"], g["sat"])
    for _ in range(3):
        rho = oracle.lod_steps(rho, dt, dx, g["D"], g["lam"], 1, None, np.zeros((6, S), np.uint8))
        rho = oracle.cells_step(rho, np.where(vox < 0, 0, vox), t1, t2)
    assert np.array_equal(rho, g["out"])


needs_ref = pytest.mark.skipif(not REF_SO.exists(), reason="reference library not built here")


@needs_ref
@pytest.mark.parametrize("shape,S", [((5, 6, 7), 4), ((3, 1, 2), 1), ((11, 4, 2), 6), ((2, 2, 2), 3)])
def test_live_reference_bitexact(oracle, rng, shape, S):
    ref = RefLib()
    dx, dt = 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    e = RefEnv(ref, (0, 0, 0, *(np.array(shape) * dx)), dx, D, lam)
    rho0 = rng.random(e.shape)
    act = (rng.random(S) < 0.5).astype(np.uint8)
    vals = rng.random(e.shape) * 10
    e.set_field(rho0)
    e.set_dirichlet(act, face_values=vals)
    e.step(dt, 3)
    out = oracle.lod_steps(rho0, dt, dx, D, lam, 3, vals, face_mask_all(act))
    assert np.array_equal(out, e.field())


@needs_ref
def test_golden_fixtures_reproduce_from_the_reference():
    """The committed fixtures are what the reference library computes today:
    tests/golden/make_golden.py's cases, rerun, give the same arrays."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLD / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    cases = mg.make_cases(RefLib())
    assert sorted(cases) == sorted(p.stem for p in GOLD.glob("*.npz"))
    for name, data in cases.items():
        g = golden(name)
        assert sorted(g) == sorted(data), name
        for k, v in data.items():
            assert np.array_equal(np.asarray(v), g[k]), (name, k)


@needs_ref
def test_live_reference_default_dirichlet_is_100(oracle):
    """dirichlet_test's 'should be 100' (examples/dirichlet_test.cpp:277): after
    resize the reference's Dirichlet value is 100.0 with activation true."""
    ref = RefLib()
    e = RefEnv(ref, (0, 0, 0, 100, 100, 100), 20.0, [1e3], [0.1])
    e.set_field(np.zeros(e.shape))
    e.apply_dirichlet()
    f = e.field()
    assert f[0, 0, 0, 0] == 100.0 and f[2, 2, 2, 0] == 0.0


@needs_ref
def test_live_reference_non_multiple_domain_binning(oracle, rng):
    """Domain length not a multiple of dx: the node count uses ceil while the
    binning extents truncate (BioFVM_parallel.cpp:100-102 vs 440-446)."""
    ref = RefLib()
    dx = 20.0
    box = (0.0, 0.0, 0.0, 105.0, 93.0, 71.0)
    e = RefEnv(ref, box, dx, [1e3, 1e4], [0.1, 0.2])
    pos = rng.uniform(-5, 110, (500, 3))
    vol = np.ones(500)
    z = np.zeros((500, 2))
    e.add_agents(pos, vol, z, z, z, 0.01)
    ov = oracle.bin_agents(pos, box, dx, e.shape[:3])
    assert np.array_equal(np.where(ov < 0, 0, ov), e.agent_voxels())


@needs_ref
@pytest.mark.parametrize("solver", [0, 1], ids=["LOD_3D", "LOD_3D_AVX256D"])
@pytest.mark.parametrize("shape,S", [((6, 5, 7), 3), ((4, 9, 3), 5), ((7, 4, 6), 8), ((3, 3, 12), 1)])
def test_live_reference_both_solvers_bitexact(oracle, rng, solver, shape, S):
    """Both reference solvers (BioFVM_parallel.cpp:693-1395 and its AVX2 form
    :1411-2326, whose factor tables are replicated to lcm(S, 4) entries) give
    the oracle's bits, for S below, above and at a multiple of 4, with
    per-voxel Dirichlet values on a random subset of substrates."""
    ref = RefLib()
    dx, dt = 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    e = RefEnv(ref, (0, 0, 0, *(np.array(shape) * dx)), dx, D, lam)
    e.set_solver(solver)
    rho0 = rng.random(e.shape) * 5
    act = (rng.random(S) < 0.5).astype(np.uint8)
    vals = rng.random(e.shape) * 10
    e.set_field(rho0)
    e.set_dirichlet(act, face_values=vals)
    e.step(dt, 4)
    out = oracle.lod_steps(rho0, dt, dx, D, lam, 4, vals, face_mask_all(act))
    assert np.array_equal(out, e.field())


@needs_ref
def test_live_reference_bulk_diffusion_agents_bitexact(oracle, rng):
    """A step order of the reference's drivers (examples/3D_tumor_example_X.cpp
    346-348: bulk sources and sinks, diffusion, then the agents), on random
    rates with many agents per voxel, so the list-ordered per-voxel update
    (BioFVM_basic_agent.cpp:279-300) is exercised; bit-exact for 3 steps."""
    ref = RefLib()
    shape, S, dx, dt = (8, 7, 6), 3, 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    box = (0.0, 0.0, 0.0, *(np.array(shape) * dx))
    e = RefEnv(ref, box, dx, D, lam)
    rho0 = rng.random(e.shape) * 4
    e.set_field(rho0)
    e.set_dirichlet([0] * S)
    S_rate, T_target, U_rate = (log_uniform(rng, 1e-2, 10.0, e.shape) for _ in range(3))
    e.set_bulk(S_rate, T_target, U_rate)
    n = 400  # in a 60 um cube: 27 voxels, ~15 agents per voxel
    pos = rng.uniform(40.0, 100.0, (n, 3))
    vol = log_uniform(rng, 1e2, 1e3, n)
    sec, upt, sat = (log_uniform(rng, 1e-2, 10.0, (n, S)) for _ in range(3))
    e.add_agents(pos, vol, sec, upt, sat, dt)
    vox = oracle.bin_agents(pos, box, dx, shape)
    assert (vox >= 0).all() and np.array_equal(vox, e.agent_voxels())
    assert np.bincount(vox).max() >= 10
    t1, t2 = oracle.agent_constants(dt, dx, vol, sec, upt, sat)
    rho = rho0
    for _ in range(3):
        e.bulk_step(dt)
        e.step(dt, 1)
        e.cells_step(dt)
        rho = oracle.bulk_step(rho, dt, S_rate, T_target, U_rate)
        rho = oracle.lod_steps(rho, dt, dx, D, lam, 1, None, np.zeros((6, S), np.uint8))
        rho = oracle.cells_step(rho, vox, t1, t2)
    assert np.array_equal(rho, e.field())


def test_adjoint_oracle_matches_finite_differences(oracle, rng):
    shape, S = (4, 3, 5), 2
    dx, dt = 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-2, 1.0, S)
    rho = rng.random((*shape, S))
    vals = rng.random((*shape, S))
    fm = np.zeros((6, S), np.uint8)
    fm[0, 0] = fm[1, 0] = 1
    w = rng.random((*shape, S))

    def loss(r, Dv, lv):
        return float((oracle.lod_steps(r, dt, dx, Dv, lv, 1, vals, fm) * w).sum())

    g_rho, gD, gL = oracle.lod_step_adjoint(rho, w, dt, dx, D, lam, vals, fm)
    for q in range(S):
        h = D[q] * 1e-6
        Dp, Dm = D.copy(), D.copy()
        Dp[q] += h
        Dm[q] -= h
        fd = (loss(rho, Dp, lam) - loss(rho, Dm, lam)) / (2 * h)
        assert abs(fd - gD[q]) <= 1e-6 * max(1.0, abs(fd))
        h = lam[q] * 1e-6
        Lp, Lm = lam.copy(), lam.copy()
        Lp[q] += h
        Lm[q] -= h
        fd = (loss(rho, D, Lp) - loss(rho, D, Lm)) / (2 * h)
        assert abs(fd - gL[q]) <= 1e-6 * max(1.0, abs(fd))
    # the step is affine in rho: the gradient is exact up to rounding
    for idx in [(0, 0, 0, 0), (1, 2, 3, 1), (3, 1, 4, 0), (2, 1, 2, 1)]:
        e = np.zeros_like(rho)
        e[idx] = 1.0
        fd = (loss(rho + e, D, lam) - loss(rho - e, D, lam)) / 2
        assert abs(fd - g_rho[idx]) <= 1e-10


def test_oracle_multistep_adjoint_with_agents_matches_finite_differences(oracle, rng):
    """The composed reverse mode the GPU tests compare against (tests/adjoint_ref.py):
    3 steps of (LOD step, agents) with Dirichlet faces, checked by central
    differences of the oracle's own forward."""
    from adjoint_ref import oracle_adjoint
    shape, S, n = (5, 4, 6), 2, 3
    dx, dt = 20.0, 0.01
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-2, 1.0, S)
    rho = rng.random((*shape, S))
    vals = rng.random((*shape, S))
    fm = np.zeros((6, S), np.uint8)
    fm[0, 0] = fm[3, 1] = fm[4, 0] = 1
    na = 12
    pos = rng.uniform(0, 1, (na, 3)) * np.array(shape) * dx
    pos[:4] = pos[0]
    ag = dict(pos=pos, vol=rng.uniform(500, 3000, na), active=(np.arange(na) % 5 != 3).astype(np.uint8))
    ag["sec"], ag["upt"], ag["sat"] = log_uniform(rng, 1e-2, 10.0, (3, na, S))
    w = rng.standard_normal((*shape, S))
    g = oracle_adjoint(oracle, rho, w, n, dt, dx, D, lam, (vals, fm), ag)

    def loss(r=rho, Dv=D, lv=lam, a=ag):
        return float((oracle_adjoint(oracle, r, w, n, dt, dx, Dv, lv, (vals, fm), a)["final"] * w).sum())

    def central(f, h):
        return (f(h) - f(-h)) / (2 * h)

    for q in range(S):
        def fD(e, q=q):
            Dp = D.copy()
            Dp[q] += e
            return loss(Dv=Dp)
        assert abs(central(fD, 1e-4 * D[q]) - g["D"][q]) <= 1e-6 * max(1e-3, abs(g["D"][q]))

        def fL(e, q=q):
            Lp = lam.copy()
            Lp[q] += e
            return loss(lv=Lp)
        assert abs(central(fL, 1e-4 * lam[q]) - g["lambda"][q]) <= 1e-6 * max(1e-3, abs(g["lambda"][q]))
    key = {"secretion": "sec", "uptake": "upt", "saturation": "sat"}
    for a in range(na):
        for name, k in key.items():
            d = a % S

            def fA(e, a=a, d=d, k=k):
                b = dict(ag)
                b[k] = ag[k].copy()
                b[k][a, d] += e
                return loss(a=b)
            fd = central(fA, 1e-3 * ag[k][a, d])
            if not ag["active"][a]:
                assert g[name][a, d] == 0.0 and fd == 0.0
            else:
                assert abs(fd - g[name][a, d]) <= 1e-6 * max(1e-6, abs(g[name][a, d])), (name, a)
    for idx in [(0, 0, 0, 0), (2, 1, 3, 1), (4, 3, 5, 0)]:
        e = np.zeros_like(rho)
        e[idx] = 1e-3
        fd = (loss(r=rho + e) - loss(r=rho - e)) / 2e-3
        assert abs(fd - g["initial"][idx]) <= 1e-9


@needs_ref
@pytest.mark.parametrize("shape,S", [((5, 4, 6), 2), ((2, 3, 2), 1), ((7, 5, 3), 3), ((3, 6, 1), 2)])
def test_gradients_oracle_bitexact_with_reference(oracle, rng, shape, S):
    """compute_all_gradient_vectors of the live reference (after one solver
    step, which sets the neighbour jumps) equals orc_gradients bit for bit,
    and so does the per-voxel accessor path on this uniform mesh."""
    ref = RefLib()
    dx = 20.0
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-2, 1.0, S)
    e = RefEnv(ref, (0.0, 0.0, 0.0, shape[0] * dx, shape[1] * dx, shape[2] * dx), dx, D, lam)
    e.set_dirichlet([0] * S)
    e.set_field(rng.random((*shape, S)))
    e.step(0.01, 1)
    rho = e.field()
    want = oracle.gradients(rho, dx)
    got = e.gradients()
    if shape[2] == 1:  # the reference leaves z untouched (0) when nz == 1
        assert np.all(got[..., 2] == 0.0)
    assert np.array_equal(got, want)
    assert np.array_equal(e.gradients(per_voxel=True), want)


@pytest.mark.parametrize("shape,S,steps", [((9, 7, 8), 3, 40), ((1, 5, 6), 2, 20), ((12, 1, 3), 1, 20),
                                           ((2, 2, 9), 4, 30), ((16, 16, 16), 8, 100)])
def test_fp32_restatement_tracks_the_fp64_oracle(oracle, rng, shape, S, steps):
    """The FP32 path's C restatement (orc_lod_steps_f32: FP32 tables rounded
    once from the reference's factors, deviation form, hi + lo reciprocal)
    stays within 1e-5 relative L-inf of the FP64 oracle, the FP32 target, on
    grids with one- and two-voxel axes and Dirichlet faces."""
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((*shape, S)) * 3
    act = (rng.random(S) < 0.6).astype(np.uint8)
    vals = rng.random((*shape, S)) * 5
    r64 = oracle.lod_steps(rho0, 0.01, 20.0, D, lam, steps, vals, face_mask_all(act))
    r32 = oracle.lod_steps_f32(rho0, 0.01, 20.0, D, lam, steps, vals, face_mask_all(act))
    assert r32.dtype == np.float32
    err = np.abs(r32.astype(np.float64) - r64).max() / np.abs(r64).max()
    assert err <= 1e-5, err
    # deterministic, and the Dirichlet faces carry the FP32-rounded values exactly
    assert np.array_equal(r32, oracle.lod_steps_f32(rho0, 0.01, 20.0, D, lam, steps, vals, face_mask_all(act)))
    if act.any():
        d = int(np.argmax(act))
        assert np.array_equal(r32[0, ..., d], vals[0, ..., d].astype(np.float32))
