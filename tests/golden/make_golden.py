"""Generate the golden fixtures in this directory by running the REFERENCE
BioFVM-B library, compiled from its own sources (oracle/Makefile `ref`).

    make -C oracle ref && python tests/golden/make_golden.py [out_dir]

Every case uses seeded inputs; the outputs are what the reference computes.
The committed .npz files let the oracle restatement and the GPU path be
checked without the reference present. Regenerate only when a case changes.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle.oracle import RefEnv, RefLib  # noqa: E402


def lu(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def case_lod_15cube_dirichlet(ref):
    """The 75^3 single-substrate recipe (1 substrate, D=1e5, lambda=0.1, dt=0.01, Dirichlet 1.0
    on all faces, U[0,1) field) on a 15^3 grid, 20 steps, both solvers."""
    rng = np.random.default_rng(1)
    dx, dt, steps = 20.0, 0.01, 20
    e = RefEnv(ref, (0, 0, 0, 300, 300, 300), dx, [1e5], [0.1])
    rho0 = rng.random(e.shape)
    e.set_field(rho0)
    e.set_dirichlet([1], value=[1.0])
    e.step(dt, steps)
    out = e.field()
    e2 = RefEnv(ref, (0, 0, 0, 300, 300, 300), dx, [1e5], [0.1])
    e2.set_solver(1)
    e2.set_field(rho0)
    e2.set_dirichlet([1], value=[1.0])
    e2.step(dt, steps)
    return dict(rho0=rho0, out=out, out_avx=e2.field(), dx=dx, dt=dt, steps=steps, D=[1e5], lam=[0.1],
                dir_value=[1.0], activation=[1])


def case_multi(ref, seed, shape, S, steps):
    """Multi-substrate, log-uniform D/lambda, per-voxel Dirichlet values with a
    random activation vector (the reference applies it on all six faces)."""
    rng = np.random.default_rng(seed)
    dx, dt = 20.0, 0.01
    D, lam = lu(rng, 1e2, 1e5, S), lu(rng, 1e-3, 1.0, S)
    box = (0, 0, 0, shape[0] * dx, shape[1] * dx, shape[2] * dx)
    e = RefEnv(ref, box, dx, D, lam)
    assert e.shape == (*shape, S)
    rho0 = rng.random(e.shape)
    act = (rng.random(S) < 0.6).astype(np.uint8)
    vals = rng.random(e.shape) * 40.0
    e.set_field(rho0)
    e.set_dirichlet(act, face_values=vals)
    e.step(dt, steps)
    return dict(rho0=rho0, out=e.field(), dx=dx, dt=dt, steps=steps, D=D, lam=lam, activation=act, dir_values=vals)


def case_bulk(ref):
    rng = np.random.default_rng(7)
    dx, dt = 20.0, 0.01
    shape, S = (9, 8, 7), 3
    D, lam = lu(rng, 1e2, 1e5, S), lu(rng, 1e-3, 1.0, S)
    e = RefEnv(ref, (0, 0, 0, 180, 160, 140), dx, D, lam)
    rho0 = rng.random(e.shape)
    Sr, Tt, Ur = rng.random((3, *e.shape)) * 5.0
    e.set_field(rho0)
    e.set_dirichlet([0] * S)
    e.set_bulk(Sr, Tt, Ur)
    outs = []
    for _ in range(3):  # bulk -> diffusion, three steps (examples/performance_test_voxels.cpp:253-254)
        e.bulk_step(dt)
        e.step(dt, 1)
        outs.append(e.field())
    return dict(rho0=rho0, out=outs[-1], dx=dx, dt=dt, D=D, lam=lam, S_rate=Sr, T_target=Tt, U_rate=Ur)


def case_agents(ref):
    """Agents in a ball, many sharing voxels, plus boundary and outside
    positions; 3 steps of diffusion -> cells (serial, list order)."""
    rng = np.random.default_rng(11)
    dx, dt = 20.0, 0.01
    shape, S = (12, 10, 9), 2
    D, lam = lu(rng, 1e2, 1e5, S), lu(rng, 1e-3, 1.0, S)
    box = (0, 0, 0, shape[0] * dx, shape[1] * dx, shape[2] * dx)
    e = RefEnv(ref, box, dx, D, lam)
    n = 600
    ctr = np.array(box[3:]) / 2
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = ctr + u * (60.0 * rng.random((n, 1)) ** (1 / 3))
    pos[:6] = [[0, 0, 0], box[3:], [20, 20, 20], [19.999999999, 40, 60], [-1, 5, 5], [241, 100, 100]]
    vol = np.full(n, 4.0 / 3.0 * np.pi * 125.0)
    sec, upt, sat = lu(rng, 1e-2, 10, (3, n, S))
    rho0 = rng.random(e.shape)
    e.set_field(rho0)
    e.set_dirichlet([0] * S)
    e.add_agents(pos, vol, sec, upt, sat, dt)
    vox = e.agent_voxels()
    for _ in range(3):
        e.step(dt, 1)
        e.cells_step(dt)
    return dict(rho0=rho0, out=e.field(), dx=dx, dt=dt, D=D, lam=lam, pos=pos, vol=vol, sec=sec, upt=upt, sat=sat,
                voxels=vox, bbox=np.array(box, dtype=float))


def make_cases(ref):
    """Every fixture's arrays, computed by the reference library `ref`."""
    return {
        "lod_15cube_s1_dirichlet": case_lod_15cube_dirichlet(ref),
        "multi_7x5x9_S3": case_multi(ref, 21, (7, 5, 9), 3, 6),
        "multi_1x4x6_S2": case_multi(ref, 22, (1, 4, 6), 2, 4),
        "multi_2x3x1_S2": case_multi(ref, 23, (2, 3, 1), 2, 4),
        "multi_17x3x33_S5": case_multi(ref, 24, (17, 3, 33), 5, 3),
        "bulk_9x8x7_S3": case_bulk(ref),
        "agents_12x10x9_S2": case_agents(ref),
    }


def main(out_dir: Path = HERE):
    for name, data in make_cases(RefLib()).items():
        np.savez_compressed(Path(out_dir) / f"{name}.npz", **{k: np.asarray(v) for k, v in data.items()})
        print("wrote", name)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE)
