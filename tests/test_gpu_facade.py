"""The C++ facade (reference-shaped Microenvironment / Basic_Agent API) run
as a compiled driver, checked against the oracle on the same inputs."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from oracle.oracle import face_mask_all

pytestmark = pytest.mark.gpu


def hash01(a, b):
    h = (a * 2654435761 + b * 40503 + 12345) & 0xFFFFFFFF
    h ^= h >> 13
    h = (h * 0x5BD1E995) & 0xFFFFFFFF
    h ^= h >> 15
    return (h % 100003) / 100003.0


def oracle_demo(oracle, steps, bulk=False):
    shape, S, dx, dt = (20, 18, 16), 2, 20.0, 0.01
    D, lam = [1e5, 3e3], [0.1, 0.01]
    V = shape[0] * shape[1] * shape[2]
    rho = np.array([[hash01(n, d) for d in range(S)] for n in range(V)]).reshape(*shape, S)
    vals = np.empty_like(rho)
    vals[..., 0] = 38.0
    vals[..., 1] = 100.0
    n = 200
    pos = np.array([[400.0 * hash01(a, 7), 360.0 * hash01(a, 8), 320.0 * hash01(a, 9)] for a in range(n)])
    sec = np.array([[10.0 * hash01(a, 20 + d) for d in range(S)] for a in range(n)])
    upt = np.array([[10.0 * hash01(a, 30 + d) for d in range(S)] for a in range(n)])
    sat = np.array([[10.0 * hash01(a, 40 + d) for d in range(S)] for a in range(n)])
    vol = np.full(n, 4.0 / 3.0 * np.pi * 125.0)
    vox = oracle.bin_agents(pos, (0, 0, 0, 400, 360, 320), dx, shape)
    assert (vox >= 0).all()
    t1, t2 = oracle.agent_constants(dt, dx, vol, sec, upt, sat)
    if bulk:
        Sr = np.array([[2.0 * hash01(n, 50 + d) for d in range(S)] for n in range(V)]).reshape(*shape, S)
        Tt = np.array([[5.0 * hash01(n, 60 + d) for d in range(S)] for n in range(V)]).reshape(*shape, S)
        Ur = np.array([[0.5 * hash01(n, 70 + d) for d in range(S)] for n in range(V)]).reshape(*shape, S)
    for _ in range(steps):
        if bulk:
            rho = oracle.bulk_step(rho, dt, Sr, Tt, Ur)
        rho = oracle.lod_steps(rho, dt, dx, D, lam, 1, vals, face_mask_all([1, 0]))
        rho = oracle.cells_step(rho, vox, t1, t2)
    return rho


@pytest.mark.parametrize("precision,sync", [(0, 0), (0, 1), (1, 0)])
def test_facade_demo_matches_oracle(bfb, oracle, tmp_path, precision, sync):
    demo = bfb.PKG / "lib" / "facade_demo"
    assert demo.exists(), "build with python biofvm-b_b200/build.py"
    out = tmp_path / "field.bin"
    r = subprocess.run([str(demo), str(out), str(precision), str(sync), "10"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(20, 18, 16, 2)
    want = oracle_demo(oracle, 10)
    grad = np.fromfile(str(out) + ".grad", dtype=np.float64).reshape(20, 18, 16, 2, 3)
    raw = (tmp_path / "field.bin.mat").read_bytes()
    hdr = np.frombuffer(raw[:20], dtype="<u4")
    assert list(hdr) == [0, 6, 20 * 18 * 16, 0, 27] and raw[20:47] == b"multiscale_microenvironment"
    mat = np.frombuffer(raw[47:], dtype="<f8").reshape(-1, 6)
    assert np.array_equal(mat[:, 4:], got.reshape(-1, 2))  # the field the demo wrote, in voxel columns
    if precision == 0:
        assert np.array_equal(got, want)
        assert np.array_equal(grad, oracle.gradients(want, 20.0))
    else:
        assert np.abs(got - want).max() / np.abs(want).max() <= 1e-5
        # gradients of the FP32 field itself, in FP32 arithmetic
        from test_gpu_gradient import fp32_gradients
        assert np.array_equal(grad, fp32_gradients(got, 20.0).astype(np.float64))


@pytest.mark.parametrize("mode", [1, 2], ids=["callbacks_every_call", "callbacks_tabulated_once"])
def test_facade_bulk_callbacks(bfb, oracle, tmp_path, mode):
    """simulate_bulk_sources_and_sinks with the reference's callback signature,
    evaluated every call (the reference's semantics) or tabulated once."""
    demo = bfb.PKG / "lib" / "facade_demo"
    out = tmp_path / "field.bin"
    r = subprocess.run([str(demo), str(out), "0", "1", "6", str(mode)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(20, 18, 16, 2)
    assert np.array_equal(got, oracle_demo(oracle, 6, bulk=True))
