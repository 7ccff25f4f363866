"""MATLAB v4 snapshots (bfb_write_matlab) against the reference's own writer
(Microenvironment::write_to_matlab, run from oracle/_ref)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import log_uniform
from oracle.oracle import REF_SO, RefEnv, RefLib

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not REF_SO.exists(), reason="reference library not built")


def read_mat4(path):
    raw = open(path, "rb").read()
    typ, rows, cols, imag, nlen = np.frombuffer(raw[:20], dtype="<u4")
    name = raw[20:20 + nlen].decode()
    data = np.frombuffer(raw[20 + nlen:], dtype="<f8")
    assert typ == 0 and imag == 0 and data.size == rows * cols
    return name, data.reshape(cols, rows)  # one row per voxel (MAT columns)


@needs_ref
@pytest.mark.parametrize("box,S", [((-30.0, 110.0, 0.0, 100.0, 20.0, 100.0), 3), ((0.0, 200.0, 0.0, 160.0, 0.0, 60.0), 1)])
def test_matlab_fp64_byte_identical_to_reference(bfb, tmp_path, box, S):
    rng = np.random.default_rng(S)
    dx = 20.0
    D, lam = log_uniform(rng, 1e2, 1e5, S), log_uniform(rng, 1e-2, 1.0, S)
    x0, x1, y0, y1, z0, z1 = box
    ref = RefLib()
    r = RefEnv(ref, (x0, y0, z0, x1, y1, z1), dx, D, lam)
    env = bfb.Env(None, S, dx=dx, precision=bfb.FP64, domain=box)
    assert env.shape == r.shape
    rho = rng.random(r.shape) * 7
    r.set_field(rho)
    env.set_field(rho)
    r.write_matlab(tmp_path / "ref.mat")
    env.write_matlab(tmp_path / "gpu.mat")
    assert (tmp_path / "gpu.mat").read_bytes() == (tmp_path / "ref.mat").read_bytes()
    env.close()


# (12, 10, 9) x 4: rows of 36 floats (packed); (7, 5, 3) x 3: rows of 9 floats,
# padded on the device to 12
@pytest.mark.parametrize("shape,S", [((12, 10, 9), 4), ((7, 5, 3), 3)])
def test_matlab_fp32_layout(bfb, tmp_path, shape, S):
    rng = np.random.default_rng(7)
    dx = 20.0
    env = bfb.Env(shape, S, dx=dx, precision=bfb.FP32)
    env.set_field(rng.random((*shape, S)))
    env.write_matlab(tmp_path / "f.mat")
    name, m = read_mat4(tmp_path / "f.mat")
    assert name == "multiscale_microenvironment" and m.shape == (np.prod(shape), 4 + S)
    i, j, k = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    assert np.array_equal(m[:, 0], ((i + 0.5) * dx).ravel())
    assert np.array_equal(m[:, 1], ((j + 0.5) * dx).ravel())
    assert np.array_equal(m[:, 2], ((k + 0.5) * dx).ravel())
    assert np.all(m[:, 3] == dx * dx * dx)
    assert np.array_equal(m[:, 4:], env.get_field_raw().astype(np.float64).reshape(-1, S))
    env.close()
