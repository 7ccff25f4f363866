"""x-slab decomposition on the device: one grid split into 2-4 slab envs
(bfb_create_slab), stepped by the pipelined schedule of slabs.py with the
ranks emulated one after another on one GPU (plane copies stand in for the
messages; no kernel waits for another), must give the whole grid's FP64 step
bit for bit -- with Dirichlet faces (uniform and per-voxel values, the x
faces held only by the end slabs), several blocks of lines, and slabs of one
plane. The reference splits x at BioFVM_parallel.cpp:108-144 and pipelines
the x lines' solve at :948-1255 (messages at :832-873)."""
import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent))
from conftest import load_bfb  # noqa: E402

bfb = load_bfb()
slabs = importlib.import_module(bfb.__name__ + ".slabs")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

DT = 0.01


class TorchPlanes:
    """The four boundary planes of one slab as device tensors."""

    def __init__(self, lines):
        self.t = {n: torch.zeros(lines, dtype=torch.float64, device="cuda") for n in slabs.PLANES}

    def ptr(self, name):
        return self.t[name].data_ptr()

    def copy_from(self, name, src, src_name, l0, l1):
        self.t[name][l0:l1].copy_(src.t[src_name][l0:l1])
        torch.cuda.synchronize()


def coefficients(S, rng):
    return np.exp(rng.uniform(np.log(1e2), np.log(1e5), S)), np.exp(rng.uniform(np.log(1e-3), 0.0, S))


def dirichlet(env, kind, S, vox=None):
    if kind == "none":
        return
    act = np.ones(S, np.uint8)
    if S > 2:
        act[1] = 0  # one substrate without faces
    fm = np.zeros((6, S), np.uint8)
    fm[:, 0] = 1          # substrate 0: every face
    fm[0:2, 1:] = 1       # the others: the x faces ...
    fm[4, 1:] = 1         # ... and z-lo
    if kind == "uniform":
        env.set_dirichlet_uniform(act, np.linspace(1.0, 2.0, S), face_mask=fm)
    else:
        env.set_dirichlet(act, values=vox, face_mask=fm)


def run_both(shape, S, R, blocks, kind, steps, seed=11):
    rng = np.random.default_rng(seed)
    nxg, ny, nz = shape
    rho = rng.random((nxg, ny, nz, S))
    vox = rng.uniform(0.5, 3.0, (nxg, ny, nz, S))
    D, lam = coefficients(S, rng)
    whole = bfb.Env(shape, S, precision=bfb.FP64)
    whole.set_coefficients(D, lam)
    whole.set_field(rho)
    dirichlet(whole, kind, S, vox)
    whole.simulate(DT, steps)
    want = whole.get_field()
    whole.close()
    parts = slabs.split_planes(nxg, R)
    ss = []
    for x0, m in parts:
        s = bfb.SlabEnv(nxg, x0, m, ny, nz, S)
        s.set_coefficients(D, lam)
        s.set_field(rho[x0:x0 + m])
        dirichlet(s, kind, S, vox[x0:x0 + m])
        ss.append(s)
    planes = [TorchPlanes(s.lines) for s in ss]
    for _ in range(steps):
        slabs.emulate_step(ss, DT, planes, blocks)
    got = np.concatenate([s.get_field() for s in ss])
    for s in ss:
        s.close()
    return got, want


@pytest.mark.parametrize(
    "shape,S,R,blocks,kind",
    [
        ((16, 12, 10), 1, 2, 1, "none"),
        ((16, 12, 10), 3, 2, 3, "uniform"),
        ((17, 9, 13), 5, 3, 2, "voxel"),
        ((4, 20, 8), 2, 4, 2, "uniform"),       # one plane per slab
        ((40, 33, 24), 8, 4, 5, "voxel"),
        ((64, 48, 40), 3, 3, 4, "uniform"),     # y and z take the TMA tiles
        ((96, 64, 64), 4, 2, 8, "none"),
    ],
)
def test_slabs_reproduce_the_whole_grid(shape, S, R, blocks, kind):
    got, want = run_both(shape, S, R, blocks, kind, steps=3)
    assert got.tobytes() == want.tobytes()


def test_slab_envs_refuse_the_whole_grid_calls():
    s = bfb.SlabEnv(10, 5, 5, 8, 8, 2)
    s.set_coefficients(np.array([1e3, 1e4]), np.array([0.1, 0.01]))
    with pytest.raises(bfb.BFBError) as e:
        s.simulate(DT, 1)
    assert e.value.code == -7  # BFB_ERR_UNSUPPORTED
    with pytest.raises(bfb.BFBError):
        s.profile_steps(DT, 1)
    with pytest.raises(bfb.BFBError):
        s.x_forward(DT, 0, 0)  # past the grid's first plane a previous plane is needed
    s.close()
    with pytest.raises(bfb.BFBError):
        bfb.SlabEnv(10, 8, 5, 8, 8, 2)  # past the grid's last plane
