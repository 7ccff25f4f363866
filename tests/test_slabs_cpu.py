"""x-slab decomposition, host side (no GPU): the pipelined schedule of
slabs.py, run with a numpy stand-in for the two halves of the x sweep, must
reproduce the whole line's Thomas solve bit for bit -- in one process
(emulate_step) and across two gloo ranks (step with a torch.distributed
transport). The reference's exchange is BioFVM_parallel.cpp:948-1255 with the
sends and receives at :832-873; its split of the x planes is :108-144."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent))
from conftest import load_bfb  # noqa: E402

bfb = load_bfb()
import importlib  # noqa: E402

slabs = importlib.import_module(bfb.__name__ + ".slabs")


def factors(n, seed=3):
    rng = np.random.default_rng(seed)
    c1 = rng.uniform(0.1, 2.0)
    den = 1.0 + 2.0 * c1 + rng.uniform(0.0, 0.1, n)
    cb = -c1 / den
    return c1, den, cb


def whole_solve(x, c1, den, cb):
    """Thomas over axis 0 of x (rows, lines) in the order the halves use."""
    y = np.empty_like(x)
    p = x[0] / den[0]
    y[0] = p
    for r in range(1, x.shape[0]):
        p = (x[r] + c1 * p) / den[r]
        y[r] = p
    nxt = y[-1]
    for r in range(x.shape[0] - 2, -1, -1):
        nxt = y[r] - cb[r] * nxt
        y[r] = nxt
    return y


class NumpySlab:
    """Rows [x0, x0 + n) of the lines, with the two halves of the solve."""

    def __init__(self, x, x0, n_global, c1, den, cb):
        self.f = x.copy()
        self.x0, self.nx, self.nx_global = x0, x.shape[0], n_global
        self.lines = x.shape[1]
        self.c1, self.den, self.cb = c1, den, cb

    first = property(lambda s: s.x0 == 0)
    last = property(lambda s: s.x0 + s.nx == s.nx_global)

    def x_forward(self, dt, prev_in, prev_out, l0, l1):
        f = self.f[:, l0:l1]
        r = 0
        if self.first:
            p = f[0] / self.den[0]
            f[0] = p
            r = 1
        else:
            p = prev_in[l0:l1].copy()
        for q in range(r, self.nx):
            p = (f[q] + self.c1 * p) / self.den[self.x0 + q]
            f[q] = p
        if not self.last:
            prev_out[l0:l1] = p

    def x_backward(self, dt, next_in, next_out, l0, l1):
        f = self.f[:, l0:l1]
        r = self.nx - 1
        if self.last:
            nxt = f[r].copy()
            r -= 1
        else:
            nxt = next_in[l0:l1].copy()
        for q in range(r, -1, -1):
            nxt = f[q] - self.cb[self.x0 + q] * nxt
            f[q] = nxt
        if not self.first:
            next_out[l0:l1] = nxt

    def yz(self, dt):
        pass

    def synchronize(self):
        pass


class NumpyPlanes:
    def __init__(self, lines):
        self.t = {n: np.zeros(lines) for n in slabs.PLANES}

    def ptr(self, name):
        return self.t[name]

    def copy_from(self, name, src, src_name, l0, l1):
        self.t[name][l0:l1] = src.t[src_name][l0:l1]


def test_split_planes_cover_the_grid():
    for n in (2, 5, 17, 64):
        for R in range(1, min(n, 7) + 1):
            parts = slabs.split_planes(n, R)
            assert sum(m for _, m in parts) == n and all(m >= 1 for _, m in parts)
            assert [x0 for x0, _ in parts] == list(np.cumsum([0] + [m for _, m in parts])[:-1])
    with pytest.raises(ValueError):
        slabs.split_planes(3, 4)


def test_schedule_sends_match_receives():
    for R in (1, 2, 3, 5):
        for blocks in (1, 3, 8):
            sends, recvs = set(), set()
            for r in range(R):
                for op in slabs.schedule(r, R, 20, blocks):
                    if op[0] == "send":
                        sends.add((r, op[4], "prev_in" if op[1] == "prev_out" else "next_in", op[2], op[3]))
                    elif op[0] == "recv":
                        recvs.add((op[4], r, op[1], op[2], op[3]))
            assert sends == recvs
            ranges = slabs.line_ranges(20, blocks)
            assert ranges[0][0] == 0 and ranges[-1][1] == 20
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))


@pytest.mark.parametrize("n,R,blocks", [(9, 1, 2), (9, 2, 1), (9, 3, 4), (10, 5, 3), (7, 7, 2), (33, 4, 5)])
def test_emulated_slabs_reproduce_the_whole_line(n, R, blocks):
    rng = np.random.default_rng(n * 10 + R)
    lines = 37
    x = rng.random((n, lines))
    c1, den, cb = factors(n)
    want = whole_solve(x, c1, den, cb)
    parts = slabs.split_planes(n, R)
    ss = [NumpySlab(x[x0:x0 + m], x0, n, c1, den, cb) for x0, m in parts]
    planes = [NumpyPlanes(lines) for _ in ss]
    slabs.emulate_step(ss, 0.01, planes, blocks)
    got = np.concatenate([s.f for s in ss])
    assert got.tobytes() == want.tobytes()


def _gloo_rank(rank, world, port, n, lines, blocks, out_dir, q):
    try:
        import datetime

        import torch
        import torch.distributed as dist

        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        rng = np.random.default_rng(5)
        x = rng.random((n, lines))
        c1, den, cb = factors(n)
        x0, m = slabs.split_planes(n, world)[rank]
        slab = NumpySlab(x[x0:x0 + m], x0, n, c1, den, cb)
        planes = {k: torch.zeros(lines, dtype=torch.float64) for k in slabs.PLANES}

        class P:
            def ptr(self, name):
                return planes[name].numpy()

        class T:  # blocking point-to-point messages over gloo
            def send(self, name, l0, l1, peer):
                dist.send(planes[name][l0:l1].contiguous(), dst=peer)

            def recv(self, name, l0, l1, peer):
                buf = torch.empty(l1 - l0, dtype=torch.float64)
                dist.recv(buf, src=peer)
                planes[name][l0:l1] = buf

        slabs.step(slab, 0.01, rank, world, P(), T(), blocks)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), slab.f)
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging the other rank
        q.put((rank, f"{type(e).__name__}: {e}"))


@pytest.mark.parametrize("world,blocks", [(2, 1), (2, 3)])
def test_gloo_ranks_reproduce_the_whole_line(tmp_path, world, blocks):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    n, lines = 11, 29
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, n, lines, blocks, str(tmp_path), q))
             for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == {r: "ok" for r in range(world)}, results
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)])
    rng = np.random.default_rng(5)
    x = rng.random((n, lines))
    want = whole_solve(x, *factors(n))
    assert got.tobytes() == want.tobytes()
