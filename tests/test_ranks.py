"""Multi-rank host logic on CPU: the partition (biofvm-b_b200/ranks.py) and
the collectives of the benchmark driver (bench.py), with two gloo ranks.

The multi-GPU runs are replicas of one grid (barrier + max over ranks of the
timed region) or an ensemble of independent instances sharded across ranks
(greedy bytes balancing, per-instance results gathered at the end). Both use
only the collectives exercised here; no GPU is needed.
"""
from __future__ import annotations

import importlib.util
import os
import socket
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def load_ranks():
    spec = importlib.util.spec_from_file_location("bfb_ranks", ROOT / "biofvm-b_b200" / "ranks.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_bench():
    spec = importlib.util.spec_from_file_location("bfb_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def ensemble_weights(seed=4, n=256):
    """Field bytes of an uneven ensemble of 256 grids: edges U{32..160} per axis, 1-6 substrates, FP32."""
    rng = np.random.default_rng(seed)
    ranks = load_ranks()
    return [ranks.instance_bytes(rng.integers(32, 161, 3), int(rng.integers(1, 7)), 4) for _ in range(n)]


def test_shard_is_a_balanced_partition():
    ranks = load_ranks()
    w = ensemble_weights()
    for world in (1, 2, 3, 4, 8):
        owner = ranks.shard_instances(w, world)
        assert sorted(set(owner)) == list(range(min(world, len(w))))
        loads = [sum(x for x, o in zip(w, owner) if o == r) for r in range(world)]
        assert sum(loads) == sum(w)
        # greedy largest-first: no rank exceeds the mean by more than one instance
        assert max(loads) - sum(w) / world <= max(w)
        parts = [ranks.local_instances(w, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(w)))
    assert ranks.shard_instances([5, 5, 5], 2) == [0, 1, 0]  # ties go to the lower rank
    with pytest.raises(ValueError):
        ranks.shard_instances(w, 0)


def test_single_process_is_collective_free():
    bench = load_bench()
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.sum_over_ranks(2.0) == 2.0
    g = bench.gather_by_instance([1], [[7.0, 8.0]], 3, 2)
    assert np.array_equal(g, [[0, 0], [7, 8], [0, 0]])
    bench.rank_barrier()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    try:
        import torch.distributed as dist
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        ranks, bench = load_ranks(), load_bench()
        # the benchmark's uneven ensemble: every rank derives the same specs and
        # the same partition without communicating
        specs = bench.ensemble_specs()
        w = [ranks.instance_bytes(sp["shape"], sp["S"], 4) for sp in specs]
        owner = ranks.shard_instances(w, world)
        mine = ranks.local_instances(w, rank, world)
        assert all(owner[i] == rank for i in mine)
        loads = [sum(x for x, o in zip(w, owner) if o == r) for r in range(world)]
        assert max(loads) - sum(w) / world <= max(w)
        # host-computed per-instance values, gathered by instance id
        vals = [[float(specs[i]["D"].sum()), float(specs[i]["lam"].sum()), float(specs[i]["agents"])] for i in mine]
        g = bench.gather_by_instance(mine, vals, len(specs), 3)
        expect = np.array([[sp["D"].sum(), sp["lam"].sum(), sp["agents"]] for sp in specs])
        assert np.array_equal(g, expect)
        # timed region of a multi-GPU run: the slowest rank's
        t = 1.25 + rank
        assert bench.max_over_ranks(t) == 1.25 + (world - 1)
        # whole-job throughput: units of all ranks
        assert bench.sum_over_ranks(float(len(mine))) == float(len(w))
        bench.rank_barrier()
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging the other rank
        q.put((rank, f"{type(e).__name__}: {e}"))


def test_two_gloo_ranks_shard_gather_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, msg = q.get(timeout=120)
        results[r] = msg
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == {0: "ok", 1: "ok"}, results
