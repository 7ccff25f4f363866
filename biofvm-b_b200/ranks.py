"""Multi-rank partition of the work: one process per GPU.

The LOD step of one grid does not shard (every configuration fits one GPU),
so several GPUs run either
  * replicas of one grid -- each rank steps its own copy; the ranks meet only
    in a barrier and in the max over ranks of the device-timed region; or
  * an ensemble of independent instances (uneven grids, substrate counts and
    agents), partitioned across ranks by greedy bytes balancing -- each rank
    steps its share as one batch; no collective touches the fields, and
    per-instance results (checksums, timings) are gathered at the end.

This module holds the partition: which rank steps which instances, derived
by every rank alone from the instances' sizes, so that no rank needs to ask
another. The collectives around it (barrier, max and sum over ranks, the
final gather of per-instance results) live in the benchmark driver, which
owns the process group; the library itself needs no torch.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


def shard_instances(weights: Sequence[float], world: int) -> list[int]:
    """Owner rank of each instance: largest first, each to the least loaded
    rank (ties to the lower rank). Deterministic, so every rank computes the
    same partition without communicating. The most loaded rank exceeds the
    mean load by at most one instance's weight."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(weights[i])
    return owner


def local_instances(weights: Sequence[float], rank: int, world: int) -> list[int]:
    """The instances rank `rank` steps, in instance order."""
    return [i for i, o in enumerate(shard_instances(weights, world)) if o == rank]


def instance_bytes(shape: Sequence[int], n_substrates: int, elem_bytes: int) -> int:
    """Field bytes of one instance, the weight of the partition."""
    return int(np.prod(shape)) * int(n_substrates) * int(elem_bytes)
