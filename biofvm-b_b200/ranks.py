"""Multi-rank plumbing: one process per GPU, torch.distributed between them.

The LOD step of one grid does not shard (every configuration fits one GPU),
so several GPUs run either
  * replicas of one grid -- each rank steps its own copy; the ranks meet only
    in a barrier and in the max over ranks of the device-timed region; or
  * an ensemble of independent instances (uneven grids, substrate counts and
    agents), partitioned across ranks by greedy bytes balancing -- each rank
    steps its share as one batch; no collective touches the fields, and
    per-instance results (checksums, timings) are gathered at the end.

This module holds that host logic. It runs with the NCCL backend on GPUs and
with gloo on CPU (the tests), and does nothing collective when
torch.distributed is not initialised (one process).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch
import torch.distributed as dist


def _active() -> bool:
    return dist.is_available() and dist.is_initialized()


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


def barrier(device: torch.device | None = None) -> None:
    """Barrier across ranks (a no-op in one process), then a device sync."""
    if _active():
        dist.barrier()
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(x: float, device: torch.device | None = None) -> float:
    """The maximum of x over all ranks (x itself in one process). The timed
    region of a multi-GPU run is the slowest rank's."""
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device: torch.device | None = None) -> float:
    """The sum of x over all ranks (x itself in one process)."""
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_by_instance(local_ids: Sequence[int], local_values: Sequence[Sequence[float]], n_instances: int,
                       width: int, device: torch.device | None = None) -> np.ndarray:
    """Every rank receives the [n_instances, width] array of per-instance
    values (per-substrate checksums, for example), each row filled by the rank
    that owns the instance. Rows no rank owns stay 0. One all-reduce."""
    buf = torch.zeros((n_instances, width), dtype=torch.float64, device=device)
    for i, v in zip(local_ids, local_values):
        row = torch.as_tensor(np.asarray(v, dtype=np.float64).reshape(-1)[:width], device=device)
        buf[i, :row.numel()] = row
    if _active():
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)  # every row has exactly one owner
    return buf.cpu().numpy()
