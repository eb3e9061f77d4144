"""One process per GPU: process-group setup, max-over-ranks timing, and the
split of a batch's instances over ranks.

A single DiffPhD instance does not shard: its inverse factor ``S^T S`` is
dense-ish and every local/global iteration would need an all-gather of the
positions, so several GPUs run independent replicas. Independent instances
of a batched rollout shard by instance: each rank runs the instances it owns
with no collective inside the rollout, and one gather after it collects the
per-instance results (losses, gradients) on rank 0.

``torchrun`` (or any launcher that sets ``WORLD_SIZE``, ``RANK``,
``LOCAL_RANK``, ``MASTER_ADDR``, ``MASTER_PORT``) starts the processes; NCCL
serves the GPU ranks and gloo the CPU tests of this module.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    group: object  # torch.distributed when world > 1, else None
    device: torch.device


def setup(backend: str = "nccl", timeout_s: float = 600.0, device: torch.device | None = None) -> Ranks:
    """Join the job's process group (when ``WORLD_SIZE`` > 1) with a bounded collective timeout."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if device is None:
        device = torch.device("cuda", local) if backend == "nccl" else torch.device("cpu")
    group = None
    if world > 1:
        import torch.distributed as dist

        kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if backend == "nccl":
            kwargs["device_id"] = device
        dist.init_process_group(backend, **kwargs)
        group = dist
    return Ranks(world, rank, local, group, device)


def barrier(ranks: Ranks) -> None:
    if ranks.group is not None:
        ranks.group.barrier()


def max_over_ranks(value: float, ranks: Ranks) -> float:
    """The largest of every rank's ``value`` (a device time), on every rank."""
    if ranks.group is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=ranks.device)
    ranks.group.all_reduce(t, op=ranks.group.ReduceOp.MAX)
    return float(t.item())


def shard_instances(costs, world: int) -> list[list[int]]:
    """Split instances over ``world`` ranks, longest first onto the least loaded rank
    (ties to the lower rank); each rank's list is in ascending instance order."""
    costs = np.asarray(costs, dtype=np.float64)
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [sorted(np.flatnonzero(owner == r).tolist()) for r in range(world)]


def gather_instances(local: torch.Tensor, owned: list[int], shards: list[list[int]], ranks: Ranks):
    """Rows of ``local`` (one per owned instance, in ``owned`` order) from every rank, as one
    tensor in instance order on rank 0 (None elsewhere)."""
    if ranks.group is None:
        out = torch.empty_like(local)
        out[torch.as_tensor(owned, dtype=torch.long, device=local.device)] = local
        return out
    width = max(len(s) for s in shards)
    padded = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: len(owned)] = local
    pieces = [torch.empty_like(padded) for _ in range(ranks.world)]
    ranks.group.all_gather(pieces, padded)
    if ranks.rank != 0:
        return None
    count = sum(len(s) for s in shards)
    out = torch.empty((count,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, shard in enumerate(shards):
        if shard:
            out[torch.as_tensor(shard, dtype=torch.long, device=local.device)] = pieces[r][: len(shard)]
    return out


def teardown(ranks: Ranks) -> None:
    if ranks.group is not None:
        ranks.group.destroy_process_group()
