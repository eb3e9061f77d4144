"""The multi-rank plumbing of bench.py and batched sharding, as two gloo ranks on the CPU."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from newton_solver_diff_phd_b200 import distributed


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})


def _collectives(rank, world, port):
    _env(rank, world, port)
    ranks = distributed.setup("gloo", timeout_s=30.0)
    assert (ranks.world, ranks.rank) == (world, rank)
    # Timing: the slowest rank's device time on every rank.
    assert distributed.max_over_ranks(10.0 + rank, ranks) == 10.0 + world - 1
    # Batched instances: a deterministic split, then one gather in instance order.
    costs = np.arange(1, 12, dtype=np.float64) ** 2
    shards = distributed.shard_instances(costs, world)
    owned = shards[rank]
    local = torch.tensor([[float(i), float(i) ** 2] for i in owned], dtype=torch.float64).reshape(-1, 2)
    gathered = distributed.gather_instances(local, owned, shards, ranks)
    if rank == 0:
        expected = torch.tensor([[float(i), float(i) ** 2] for i in range(len(costs))], dtype=torch.float64)
        assert torch.equal(gathered, expected)
    else:
        assert gathered is None
    distributed.barrier(ranks)
    distributed.teardown(ranks)


def _lost_rank(rank, world, port):
    _env(rank, world, port)
    ranks = distributed.setup("gloo", timeout_s=5.0)
    distributed.barrier(ranks)
    if rank == 1:
        return  # leaves between steps, before the next collective
    with pytest.raises(RuntimeError):
        distributed.max_over_ranks(1.0, ranks)


def test_two_gloo_ranks_time_split_and_gather():
    mp.spawn(_collectives, args=(2, _free_port()), nprocs=2, join=True)


@pytest.mark.timeout(120)
def test_a_rank_that_leaves_ends_the_next_collective_with_an_error():
    mp.spawn(_lost_rank, args=(2, _free_port()), nprocs=2, join=True)


def test_shards_are_disjoint_balanced_and_cover_every_instance():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1.0, 100.0, 257)
    for world in (1, 2, 3, 8):
        shards = distributed.shard_instances(costs, world)
        assert sorted(i for s in shards for i in s) == list(range(len(costs)))
        loads = [costs[s].sum() for s in shards]
        assert max(loads) - min(loads) <= costs.max()
        assert shards == distributed.shard_instances(costs, world)


def test_single_process_defaults():
    for name in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(name, None)
    ranks = distributed.setup("gloo")
    assert ranks.world == 1 and ranks.group is None
    assert distributed.max_over_ranks(3.5, ranks) == 3.5
    local = torch.arange(6, dtype=torch.float64).reshape(3, 2)
    assert torch.equal(distributed.gather_instances(local, [2, 0, 1], [[0, 1, 2]], ranks), local[[1, 2, 0]])
