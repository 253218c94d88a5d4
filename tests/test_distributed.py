"""Multi-rank plumbing on CPU: two gloo ranks (the N>1 paths of bench.py and
of data-parallel training use the same functions over NCCL on GPUs)."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from vgr_b200.distributed import (
    allreduce_gradients,
    camera_costs,
    camera_shard,
    max_over_ranks,
    weighted_camera_shards,
)


def test_camera_shards_cover_the_batch_once():
    for batch in (0, 1, 7, 64, 1024):
        for world in (1, 2, 3, 8):
            covered = []
            for rank in range(world):
                s = camera_shard(batch, world, rank)
                covered.extend(range(batch)[s])
            assert covered == list(range(batch)), (batch, world)
            sizes = [len(range(batch)[camera_shard(batch, world, r)]) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        camera_shard(4, 2, 2)


def test_camera_costs_read_intersections_from_tile_ranges():
    # Three cameras of 2, 1 and 3 tiles; empty tiles hold start >= end.
    starts = torch.tensor([0, 5, -1, 9, 9, 20], dtype=torch.int32)
    ends = torch.tensor([5, 9, -1, 9, 20, 26], dtype=torch.int32)
    costs = camera_costs(starts, ends, [0, 2, 3, 6], [100, 50, 300], intersection_weight=4.0)
    assert costs == [100 + 4 * 9, 50 + 0, 300 + 4 * (0 + 11 + 6)]


def test_weighted_shards_are_contiguous_balanced_and_cover_the_batch():
    gen = torch.Generator().manual_seed(3)
    for world in (1, 2, 3, 4, 8):
        for count in (0, 1, 5, 64, 1024):
            costs = (torch.rand(count, generator=gen) ** 3 * 100).tolist()
            shards = weighted_camera_shards(costs, world)
            assert len(shards) == world
            assert [i for s in shards for i in range(count)[s]] == list(range(count))
            if count >= world:
                assert all(s.stop > s.start for s in shards)
            if count >= 16 * world and world > 1:
                # Each shard is within the largest single cost of the even share.
                share = sum(costs) / world
                worst = max(costs)
                assert all(abs(sum(costs[s]) - share) <= worst + 1e-6 for s in shards)
    # One very expensive camera gets a rank of its own.
    assert weighted_camera_shards([1000.0] + [1.0] * 20, 2) == [slice(0, 1), slice(1, 21)]
    with pytest.raises(ValueError):
        weighted_camera_shards([1.0, -1.0], 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, results) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # Each rank holds different gradients of the same parameters.
        grads = [
            torch.full((5, 3), float(rank + 1)),
            torch.arange(7, dtype=torch.float32) * (rank + 1),
            torch.full((4,), float(10 * rank)),
        ]
        allreduce_gradients(grads, bucket_bytes=64)  # small buckets: several collectives
        slowest = max_over_ranks(1.5 + rank)
        shard = camera_shard(10, world, rank)
        # Both ranks derive the work split from the same calibration costs
        # with no exchange; the gathered splits must agree.
        costs = [float((7 * c) % 13 + 1) for c in range(40)]
        mine = [(s.start, s.stop) for s in weighted_camera_shards(costs, world)]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        results[rank] = (
            [g.tolist() for g in grads],
            slowest,
            (shard.start, shard.stop),
            gathered,
        )
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_average_gradients_and_time_by_max():
    world = 2
    manager = mp.Manager()
    results = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), results), nprocs=world, join=True)
    assert set(results.keys()) == {0, 1}
    for rank in range(world):
        grads, slowest, shard, splits = results[rank]
        assert splits[0] == splits[1]
        assert grads[0] == torch.full((5, 3), 1.5).tolist()
        assert grads[1] == (torch.arange(7, dtype=torch.float32) * 1.5).tolist()
        assert grads[2] == torch.full((4,), 5.0).tolist()
        assert slowest == 2.5
    assert results[0][2] == (0, 5) and results[1][2] == (5, 10)
