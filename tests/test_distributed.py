"""Multi-rank plumbing on CPU: two gloo ranks (the N>1 paths of bench.py and
of data-parallel training use the same functions over NCCL on GPUs)."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from vgr_b200.distributed import allreduce_gradients, camera_shard, max_over_ranks


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
        results[rank] = (
            [g.tolist() for g in grads],
            slowest,
            (shard.start, shard.stop),
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
        grads, slowest, shard = results[rank]
        assert grads[0] == torch.full((5, 3), 1.5).tolist()
        assert grads[1] == (torch.arange(7, dtype=torch.float32) * 1.5).tolist()
        assert grads[2] == torch.full((4,), 5.0).tolist()
        assert slowest == 2.5
    assert results[0][2] == (0, 5) and results[1][2] == (5, 10)
