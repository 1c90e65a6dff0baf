"""Host logic of runs over several GPUs (mdbas_b200/ranks.py), on CPU: the
size-balanced split of a batch of boxes over ranks, and the cross-rank
bookkeeping (slowest rank's time, units of all ranks) with two gloo ranks in
separate processes."""
import os
import socket

import pytest

from mdbas_b200 import ranks, systems


def test_rank_seed():
    assert [ranks.rank_seed(7, r) for r in range(4)] == [7, 8, 9, 10]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8, 100])
def test_shard_sizes_cover_and_balance(world):
    sizes = systems.replica_sizes(64, seed=1)
    parts = ranks.shard_sizes(sizes, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(sizes[i] for i in p) for p in parts]
    # longest-first greedy: within one box of the even share
    assert max(loads) <= sum(sizes) / world + max(sizes)
    if world <= 64:
        assert all(p for p in parts)
    assert parts == ranks.shard_sizes(sizes, world)  # deterministic


def test_shard_sizes_rejects_no_ranks():
    with pytest.raises(ValueError):
        ranks.shard_sizes([3, 3], 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        total, slow, rate = ranks.job_rate(1000.0 * (rank + 1), 2.0 + rank)
        assert total == 3000.0 and slow == 3.0 and rate == pytest.approx(1.0e6)
        assert ranks.max_over_ranks([rank, -rank]) == [1.0, 0.0]
        assert ranks.sum_over_ranks([1.5, rank]) == [3.0, 1.0]
        share = ranks.shard_sizes(systems.replica_sizes(64, seed=1), world)
        got = [None] * world
        dist.all_gather_object(got, share[rank])
        assert got == share            # every rank computes the same split
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port()), nprocs=2, join=True)


def test_single_process_needs_no_group():
    total, slow, rate = ranks.job_rate(500.0, 0.5)
    assert (total, slow) == (500.0, 0.5) and rate == pytest.approx(1.0e6)
