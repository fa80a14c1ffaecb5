"""World-sharded batches (melon3d_b200/shard.py): the greedy prefix split of
the worlds by cumulative body count, and the single all-gather of per-world
results, on world_size-2 gloo process groups on the CPU."""
import os
import socket

import numpy as np
import pytest

from melon3d_b200 import shard


def _batch_counts(worlds, seed=4):
    # body counts of the batched-worlds workload: floor(exp(U[ln 16, ln 512]))
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(np.log(16.0) + rng.uniform(size=worlds) * (np.log(512.0) - np.log(16.0)))).astype(int)


@pytest.mark.parametrize("ranks", [1, 2, 3, 4, 8])
def test_partition_is_contiguous_complete_and_balanced(ranks):
    counts = _batch_counts(4096)
    ranges = shard.partition_worlds(counts, ranks)
    assert len(ranges) == ranks
    assert ranges[0][0] == 0 and ranges[-1][1] == len(counts)
    for (s0, e0), (s1, e1) in zip(ranges, ranges[1:]):
        assert e0 == s1 and s0 <= e0
    total = counts.sum()
    for s, e in ranges:
        # each rank is within one world's bodies of its fair share
        assert abs(counts[s:e].sum() - total / ranks) <= counts.max()


def test_partition_edge_cases():
    assert shard.partition_worlds([], 2) == [(0, 0), (0, 0)]
    assert shard.partition_worlds([5], 3) == [(0, 1), (1, 1), (1, 1)]
    assert shard.partition_worlds([1, 1, 1, 1], 2) == [(0, 2), (2, 4)]
    with pytest.raises(ValueError):
        shard.partition_worlds([1, 2], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, counts, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    try:
        ranges = shard.partition_worlds(counts, world_size)
        s, e = ranges[rank]
        # stand-in per-world results: (world index, body count, rank)
        local = np.array([[k, counts[k], rank] for k in range(s, e)], dtype=np.float64).reshape(-1, 3)
        full = shard.gather_world_results(local, ranges, rank, dist)
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), full)
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    counts = _batch_counts(37, seed=9)
    mp.spawn(_rank_main, args=(2, _free_port(), counts, str(tmp_path)), nprocs=2, join=True)
    ranges = shard.partition_worlds(counts, 2)
    for r in range(2):
        full = np.load(os.path.join(str(tmp_path), "rank%d.npy" % r))
        assert full.shape == (37, 3)
        assert np.array_equal(full[:, 0], np.arange(37))
        assert np.array_equal(full[:, 1], counts)
        owner = np.concatenate([np.full(e - s, k) for k, (s, e) in enumerate(ranges)])
        assert np.array_equal(full[:, 2], owner)
