"""World-sharded batches on the GPU: two ranks (processes) each step their
range of the batched-worlds workload as one batch - no kernel of one rank
waits on the other - and one all-gather (gloo, on the CPU) collects the
per-world centroids; they must equal, bit for bit, the centroids of the same
worlds stepped as one batch in a single process."""
import os
import socket

import numpy as np
import pytest

from melon3d_b200 import harness, shard

pytestmark = pytest.mark.gpu

WORLDS, STEPS = 24, 20


def _centroids(lib, first, count):
    import ctypes as C
    scenes = [harness.Scene(lib, harness.BATCH_WORLD, k) for k in range(first, first + count)]
    arr = (C.c_void_p * count)(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, count)
    for s in scenes:
        s.close()
    assert batch
    for _ in range(STEPS):
        lib.m3d_world_step(batch, 1.0 / 60.0, 4)
    assert lib.m3d_gpu_status(batch) == 0
    n = lib.m3d_gpu_body_capacity(batch)
    pos = (C.c_float * (3 * n))()
    lib.m3d_gpu_read_poses(batch, pos, None, n)
    p = np.frombuffer(pos, dtype=np.float32).reshape(n, 3).astype(np.float64)
    out = np.zeros((count, 3))
    for k in range(count):
        f0, f1 = lib.m3d_gpu_batch_first_body(batch, k), lib.m3d_gpu_batch_first_body(batch, k + 1)
        out[k] = p[f0 + 1:f1].mean(axis=0)  # slot f0 is the world's ground box
    lib.m3d_world_destroy(batch)
    return out


def _rank(rank, world_size, port, out_dir):
    import datetime

    import torch.distributed as dist

    from melon3d_b200 import api
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=120))
    try:
        counts = [harness.batch_world_bodies(k) for k in range(WORLDS)]
        ranges = shard.partition_worlds(counts, world_size)
        s, e = ranges[rank]
        mine = _centroids(api.load_gpu(), s, e - s) if e > s else np.zeros((0, 3))
        full = shard.gather_world_results(mine, ranges, rank, dist)
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), full)
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_batch(tmp_path):
    import torch.multiprocessing as mp

    from melon3d_b200 import api
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    whole = _centroids(api.load_gpu(), 0, WORLDS)
    for r in range(2):
        got = np.load(os.path.join(str(tmp_path), "rank%d.npy" % r))
        assert got.shape == whole.shape
        assert np.array_equal(got.view(np.uint64), whole.view(np.uint64)), r
