"""World-sharded batches over several GPUs.

A batch of independent worlds (m3d_gpu_batch_create) has no coupling between
worlds, so N ranks (one process per GPU) each step a contiguous range of the
worlds as their own batch and exchange nothing while stepping.  The ranges
are a greedy prefix split of the cumulative body count, which balances the
per-rank solve work (it grows with bodies, not with worlds).  The only
collective is one all-gather of the per-world results at the end (final
centroids, body-substeps), over NCCL on GPUs or gloo on the CPU.

The reference is single-process (its parallel unit is a thread pool inside
one world, src/m3d_internal.h:550-568); this split is this project's own.
"""
import numpy as np


def partition_worlds(body_counts, ranks):
    """Contiguous world ranges [(start, end)] for `ranks` ranks: rank r ends
    at the first world where the cumulative body count reaches
    (r + 1) / ranks of the total (greedy prefix split).  Every world belongs
    to exactly one range; a rank may get an empty range when there are fewer
    worlds than ranks."""
    counts = np.asarray(body_counts, dtype=np.int64)
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    n = len(counts)
    cum = np.cumsum(counts)
    total = int(cum[-1]) if n else 0
    bounds = [0]
    for r in range(1, ranks):
        target = total * r / ranks
        # first world index whose inclusive cumulative count reaches the target
        k = int(np.searchsorted(cum, target, side="left")) + 1 if total > 0 else (n * r) // ranks
        k = min(max(k, bounds[-1]), n)
        bounds.append(k)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(ranks)]


def gather_world_results(local, ranges, rank, dist, device="cpu"):
    """All-gather per-world result rows (a float64 array of shape
    [worlds in this rank's range, k]) into the full [worlds, k] array on
    every rank, in world order.  One collective: rows are padded to the
    largest range so every rank sends the same shape."""
    import torch

    local = np.asarray(local, dtype=np.float64)
    k = local.shape[1] if local.ndim == 2 else 1
    local = local.reshape(-1, k)
    start, end = ranges[rank]
    if local.shape[0] != end - start:
        raise ValueError("rank %d holds %d rows for the range [%d, %d)" % (rank, local.shape[0], start, end))
    width = max(e - s for s, e in ranges)
    buf = torch.zeros((max(width, 1), k), dtype=torch.float64, device=device)
    if end > start:
        buf[: end - start] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(buf) for _ in ranges]
    dist.all_gather(parts, buf)
    rows = [p[: e - s].cpu().numpy() for p, (s, e) in zip(parts, ranges)]
    return np.concatenate(rows, axis=0) if rows else np.zeros((0, k))
