"""Subset sharding over ranks (one process per GPU).

With USE_FIELD_VALUES every subset depends only on its own previous-frame
solution (DICe_Initializer.cpp:399-421), so the subsets of a frame split into
independent contiguous ranges, one per rank, with the images replicated.  The
only exchange is at frame end: the per-subset result rows are gathered so
that every rank (or the caller) holds the whole field, as the reference's
MPI ranks write their parts of the output (DICe_MainPage.md:143-147).

`partition` balances the ranges by expected work (pixels x expected
iterations per subset); `gather_rows` is one all-gather of the ranks' row
blocks over torch.distributed (NCCL between GPUs, gloo on the CPU).
"""
import numpy as np


def partition(work, world):
    """Contiguous ranges [starts[r], starts[r+1]) of subsets, one per rank,
    with nearly equal summed `work` (one value per subset, e.g. active pixels
    times expected iterations).  Every rank gets at least one subset while
    there are enough subsets."""
    work = np.asarray(work, dtype=np.float64)
    n = len(work)
    if world < 1:
        raise ValueError("world must be >= 1")
    if n == 0:
        return np.zeros(world + 1, dtype=np.int64)
    c = np.concatenate([[0.0], np.cumsum(np.maximum(work, 0.0))])
    total = c[-1]
    starts = np.zeros(world + 1, dtype=np.int64)
    for r in range(1, world):
        starts[r] = int(np.searchsorted(c, total * r / world, side="left"))
    starts[world] = n
    # ordered ranges, each non-empty when there are at least `world` subsets
    lo_gap = 1 if n >= world else 0
    for r in range(1, world):
        hi = n - lo_gap * (world - r)
        starts[r] = min(max(starts[r], starts[r - 1] + lo_gap), hi)
    return starts


def gather_rows(local, starts, group=None):
    """All-gather of the ranks' row blocks (rank r holds rows
    starts[r]:starts[r+1] of the full array, as a tensor of shape
    (rows, ...)).  Returns the full array on every rank.  Blocks are padded
    to the largest so that one collective moves them all."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [int(starts[r + 1] - starts[r]) for r in range(world)]
    m = max(counts)
    rank = dist.get_rank(group)
    assert local.shape[0] == counts[rank]
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:counts[rank]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:c] for b, c in zip(bufs, counts)], 0)
