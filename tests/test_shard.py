"""Sharding of the subsets over ranks and the frame-end gather of their
result rows (dice_b200.shard), on the CPU with world_size-2 gloo ranks.

Each rank correlates only its contiguous range (the CPU oracle stands in
for the rank's GPU here) and one all-gather assembles the frame's field rows;
the assembled field must equal a single-process run exactly, since subsets
are independent under USE_FIELD_VALUES.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from dice_b200 import abi
from dice_b200 import shard
from dice_b200 import synthetic as syn


def test_partition_is_contiguous_balanced_and_complete():
    rng = np.random.default_rng(0)
    work = rng.uniform(100, 2000, 1000)
    for world in (1, 2, 3, 8):
        st = shard.partition(work, world)
        assert st[0] == 0 and st[-1] == len(work) and np.all(np.diff(st) > 0)
        sums = [work[st[r]:st[r + 1]].sum() for r in range(world)]
        assert max(sums) - min(sums) <= 2 * work.max()
    st = shard.partition(np.ones(3), 5)          # more ranks than subsets
    assert st[0] == 0 and st[-1] == 3 and np.all(np.diff(st) >= 0)
    assert np.array_equal(shard.partition([], 2), [0, 0, 0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    from datetime import timedelta
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ref, deff = syn.config1(w=160, h=128)
        ref, deff = ref.numpy(), deff.numpy()
        cx, cy = syn.grid_points(160, 128, 21, 9)
        p = abi.default_params(subset_size=21, enable_rotation=1, fast_solver_tolerance=1e-5)
        st = shard.partition(np.full(len(cx), 441.0), world)
        f = syn.init_fields(cx[st[rank]:st[rank + 1]], cy[st[rank]:st[rank + 1]])
        O.execute_frame(p, ref, deff, f, first_frame=True, nthreads=1)
        full = shard.gather_rows(torch.from_numpy(f), st)
        if rank == 0:
            np.save(out_path, full.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_gather_the_frame(tmp_path):
    from oracle import oracle as O
    out = str(tmp_path / "gathered.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    ref, deff = syn.config1(w=160, h=128)
    cx, cy = syn.grid_points(160, 128, 21, 9)
    p = abi.default_params(subset_size=21, enable_rotation=1, fast_solver_tolerance=1e-5)
    f = syn.init_fields(cx, cy)
    O.execute_frame(p, ref.numpy(), deff.numpy(), f, first_frame=True, nthreads=1)
    assert got.shape == f.shape
    assert np.array_equal(got, f)
