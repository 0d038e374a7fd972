"""Sharding across ranks (bdsim_b200.sharding), world size 2 over gloo on CPU:
each rank's contiguous trajectory range, the MAX of per-rank times and the SUM
of ensemble sums -- the host logic bench.py and a multi-GPU ensemble use."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from bdsim_b200.sharding import bead_cost, reduce_max, reduce_sum, shard_bounds


def test_bounds_tile_the_range_and_balance_cost():
    rng = np.random.default_rng(0)
    Ns = rng.integers(20, 201, size=8192)
    for world in (1, 2, 3, 8):
        b = shard_bounds(bead_cost(Ns), world)
        assert b[0][0] == 0 and b[-1][1] == len(Ns)
        assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
        loads = [bead_cost(Ns[lo:hi]).sum() for lo, hi in b]
        assert max(loads) - min(loads) <= 2 * bead_cost([200])[0]
    assert shard_bounds(np.ones(4096), 2) == [(0, 2048), (2048, 4096)]
    assert shard_bounds(np.ones(3), 4)[-1][1] == 3
    assert shard_bounds([], 2) == [(0, 0), (0, 0)]
    with pytest.raises(ValueError):
        shard_bounds([1.0], 0)


def test_reductions_without_a_process_group():
    assert reduce_max(3.5) == 3.5
    assert np.array_equal(reduce_sum([1.0, 2.0]), [1.0, 2.0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 1000
        lo, hi = shard_bounds(np.ones(n), world)[rank]
        # per-rank "device time" and ensemble sums over its chains
        t = 1.0 + rank
        seeds = np.arange(lo, hi)
        sums = np.array([hi - lo, seeds.sum(), (seeds ** 2).sum()], dtype=np.float64)
        out[rank] = (lo, hi, reduce_max(t, dist), list(reduce_sum(sums, dist)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (lo0, hi0, t0, s0), (lo1, hi1, t1, s1) = res[0], res[1]
    assert (lo0, hi0, lo1, hi1) == (0, 500, 500, 1000)  # union = the single-GPU ensemble
    assert t0 == t1 == 2.0  # MAX over ranks
    allseeds = np.arange(1000)
    assert s0 == s1 == [1000.0, float(allseeds.sum()), float((allseeds ** 2).sum())]
