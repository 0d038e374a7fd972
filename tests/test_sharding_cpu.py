"""Sharding across ranks (bdsim_b200.sharding), world size 2 over gloo on CPU:
each rank's contiguous trajectory range, the MAX of per-rank times and the SUM
of ensemble sums -- the host logic bench.py and a multi-GPU ensemble use --
and ranks that integrate their shards (with the oracle: no GPU here) and give
the one-process ensemble."""
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


STEPS = 3


def _span(sim):
    from bdsim_b200.params import SimParams
    s = SimParams()
    s.dt, s.implicit_loop_tol = sim.dt, sim.implicit_loop_tol
    s.time_start, s.time_end = 0.0, (STEPS - 1) * sim.dt
    return s


def _integrate_shard(lo, hi):
    """The oracle's integration of trajectories lo..hi-1 of a seeded uneven
    ensemble, and the ensemble sums (count, sum Rg^2, sum Rg^4) over them."""
    from bdsim_b200 import properties, workloads
    from oracle import oracle as O
    phys, sims, R0, seeds = workloads.uneven_wlc(10, seed=3, Ns=[8, 12, 20, 31, 17, 40, 9, 25, 14, 33])
    port = O.port()
    outs = []
    for i in range(lo, hi):
        R, st, status, _ = port.integrate(R0[i], phys[i], _span(sims[i]), (1, -1, seeds[i]))
        outs.append((i, R, st, status))
    rg = np.array([properties.radius_of_gyration_sq(R) for _, R, _, _ in outs])
    return outs, np.array([len(outs), rg.sum(), (rg ** 2).sum()])


def _shard_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Ns = [8, 12, 20, 31, 17, 40, 9, 25, 14, 33]
        lo, hi = shard_bounds(bead_cost(Ns), world)[rank]
        outs, sums = _integrate_shard(lo, hi)
        gathered = [None] * world
        dist.all_gather_object(gathered, outs)
        total = reduce_sum(sums, dist)
        if rank == 0:
            out["chains"] = [c for part in gathered for c in part]
            out["sums"] = list(total)
            out["bounds"] = shard_bounds(bead_cost(Ns), world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_integrate_their_shards_like_one_process():
    """Each rank integrates its cost-balanced shard of an uneven ensemble; the
    union of the shards is the one-process ensemble bit for bit, and the
    reduced ensemble sums match it."""
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_shard_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (lo0, hi0), (lo1, hi1) = res["bounds"]
    assert lo0 == 0 and hi0 == lo1 and hi1 == 10 and 0 < hi0 < 10
    alone, sums = _integrate_shard(0, 10)
    got = res["chains"]
    assert [c[0] for c in got] == list(range(10))
    for (i, R, st, status), (j, R1, st1, status1) in zip(got, alone):
        assert i == j and st == st1 and status == status1
        assert np.array_equal(R, R1)
    assert res["sums"][0] == sums[0]
    assert np.allclose(res["sums"][1:], sums[1:], rtol=1e-13, atol=0)
