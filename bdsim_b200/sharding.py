"""Trajectory sharding across GPUs (one process per GPU).

Trajectories are independent and each owns its RNG stream (trajectory i is
seeded seed+i, python/bdsim/ensemble.py:197-199), so N GPUs split an ensemble
into contiguous trajectory ranges with no exchange on the data path: the union
of the shards is the single-GPU ensemble, chain for chain. Ranges are balanced
by an estimated cost per trajectory (pair work of the D.x products, ~N^2, for
ensembles of uneven N). Only the timing and the ensemble sums cross ranks
(torch.distributed: NCCL on GPUs, gloo in the CPU tests)."""
from __future__ import annotations

import numpy as np


def shard_bounds(costs, world: int) -> list:
    """Split items 0..n-1 (cost costs[i] each) into `world` contiguous ranges
    [lo, hi) of near-equal total cost; returns world (lo, hi) pairs (empty
    ranges when n < world)."""
    costs = np.asarray(costs, dtype=np.float64)
    n = costs.size
    if world < 1:
        raise ValueError("world must be >= 1")
    if n == 0:
        return [(0, 0)] * world
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(cum, target, side="left"))
        # the cut nearer the target, never before the previous cut
        if k > 0 and abs(cum[k - 1] - target) <= abs(cum[min(k, n)] - target):
            k -= 1
        cuts.append(max(cuts[-1], min(k, n)))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def bead_cost(n_beads) -> np.ndarray:
    """Estimated cost per chain-step of a chain of N beads: its pair work."""
    n = np.asarray(n_beads, dtype=np.float64)
    return n * n


def reduce_max(value: float, dist=None, device=None) -> float:
    """MAX over ranks (the value itself without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(values, dist=None, device=None) -> np.ndarray:
    """Element-wise SUM over ranks of a small float vector (ensemble sums:
    counts, sums and sums of squares of the observables)."""
    v = np.asarray(values, dtype=np.float64)
    if dist is None or not dist.is_initialized():
        return v.copy()
    import torch
    t = torch.tensor(v, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()
