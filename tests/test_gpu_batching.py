"""Batches of uneven chains through one bdcu_run: buckets by bead count with
device work lists, autotuned launch shapes, slot pools (bdcu_reserve /
bdcu_update_chains / bdcu_select) and CUDA-graph capture of a run.

Tolerances as in test_gpu_parity: CALL_TOL = 1e-10 for the plain form per
call against the oracle, MIXED_TOL = 1e-4 for the FP32-mixed form."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi, workloads
from bdsim_b200.engine import BdcuError, Context
from bdsim_b200.params import SimParams

pytestmark = pytest.mark.gpu

CALL_TOL = 1e-10
MIXED_TOL = 1e-4
STEPS = 4
# one chain or more in every bucket: warp (N <= 64, mixed form), and the block
# kernel's N <= 64, <= 128, <= 256 and larger
NS = [8, 20, 41, 64, 65, 90, 128, 129, 170, 256, 257, 300]


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, float(np.max(np.abs(b)))))


def _span(sim, steps):
    s = SimParams()
    s.dt, s.implicit_loop_tol = sim.dt, sim.implicit_loop_tol
    s.time_start, s.time_end = 0.0, (steps - 1) * sim.dt
    return s


@pytest.fixture(scope="module")
def uneven():
    return workloads.uneven_wlc(len(NS), seed=7, Ns=NS)


@pytest.fixture(scope="module")
def port_results(uneven, port):
    phys, sims, R0, seeds = uneven
    out = []
    for p, s, r, sd in zip(phys, sims, R0, seeds):
        R, st, status, _ = port.integrate(r, p, _span(s, STEPS), (1, -1, sd))
        out.append((R, st, status))
    return out


def _ensemble(uneven, form):
    phys, sims, R0, seeds = uneven
    return B.Ensemble(phys, sims, R0, [(1, -1, sd) for sd in seeds], form=form)


def test_plan_buckets_cover_the_batch(uneven):
    ens = _ensemble(uneven, "mixed")
    plan = ens.plan()
    assert sum(b["n_chains"] for b in plan) == len(NS)
    by_id = {b["bucket"]: b for b in plan}
    # FP32-mixed default team shapes: (2,1), (4,1), (4,2), (8,2) warps x beads per thread
    for bid, (T, Q, lo, hi) in enumerate([(2, 1, 8, 64), (4, 1, 65, 128), (4, 2, 129, 256), (8, 2, 257, 300)]):
        b = by_id[bid]
        assert b["kernel"] == _abi.KERNEL_TEAM and (b["team_warps"], b["team_beads_per_thread"]) == (T, Q), b
        assert (b["min_beads"], b["max_beads"]) == (lo, hi), b
        assert b["n_chains"] == sum(lo <= n <= hi for n in NS)
    # the plain form runs every chain one per block
    plain = {b["bucket"]: b for b in _ensemble(uneven, "plain").plan()}
    assert sorted(plain) == [4, 5, 6, 7]
    assert all(b["kernel"] == _abi.KERNEL_BLOCK for b in plain.values())
    assert plain[4]["n_chains"] == sum(n <= 64 for n in NS)


def test_uneven_batch_plain_matches_oracle(uneven, port_results):
    ens = _ensemble(uneven, "plain")
    ens.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
    got = ens.positions()
    states = ens.rng_states()
    status = ens.statuses()
    for i, (R, st, pst) in enumerate(port_results):
        assert int(status[i]) == int(pst), i
        assert states[i] == st, i
        assert rel(got[i], R) <= CALL_TOL, (NS[i], rel(got[i], R))
    phys, sims, R0, seeds = uneven
    for i in (0, 6, 11):  # alone (another bucket shape): the same bits
        one = B.Ensemble([phys[i]], [sims[i]], [R0[i]], [(1, -1, seeds[i])], form="plain")
        one.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
        assert np.array_equal(one.positions()[0], got[i]), NS[i]


def test_uneven_batch_mixed_matches_oracle_and_alone(uneven, port_results):
    ens = _ensemble(uneven, "mixed")
    ens.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
    got = ens.positions()
    states = ens.rng_states()
    phys, sims, R0, seeds = uneven
    for i, (R, st, _) in enumerate(port_results):
        assert states[i] == st, i
        assert rel(got[i], R) <= MIXED_TOL, (NS[i], rel(got[i], R))
    # a chain's arithmetic does not depend on its neighbours: bit-identical alone
    for i in range(len(NS)):
        one = B.Ensemble([phys[i]], [sims[i]], [R0[i]], [(1, -1, seeds[i])], form="mixed")
        one.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
        assert np.array_equal(one.positions()[0], got[i]), NS[i]


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_autotune_leaves_state_and_tunes_every_bucket(uneven, port_results, form):
    import torch
    ens = _ensemble(uneven, form)
    R0 = ens.R.clone()
    rng0 = ens.rng.clone()
    plan = ens.autotune(probe_steps=2)
    torch.cuda.synchronize()
    assert torch.equal(ens.R, R0) and torch.equal(ens.rng, rng0)
    for b in plan:
        assert b["tuned"] == 1, b  # block-kernel buckets and (mixed form) team buckets
    ens.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
    got = ens.positions()
    tol = CALL_TOL if form == "plain" else MIXED_TOL
    for i, (R, st, _) in enumerate(port_results):
        assert rel(got[i], R) <= tol, (NS[i], rel(got[i], R))


def test_slot_pool_select_and_refill(uneven, port_results):
    import torch
    phys, sims, R0, seeds = uneven
    pick = [1, 5, 8, 11]  # N = 20, 90, 170, 300
    ctx = Context(0)
    ctx.reserve(n_slots=10, bead_capacity=1200, arena_len=64)
    slots = [7, 2, 9, 4]
    offs = [900, 10, 500, 120]  # scattered, disjoint bead ranges
    ctx.fill_slots(slots, [phys[i] for i in pick], [sims[i] for i in pick], [NS[i] for i in pick], offs)
    dev = torch.device("cuda", 0)
    R = torch.full((1200, 3), 7.0, dtype=torch.float64, device=dev)
    rng = torch.zeros((10, 3), dtype=torch.int32, device=dev)
    for sl, o, i in zip(slots, offs, pick):
        R[o:o + NS[i]] = torch.from_numpy(R0[i]).to(dev)
        rng[sl] = torch.tensor([1, -1, seeds[i]], dtype=torch.int32)
    cache = torch.zeros(3 * 1200, dtype=torch.float64, device=dev)
    valid = torch.zeros(10, dtype=torch.int32, device=dev)
    t0 = torch.zeros(10, dtype=torch.float64, device=dev)
    k = torch.full((10,), STEPS, dtype=torch.int32, device=dev)
    status = torch.zeros(10, dtype=torch.int32, device=dev)
    cnt = torch.zeros((10, 8), dtype=torch.int64, device=dev)

    ctx.select([7, 9])  # two of the four
    ctx.run(R, rng, cache, valid, t0, k, status, cnt, _abi.FORM_PLAIN_FP64, _abi.CACHE_RESET_PER_CALL)
    torch.cuda.synchronize()
    Rh = R.cpu().numpy()
    for sl, o, i in zip(slots, offs, pick):
        if sl in (7, 9):
            assert rel(Rh[o:o + NS[i]], port_results[i][0]) <= CALL_TOL, NS[i]
            assert tuple(rng[sl].tolist()) == port_results[i][1]
        else:
            assert np.array_equal(Rh[o:o + NS[i]], R0[i]), NS[i]  # not selected: untouched
    assert np.all(Rh[:10] == 7.0) and np.all(Rh[1100:] == 7.0)  # free beads untouched

    # refill slot 7 with another chain at another place, then run the rest
    j = 3  # N = 64
    ctx.fill_slots([7], [phys[j]], [sims[j]], [NS[j]], [430])
    R[430:430 + NS[j]] = torch.from_numpy(R0[j]).to(dev)
    rng[7] = torch.tensor([1, -1, seeds[j]], dtype=torch.int32)
    ctx.select([7, 2, 4])
    ctx.run(R, rng, cache, valid, t0, k, status, cnt, _abi.FORM_PLAIN_FP64, _abi.CACHE_RESET_PER_CALL)
    torch.cuda.synchronize()
    Rh = R.cpu().numpy()
    assert rel(Rh[430:430 + NS[j]], port_results[j][0]) <= CALL_TOL
    for o, i in ((10, 5), (120, 11)):  # slots 2 and 4, run for the first time
        assert rel(Rh[o:o + NS[i]], port_results[i][0]) <= CALL_TOL, NS[i]


def test_slot_pool_rejects_bad_selections_and_records(uneven):
    phys, sims, R0, seeds = uneven
    ctx = Context(0)
    ctx.reserve(n_slots=4, bead_capacity=200, arena_len=0)
    ctx.fill_slots([0, 1], [phys[0], phys[1]], [sims[0], sims[1]], [NS[0], NS[1]], [0, 50])
    with pytest.raises(BdcuError, match="twice"):
        ctx.select([0, 0])
    with pytest.raises(BdcuError, match="empty"):
        ctx.select([0, 3])
    with pytest.raises(BdcuError, match="out of range"):
        ctx.select([5])
    with pytest.raises(BdcuError, match="bead_capacity"):
        ctx.fill_slots([2], [phys[1]], [sims[1]], [NS[1]], [190])
    ctx.fill_slots([2], [phys[0]], [sims[0]], [NS[0]], [4])  # overlaps slot 0's beads
    with pytest.raises(BdcuError, match="share beads"):
        ctx.select([0, 2])
    with pytest.raises(BdcuError, match="explicit selection"):
        ctx.select(None)
    ctx.select([0, 1])


def test_graph_capture_replays_an_uneven_run(uneven):
    """A captured bdcu_run (buckets forked onto their own streams and joined)
    replays to the same state as eager calls."""
    import torch
    a = _ensemble(uneven, "plain")
    b = _ensemble(uneven, "plain")
    for e in (a, b):
        e._t.zero_()
        e._k.fill_(2)
    b.plan()  # build the plan (and upload the work lists) before capture
    torch.cuda.synchronize()
    for _ in range(2):
        a.ctx.run(a.R, a.rng, a.cache, a.cache_valid, a._t, a._k, a.status, a.counters, a.form,
                  _abi.CACHE_PERSIST)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b.ctx.run(b.R, b.rng, b.cache, b.cache_valid, b._t, b._k, b.status, b.counters, b.form,
                  _abi.CACHE_PERSIST)
    torch.cuda.synchronize()
    assert np.array_equal(b.positions()[0], uneven[2][0])  # capture ran nothing
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(a.R, b.R) and torch.equal(a.rng, b.rng) and torch.equal(a.cache, b.cache)
    assert torch.equal(a.counters, b.counters)
    del g


# team shapes (warps per chain, beads per thread) compiled into the library
TEAM_SHAPES = [(1, 2), (2, 1), (2, 2), (4, 1), (4, 2), (8, 1), (8, 2)]
BUCKET_BEADS = [64, 128, 256, 512]


@pytest.mark.parametrize("bucket", [0, 1, 2, 3])
def test_every_team_shape_matches_oracle(uneven, port_results, bucket):
    """Each team shape that holds a bucket (up to twice its width) gives the
    reference's RNG stream and stays within MIXED_TOL of the oracle."""
    phys, sims, R0, seeds = uneven
    shapes = [(T, Q) for T, Q in TEAM_SHAPES
              if BUCKET_BEADS[bucket] <= 32 * T * Q <= 2 * BUCKET_BEADS[bucket]]
    assert shapes  # bucket 3 (N <= 512) has one shape, (8, 2)
    for T, Q in shapes:
        ens = _ensemble(uneven, "mixed")
        ens.ctx.set_team_shape(bucket, T, Q)
        b = {x["bucket"]: x for x in ens.plan()}[bucket]
        assert (b["team_warps"], b["team_beads_per_thread"], b["tuned"]) == (T, Q, 1), b
        ens.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
        got = ens.positions()
        states = ens.rng_states()
        for i, (R, st, _) in enumerate(port_results):
            assert states[i] == st, (T, Q, i)
            assert rel(got[i], R) <= MIXED_TOL, (T, Q, NS[i], rel(got[i], R))


def test_team_shape_rejects_a_shape_that_does_not_hold_the_bucket(uneven):
    ens = _ensemble(uneven, "mixed")
    with pytest.raises(BdcuError):
        ens.ctx.set_team_shape(0, 3, 1)
    with pytest.raises(BdcuError):
        ens.ctx.set_team_shape(2, 2, 1)  # compiled, but 64 beads cannot hold bucket 2 (N <= 256)
    ens.ctx.set_team_shape(2, 8, 1)
    ens.ctx.set_team_shape(2, 0, 0)  # back to the default
    assert {x["bucket"]: x for x in ens.plan()}[2]["team_warps"] == 4


def test_single_launch_runs_every_team_chain_in_one_bucket(uneven, port_results):
    ens = _ensemble(uneven, "mixed")
    ens.ctx.set_single_launch(True)
    plan = ens.plan()
    team = [b for b in plan if b["kernel"] == _abi.KERNEL_TEAM]
    assert len(team) == 1 and team[0]["n_chains"] == sum(n <= 512 for n in NS)
    assert team[0]["min_beads"] == min(NS) and team[0]["max_beads"] == max(n for n in NS if n <= 512)
    ens.advance(0.0, STEPS, _abi.CACHE_RESET_PER_CALL)
    got = ens.positions()
    states = ens.rng_states()
    for i, (R, st, _) in enumerate(port_results):
        assert states[i] == st, i
        assert rel(got[i], R) <= MIXED_TOL, (NS[i], rel(got[i], R))
    ens.ctx.set_single_launch(False)
    assert len([b for b in ens.plan() if b["kernel"] == _abi.KERNEL_TEAM]) == 4
