"""The serving queue of the C ABI (bdcu_queue_*), through
bdsim_b200.serving.NativeQueue.

The native queue runs the Python Server's policy; a job's snapshots must
equal, bit for bit, those the Python Server delivers for the same job (and so
those of `simulate`), whether the queue is driven by the caller or by its own
worker thread, alone or among other jobs."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi, workloads
from bdsim_b200.ensemble import Output
from bdsim_b200.params import Spring
from bdsim_b200.serving import Job, NativeQueue, Server

pytestmark = pytest.mark.gpu

# (N, n_traj, n_steps, seed): team-kernel and block-kernel chains in the mixed form
JOBS = [(12, 3, 230, 1), (40, 2, 300, 2), (70, 2, 150, 3), (130, 1, 120, 4)]
POOL = dict(max_chains=64, bead_capacity=4096, arena_capacity=1024)


def _job(N, n_traj, n_steps, seed, flow="shear", rate=1.0):
    p, s = workloads.serving_phys(N, flow, rate)
    return Job(phys=p, sim=s, n_traj=n_traj, seed=seed, n_steps=n_steps, write_every=100)


def _python_server(form, spec):
    srv = Server(device=0, form=form, **POOL)
    js = srv.submit(_job(*spec))
    srv.run_until_idle()
    assert js.state == "done"
    return js


def _collect(events):
    """job id -> {"snaps": [(snapshot, step, time, positions)], "done": event}"""
    out = {}
    for e in events:
        rec = out.setdefault(e["job"], {"snaps": [], "done": None, "rejected": False})
        if e["kind"] == "snapshot":
            rec["snaps"].append((e["snapshot"], e["step"], e["time"], e["positions"]))
        elif e["kind"] == "done":
            rec["done"] = e
        else:
            rec["rejected"] = True
    return out


def _check_against_python(rec, js, spec):
    snaps = sorted(rec["snaps"], key=lambda s: s[0])
    assert [s[0] for s in snaps] == list(range(len(js.steps)))
    assert [s[1] for s in snaps] == js.steps and [s[2] for s in snaps] == js.times
    got = np.stack([s[3] for s in snaps], axis=1)
    assert np.array_equal(got, js.trajectories()), spec
    assert np.array_equal(rec["done"]["status"], js.status)
    assert rec["done"]["step"] == spec[2]
    assert rec["done"]["counters"]["steps"] == spec[1] * spec[2]
    assert rec["done"]["counters"] == js.counters


@pytest.mark.parametrize("form", ["mixed", "plain"])
@pytest.mark.parametrize("worker", [False, True])
def test_native_queue_equals_the_python_server(form, worker):
    want = [_python_server(form, spec) for spec in JOBS]
    q = NativeQueue(device=0, form=form, worker=worker, **POOL)
    ids = [q.submit(_job(*spec), tag=i)[0] for i, spec in enumerate(JOBS[:2])]
    if not worker:
        q.step()
        q.step()
    ids += [q.submit(_job(*spec), tag=2 + i)[0] for i, spec in enumerate(JOBS[2:])]
    assert not q.wait_idle(timeout_s=300)
    recs = _collect(q.events())
    st = q.stats()
    q.close()
    assert st["done"] == 4 and st["rejected"] == 0 and st["queued"] == 0 and st["running"] == 0
    assert st["chain_steps"] == sum(n * k for _, n, k, _ in JOBS)
    for jid, js, spec in zip(ids, want, JOBS):
        _check_against_python(recs[jid], js, spec)


def test_native_queue_final_positions_only_and_simulate(tmp_path):
    spec = JOBS[2]
    q = NativeQueue(device=0, form="plain", **POOL)
    jid, ok = q.submit(_job(*spec), snapshots=False)
    assert ok
    q.wait_idle()
    ev = q.events()
    q.close()
    assert [e["kind"] for e in ev] == ["snapshot", "done"]
    assert ev[0]["step"] == spec[2]
    job = _job(*spec)
    run = B.simulate(job.phys, job.sim, n_traj=job.n_traj, seed=job.seed, n_steps=job.n_steps,
                     output=Output(directory=str(tmp_path / "run"), write_every=100), form="plain")
    for i, tr in enumerate(run):
        assert np.array_equal(tr.positions[-1], ev[0]["positions"][i])


def test_native_queue_admission_and_rejection():
    q = NativeQueue(device=0, form="mixed", max_chains=16, bead_capacity=200, arena_capacity=64, queue_limit=2)
    a, ok_a = q.submit(_job(40, 3, 200, 5))   # 120 beads
    b, ok_b = q.submit(_job(40, 3, 200, 6))   # 120 more: waits for a's beads
    c, ok_c = q.submit(_job(40, 1, 100, 7))   # two jobs queued: rejected
    d, ok_d = q.submit(_job(40, 6, 100, 8))   # 240 beads: larger than the pool
    assert ok_a and ok_b and not ok_c and not ok_d
    q.wait_idle()
    recs = _collect(q.events())
    st = q.stats()
    q.close()
    assert recs[c]["rejected"] and recs[d]["rejected"]
    assert st["done"] == 2 and st["rejected"] == 2
    assert recs[b]["done"]["t_admit"] >= recs[a]["done"]["t_done"]


def test_native_queue_sjf_and_failing_job():
    for policy, first_small in (("sjf", True), ("fifo", False)):
        q = NativeQueue(device=0, form="mixed", policy=policy, max_active_chains=2, **POOL)
        a, _ = q.submit(_job(40, 2, 200, 1))
        q.step()
        b, _ = q.submit(_job(40, 2, 300, 2))
        c, _ = q.submit(_job(12, 2, 100, 3))
        q.wait_idle()
        recs = _collect(q.events())
        q.close()
        tb, tc = recs[b]["done"]["t_admit"], recs[c]["done"]["t_admit"]
        assert (tc < tb) == first_small, policy
    q = NativeQueue(device=0, form="mixed", **POOL)
    good, _ = q.submit(_job(20, 2, 150, 8))
    bad_job = _job(20, 2, 150, 9)
    bad_job.phys.spring.type = Spring.WLCbounded  # sigma > 1: BAD_PARAM
    bad_job.phys.spring.natural_length = 30.0
    bad, _ = q.submit(bad_job)
    q.wait_idle()
    recs = _collect(q.events())
    q.close()
    assert not (recs[good]["done"]["status"] & _abi.ST_FATAL_MASK).any()
    assert (recs[bad]["done"]["status"] & _abi.ST_BAD_PARAM).all()
    js = _python_server("mixed", (20, 2, 150, 8))
    _check_against_python(recs[good], js, (20, 2, 150, 8))
