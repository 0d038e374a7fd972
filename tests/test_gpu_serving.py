"""The serving loop (bdsim_b200.serving.Server): continuous batching of
ensemble jobs of different N, n_traj and n_steps on one GPU.

Each job's snapshots must be the same whether it runs alone or among other
jobs that arrive while it runs, and the same as `simulate` with the same
arguments. Both hold bit for bit: a chain's arithmetic does not depend on the
other chains of its launch (one chain per block or per warp, block
reductions in a fixed order whatever the launch shape)."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi, workloads
from bdsim_b200.ensemble import Output
from bdsim_b200.params import Spring
from bdsim_b200.serving import Job, Server

pytestmark = pytest.mark.gpu

# (N, n_traj, n_steps, seed): warp-kernel and block-kernel chains (mixed form)
JOBS = [(12, 3, 230, 1), (40, 2, 300, 2), (70, 2, 150, 3), (130, 1, 120, 4)]


def _job(N, n_traj, n_steps, seed, flow="shear", rate=1.0):
    p, s = workloads.serving_phys(N, flow, rate)
    return Job(phys=p, sim=s, n_traj=n_traj, seed=seed, n_steps=n_steps, write_every=100)


def _server(form, **kw):
    return Server(device=0, form=form, max_chains=64, bead_capacity=4096, arena_capacity=1024, **kw)


@pytest.mark.parametrize("form", ["mixed", "plain"])
def test_each_job_is_the_same_alone_and_in_the_mix(form):
    alone = []
    for spec in JOBS:
        srv = _server(form)
        js = srv.submit(_job(*spec))
        srv.run_until_idle()
        assert js.state == "done" and not srv.failed(js).any()
        alone.append(js)
    srv = _server(form)
    mix = [srv.submit(_job(*JOBS[0])), srv.submit(_job(*JOBS[1]))]
    srv.step()
    srv.step()
    mix.append(srv.submit(_job(*JOBS[2])))  # arrives while the first two run
    srv.step()
    mix.append(srv.submit(_job(*JOBS[3])))
    srv.run_until_idle()
    assert all(j.state == "done" for j in mix)
    # the later jobs overlapped the earlier ones on the device
    assert mix[2].t_admit < mix[1].t_done and mix[3].t_admit < mix[1].t_done
    for a, m, spec in zip(alone, mix, JOBS):
        assert a.steps == m.steps and a.times == m.times
        assert a.steps[-1] == spec[2] and len(a.steps) == 1 + -(-spec[2] // 100)
        assert np.array_equal(a.trajectories(), m.trajectories()), spec
        assert np.array_equal(a.status, m.status)


def test_served_job_equals_simulate(tmp_path):
    spec = JOBS[2]
    srv = _server("plain")
    js = srv.submit(_job(*spec))
    srv.run_until_idle()
    job = _job(*spec)
    run = B.simulate(job.phys, job.sim, n_traj=job.n_traj, seed=job.seed, n_steps=job.n_steps,
                     output=Output(directory=str(tmp_path / "run"), write_every=100), form="plain")
    got = js.trajectories()
    for i, tr in enumerate(run):
        assert list(tr.step) == js.steps
        assert np.array_equal(tr.positions, got[i])
    # the same job with an output directory: the server spools each chunk as
    # it completes and writes simulate's run directory
    srv = _server("plain")
    job = _job(*spec)
    job.output = Output(directory=str(tmp_path / "served"), write_every=100)
    job.keep_snapshots = False
    js2 = srv.submit(job)
    srv.run_until_idle()
    served = B.read_run(str(tmp_path / "served"))
    assert served.manifest["files"] == run.manifest["files"] and js2.files == run.manifest["files"]
    for a, b in zip(served, run):
        assert np.array_equal(a.step, b.step) and np.array_equal(a.time, b.time)
        assert np.array_equal(a.positions, b.positions)


def test_admission_waits_for_beads_and_rejects_beyond_the_queue():
    srv = Server(device=0, form="mixed", max_chains=16, bead_capacity=200, arena_capacity=64, queue_limit=2)
    a = srv.submit(_job(40, 3, 200, 5))   # 120 beads
    b = srv.submit(_job(40, 3, 200, 6))   # 120 more: must wait for a's beads
    c = srv.submit(_job(40, 1, 100, 7))   # queue holds a (until admitted) and b: rejected
    assert c.state == "rejected"
    srv.run_until_idle()
    assert a.state == b.state == "done"
    assert b.t_admit >= a.t_done
    st = srv.stats()
    assert st["jobs_completed"] == 2 and st["jobs_rejected"] == 1
    assert st["p50_latency_s"] > 0 and st["p99_latency_s"] >= st["p50_latency_s"]


def test_a_failing_job_reports_statuses_and_leaves_the_others():
    srv = _server("mixed")
    good = srv.submit(_job(20, 2, 150, 8))
    bad_job = _job(20, 2, 150, 9)
    bad_job.phys.spring.type = Spring.WLCbounded  # sigma = natural length / sqrtb > 1: BAD_PARAM
    bad_job.phys.spring.natural_length = 30.0
    bad = srv.submit(bad_job)
    srv.run_until_idle()
    assert not srv.failed(good).any()
    assert srv.failed(bad).all() and (bad.status & _abi.ST_BAD_PARAM).all()
    alone = _server("mixed")
    g2 = alone.submit(_job(20, 2, 150, 8))
    alone.run_until_idle()
    assert np.array_equal(g2.trajectories(), good.trajectories())


def test_stream_replay_reports_latency_percentiles():
    jobs = [_job(N, nt, ns, sd) for N, nt, ns, sd in [(16, 2, 200, 11), (60, 1, 300, 12), (90, 2, 100, 13),
                                                       (24, 4, 200, 14), (150, 1, 100, 15)]]
    arrivals = np.array([0.0, 0.05, 0.1, 0.15, 0.2])
    srv = _server("mixed")
    st = srv.run_stream(jobs, arrivals)
    assert st["jobs_completed"] == 5 and st["jobs_rejected"] == 0
    assert st["chain_steps"] == sum(j.n_traj * j.n_steps for j in jobs)
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"]


def test_sjf_admits_the_smallest_queued_job_first():
    # room for two chains: A runs, B (more work) and C (less) wait; when A
    # is done the "sjf" policy admits C first, "fifo" admits B first
    for policy, first in (("sjf", 2), ("fifo", 1)):
        srv = _server("mixed", policy=policy, max_active_chains=2)
        a = srv.submit(_job(40, 2, 200, 1))
        srv.step()
        b = srv.submit(_job(40, 2, 300, 2))
        c = srv.submit(_job(12, 2, 100, 3))
        srv.run_until_idle()
        assert all(j.state == "done" for j in (a, b, c))
        order = sorted((b, c), key=lambda j: j.t_admit)
        assert order[0] is (c if first == 2 else b), policy
