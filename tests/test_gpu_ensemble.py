"""The run layer (simulate / run_ensemble, backend="cuda") against the
single-chain reference semantics."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200.params import DelSMethod, EV, PhysParams, Rng, SimParams, Spring

pytestmark = pytest.mark.gpu


def _phys():
    p = PhysParams()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 2.0, 1.0
    p.hstar, p.hi_method = 0.3, DelSMethod.Cholesky
    p.flow = B.flows.shear(1.0)
    p.number_of_beads = 10
    return p


def test_simulate_matches_chained_integrate_calls(tmp_path, port):
    p = _phys()
    s = SimParams()
    s.dt = 0.01
    run = B.simulate(p, s, n_traj=3, seed=4, n_steps=25, initial=B.Initial("fene_fraenkel", {"sigma": 1.0, "dQ": 2.0}),
                     output=B.Output(directory=str(tmp_path), write_every=10, write_forces=True))
    assert len(run) == 3
    for i, traj in enumerate(run):
        assert list(traj.step) == [0, 10, 20, 25]
        R = B.fene_fraenkel_chain(10, 1.0, 2.0, seed=4 + i)
        st = (1, -1, 4 + i)
        for k, (step, t, Rs, F) in enumerate(traj):
            if k == 0:
                assert np.array_equal(Rs, R)
                continue
            chunk = step - traj.step[k - 1]
            t0 = s.time_start + traj.step[k - 1] * s.dt
            seg = SimParams()
            seg.dt, seg.time_start, seg.time_end = s.dt, t0, t0 + (chunk - 1) * s.dt
            R, st, status, _ = port.integrate(R, p, seg, st)
            assert np.max(np.abs(Rs - R)) / max(1.0, np.max(np.abs(R))) <= 1e-12
            assert np.max(np.abs(F - port.total_force(R, p))) <= 1e-9 * max(1.0, np.max(np.abs(F)))


def test_run_ensemble_final_state_and_custom_reducer():
    p = _phys()
    s = SimParams()
    s.dt, s.time_end = 0.01, 0.2
    a = B.run_ensemble(p, s, 4, B.final_state, seed=2)
    for i, R in enumerate(a):
        R0 = B.gaussian_chain(10, seed=2 + i)
        want = B.integrate(R0, p, s, Rng(2 + i))
        assert np.max(np.abs(R - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))

    def rg2_final(R0, phys, sim, rng):
        return B.radius_of_gyration_sq(B.integrate(R0, phys, sim, rng))

    b = B.run_ensemble(p, s, 4, rg2_final, seed=2)
    assert np.allclose(b, [B.radius_of_gyration_sq(R) for R in a], rtol=1e-12)
    c = B.run_ensemble(p, s, 2, B.sampled_states, args=([0.05, 0.1, 0.2],), seed=2)
    assert len(c) == 2 and len(c[0]) == 3
    assert np.max(np.abs(c[0][-1] - B.trajectory_samples(B.gaussian_chain(10, seed=2), p, s, Rng(2),
                                                         [0.05, 0.1, 0.2])[-1][1])) <= 1e-12 * 10


def test_failed_trajectories_are_dropped_and_limited():
    from tests.golden.singular import R0_SINGULAR, SINGULAR_HSTAR  # noqa: F401
    p = _phys()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.WLCbounded, 2.0, 3.0  # sigma > 1
    s = SimParams()
    s.dt, s.time_end = 0.01, 0.05
    with pytest.raises(RuntimeError):
        B.run_ensemble(p, s, 3, B.final_state)


def test_device_observables_match_numpy():
    # Rg^2 and the Kramers stress of uneven chains, on the device vs numpy
    from bdsim_b200 import workloads
    phys, sims, R0s, seeds = workloads.uneven_wlc(24, seed=3, n_min=2, n_max=90)
    ens = B.Ensemble(phys, sims, R0s, [(1, -1, s) for s in seeds], form="mixed")
    ens.advance(0.0, 20)
    o = ens.observables()
    Rs, Fs = ens.positions(), ens.total_force()
    for i, (R, F) in enumerate(zip(Rs, Fs)):
        X = R - R.mean(axis=0)
        assert abs(o[i, 0] - np.sum(X * X) / len(R)) <= 1e-12 * max(1.0, o[i, 0])
        tau = X.T @ F
        assert np.max(np.abs(o[i, 1:].reshape(3, 3) - tau)) <= 1e-11 * max(1.0, np.max(np.abs(tau)))
