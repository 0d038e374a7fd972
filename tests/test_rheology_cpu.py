"""Host logic of the rheology series (python/bdsim/rheology.py): the control
chains of the variance-reduced viscosity, the per-sample arithmetic, and the
lockstep of a flow chain and its control on the oracle."""
import numpy as np

import bdsim_b200 as B
from bdsim_b200 import rheology as RH
from bdsim_b200.ensemble import _segment
from bdsim_b200.params import DelSMethod, PhysParams, SimParams, Spring


def _phys(rate=0.5):
    p = PhysParams()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 2.0, 1.0
    p.hstar, p.hi_method = 0.3, DelSMethod.Cholesky
    p.flow = B.flows.shear(rate)
    p.number_of_beads = 10
    return p


def test_control_phys_zeroes_only_the_flow():
    p = _phys()
    q = RH.control_phys(p)
    assert np.all(q.flow._k0 == 0.0)
    assert p.flow._k0[0, 1] == 0.5  # the original is untouched
    assert q.hstar == p.hstar and q.spring.sqrtb == p.spring.sqrtb and q.hi_method == p.hi_method


def test_batch_layout_pairs_each_trajectory_with_its_control():
    p = _phys()
    R0s = [B.fene_fraenkel_chain(10, 1.0, 2.0, seed=s) for s in range(3)]
    rngs = [B.Rng(7 + i).state() for i in range(3)]
    phys_l, R_l, rng_l = RH.batch_layout(RH.viscosity_series_vr, p, R0s, rngs)
    assert len(phys_l) == len(R_l) == len(rng_l) == 6
    for i in range(3):
        assert phys_l[i] is p
        assert np.all(phys_l[3 + i].flow._k0 == 0.0)
        assert np.array_equal(R_l[i], R0s[i]) and np.array_equal(R_l[3 + i], R0s[i])
        assert R_l[3 + i] is not R_l[i]
        assert rng_l[i] == rng_l[3 + i] == rngs[i]
    for fn in (RH.stress_series, RH.viscosity_series):
        phys_l, R_l, rng_l = RH.batch_layout(fn, p, R0s, rngs)
        assert len(phys_l) == 3 and rng_l == [tuple(s) for s in rngs]


def test_series_from_tau():
    tau = np.array([1.0, -2.0, 3.0, 0.5, -1.0, 2.0])
    assert np.array_equal(RH.series_from_tau(RH.stress_series, tau[:3], 3, None), tau[:3])
    assert np.allclose(RH.series_from_tau(RH.viscosity_series, tau[:3], 3, 2.0), -tau[:3] / 2.0)
    assert np.allclose(RH.series_from_tau(RH.viscosity_series_vr, tau, 3, 2.0), -(tau[:3] - tau[3:]) / 2.0)


def test_run_ensemble_batches_the_rheology_series():
    assert RH.BATCHED == (RH.stress_series, RH.viscosity_series, RH.viscosity_series_vr)
    assert B.rheology is RH


def test_flow_and_control_chains_stay_in_lockstep_on_the_oracle(port):
    """The pair consumes one random stream: exactly 3N draws per step whatever
    the configuration (rheology.py:67-70), so the two RNG states agree after
    every segment although the configurations differ."""
    p = _phys(rate=2.0)
    q = RH.control_phys(p)
    s = SimParams()
    s.dt = 0.01
    R_f = B.fene_fraenkel_chain(10, 1.0, 2.0, seed=3)
    R_e = R_f.copy()
    st_f = st_e = (1, -1, 11)
    t = s.time_start
    for ts in (0.05, 0.1, 0.2):
        seg = _segment(s, t, ts)
        R_f, st_f, status_f, _ = port.integrate(R_f, p, seg, st_f)
        R_e, st_e, status_e, _ = port.integrate(R_e, q, seg, st_e)
        assert status_f == 0 and status_e == 0
        assert st_f == st_e
        t = ts
    assert not np.array_equal(R_f, R_e)  # the flow moved one chain and not the other
