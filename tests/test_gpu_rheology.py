"""Rheology series through run_ensemble (backend="cuda", batched on the
device) against the oracle chain by chain, and against the per-trajectory
functions (python/bdsim/rheology.py:37-105)."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import rheology as RH
from bdsim_b200.ensemble import _segment
from bdsim_b200.params import DelSMethod, PhysParams, SimParams, Spring

pytestmark = pytest.mark.gpu

N, RATE, SEED = 10, 0.5, 2
TIMES = [0.05, 0.1, 0.15, 0.3]
INIT = B.Initial("fene_fraenkel", {"sigma": 1.0, "dQ": 2.0})


def _phys(method=DelSMethod.Cholesky):
    p = PhysParams()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 2.0, 1.0
    p.hstar, p.hi_method = 0.3, method
    p.flow = B.flows.shear(RATE)
    p.number_of_beads = N
    return p


def _sim():
    s = SimParams()
    s.dt = 0.01
    return s


def _tau(port, R, p):
    return float(B.kramers_stress(R, port.total_force(R, p))[0, 1])


def _oracle_vr(port, p, s, i):
    """viscosity_series_vr of trajectory i on the oracle, with the flow and
    control stresses kept apart."""
    q = RH.control_phys(p)
    R_f = B.fene_fraenkel_chain(N, 1.0, 2.0, seed=SEED + i)
    R_e = R_f.copy()
    st_f = st_e = (1, -1, SEED + i)
    out, t = [], s.time_start
    for ts in TIMES:
        seg = _segment(s, t, ts)
        R_f, st_f, _, _ = port.integrate(R_f, p, seg, st_f)
        R_e, st_e, _, _ = port.integrate(R_e, q, seg, st_e)
        out.append((_tau(port, R_f, p), _tau(port, R_e, p)))
        t = ts
    return out


def test_vr_viscosity_batched_matches_oracle(port):
    p, s = _phys(), _sim()
    got = np.asarray(B.run_ensemble(p, s, 3, RH.viscosity_series_vr, args=(TIMES, RATE), seed=SEED, initial=INIT))
    assert got.shape == (3, len(TIMES))
    for i in range(3):
        for k, (tf, te) in enumerate(_oracle_vr(port, p, s, i)):
            want = -(tf - te) / RATE
            # plain form: <= 1e-12 per step; the stresses are summed in another order
            assert abs(got[i, k] - want) <= 1e-9 * (abs(tf) + abs(te)) / RATE + 1e-14, (i, k, got[i, k], want)


def test_stress_and_viscosity_series_batched_match_oracle(port):
    p, s = _phys(), _sim()
    tau = np.asarray(B.run_ensemble(p, s, 2, RH.stress_series, args=(TIMES,), seed=SEED, initial=INIT))
    eta = np.asarray(B.run_ensemble(p, s, 2, RH.viscosity_series, args=(TIMES, RATE), seed=SEED, initial=INIT))
    for i in range(2):
        want = [tf for tf, _te in _oracle_vr(port, p, s, i)]
        assert np.allclose(tau[i], want, rtol=1e-9, atol=1e-12)
        assert np.allclose(eta[i], -np.asarray(want) / RATE, rtol=1e-9, atol=1e-12)


def test_per_trajectory_functions_match_batched():
    p, s = _phys(), _sim()
    batched = np.asarray(B.run_ensemble(p, s, 2, RH.viscosity_series_vr, args=(TIMES, RATE), seed=SEED,
                                        initial=INIT))
    for i in range(2):
        R0 = B.fene_fraenkel_chain(N, 1.0, 2.0, seed=SEED + i)
        one = RH.viscosity_series_vr(R0, p, s, B.Rng(SEED + i), TIMES, RATE)
        assert np.allclose(one, batched[i], rtol=1e-9, atol=1e-12)


def test_shear_viscosity_wrappers_mixed_form():
    """The wrappers, on the FP32-mixed form with Chebyshev HI: finite series of
    the requested shape and a finite (mean, stderr)."""
    p, s = _phys(DelSMethod.Chebyshev), _sim()
    series = RH.shear_viscosity_series(p, s, RATE, 8, TIMES, variance_reduction=True, seed=SEED, initial=INIT,
                                       form="mixed")
    assert series.shape == (8, len(TIMES)) and np.all(np.isfinite(series))
    mean, err = RH.shear_viscosity(p, s, RATE, 8, TIMES, seed=SEED, initial=INIT, form="mixed")
    assert np.isfinite(mean) and np.isfinite(err)
    eq = RH.equilibrium_stress_series(RH.control_phys(p), s, 4, TIMES, seed=SEED, initial=INIT, form="mixed")
    assert eq.shape == (4, len(TIMES)) and np.all(np.isfinite(eq))


def test_variance_reduction_pays_at_low_shear():
    """At low Weissenberg number the control chain removes most of the
    stress noise (rheology.py:72-80): over the same trajectories and seeds the
    variance-reduced series scatters far less than the direct one, with a
    compatible mean."""
    rate = 0.02
    p, s = _phys(), _sim()
    p.flow = B.flows.shear(rate)
    times = [0.5 * (k + 1) for k in range(4)]
    direct = np.asarray(B.run_ensemble(p, s, 64, RH.viscosity_series, args=(times, rate), seed=SEED,
                                       initial=INIT))
    vr = np.asarray(B.run_ensemble(p, s, 64, RH.viscosity_series_vr, args=(times, rate), seed=SEED,
                                   initial=INIT))
    assert direct.shape == vr.shape == (64, 4)
    assert vr.var() * 10 < direct.var()
    # trajectories are independent, samples along one are not: compare means
    # of the per-trajectory averages
    td, tv = direct.mean(axis=1), vr.mean(axis=1)
    e_d, e_v = td.std(ddof=1) / np.sqrt(len(td)), tv.std(ddof=1) / np.sqrt(len(tv))
    assert abs(td.mean() - tv.mean()) <= 4 * np.hypot(e_d, e_v)
