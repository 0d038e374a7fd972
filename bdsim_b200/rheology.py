"""Rheological series on the GPU: shear stress, viscosity, and the
variance-reduced viscosity with an equilibrium control chain
(python/bdsim/rheology.py of the bdsim project).

The per-trajectory functions keep the reference's signatures and meaning
(rheology.py:37-105): each takes one chain (R0, phys, sim, rng, sample_times
[, rate]) and integrates it segment by segment through `integrate`, a cold
spectral cache per segment as the reference's per-call integrator.
`run_ensemble` recognises them and runs every trajectory of the ensemble in
one device batch instead, with tau_xy from the device observables (Kramers
stress with the total force, properties.py:38-41); the values are the ones the
per-trajectory functions give chain by chain.

Variance reduction (rheology.py:53-105): each trajectory gets a control chain
with zero flow that starts from the same configuration and consumes the SAME
random stream (a copy of the trajectory's RNG state). The integrator draws
exactly 3N deviates per step whatever the configuration, so the pair stays in
lockstep, and eta_p = -<tau_xy - tau_xy^eq> / rate keeps its mean while most
of the noise cancels at low Weissenberg number. On the device the control
chains are simply the second half of the batch.
"""
from __future__ import annotations

import copy

import numpy as np

from . import properties as props
from ._abi import CACHE_RESET_PER_CALL, ST_FATAL_MASK, count_steps
from .core import IntegratorError, integrate, total_force
from .engine import Ensemble
from .failures import Failure
from .params import Flow, Rng

# column of tau_xy in Ensemble.observables(): [Rg^2, tau_xx, tau_xy, ..., tau_zz]
_TAU_XY = 2


def _tau_xy(R, phys) -> float:
    return float(props.kramers_stress(R, total_force(R, phys))[0, 1])


def stress_series(R0, phys, sim, rng, sample_times, *, form="plain", device=0):
    """tau_xy at each sample time, for one chain (rheology.py:37-46)."""
    from .ensemble import trajectory_samples
    return [_tau_xy(R, phys) for _t, R in trajectory_samples(R0, phys, sim, rng, sample_times, form=form,
                                                               device=device)]


def viscosity_series(R0, phys, sim, rng, sample_times, rate, *, form="plain", device=0):
    """Per-sample polymer viscosity contribution -tau_xy/rate, for one chain
    (rheology.py:49-52)."""
    from .ensemble import trajectory_samples
    return [-_tau_xy(R, phys) / rate for _t, R in trajectory_samples(R0, phys, sim, rng, sample_times, form=form,
                                                                       device=device)]


def control_phys(phys):
    """The control chain's parameters: phys with a zero velocity gradient
    (rheology.py:92-93)."""
    phys_eq = copy.deepcopy(phys)
    phys_eq.flow = type(phys.flow)()  # a default-constructed Flow is zero (either package's)
    return phys_eq


def viscosity_series_vr(R0, phys, sim, rng, sample_times, rate, *, form="plain", device=0):
    """`viscosity_series` with an equilibrium control chain subtracted
    (rheology.py:55-105): -(tau_xy - tau_xy^eq)/rate per sample, the control
    at zero flow from the same R0 on a copy of the same random stream. Both
    stresses use phys's total force (flow does not enter it)."""
    from .ensemble import _segment
    phys_eq = control_phys(phys)
    R_f = np.asarray(R0, dtype=np.float64)
    R_e = R_f.copy()
    rng_e = copy.deepcopy(rng)
    out, t = [], sim.time_start
    for ts in sample_times:
        seg = _segment(sim, t, ts)
        R_f = integrate(R_f, phys, seg, rng, form=form, device=device)
        R_e = integrate(R_e, phys_eq, seg, rng_e, form=form, device=device)
        out.append(-(_tau_xy(R_f, phys) - _tau_xy(R_e, phys)) / rate)
        t = ts
    return out


BATCHED = (stress_series, viscosity_series, viscosity_series_vr)


def batch_layout(fn, phys, R0s, rng_states):
    """Per-chain (phys, R0, rng state) lists of the device batch for fn: the
    trajectories, followed for viscosity_series_vr by their control chains
    (zero flow, a copy of R0, the same RNG state)."""
    n = len(R0s)
    phys_l, R_l, rng_l = [phys] * n, [np.asarray(R, dtype=np.float64) for R in R0s], [tuple(s) for s in rng_states]
    if fn is viscosity_series_vr:
        phys_l = phys_l + [control_phys(phys)] * n
        R_l = R_l + [R.copy() for R in R_l]
        rng_l = rng_l + list(rng_l)
    return phys_l, R_l, rng_l


def series_from_tau(fn, tau, n, rate):
    """One sample of fn's series for each of the n trajectories from the
    batch's tau_xy (control chains in the second half for the VR form)."""
    tau = np.asarray(tau, dtype=np.float64)
    if fn is stress_series:
        return tau[:n].copy()
    if fn is viscosity_series:
        return -tau[:n] / rate
    return -(tau[:n] - tau[n:2 * n]) / rate


def run_batched(fn, phys, sim, n_traj, args, R0s, seed, form, device):
    """run_ensemble's device path for the functions in BATCHED: every
    trajectory (and control chain) advances together, one launch per sample
    segment with a cold spectral cache, and tau_xy comes from the device
    observables. Returns one list per trajectory, or a Failure when the chain
    (or its control) hit a fatal status."""
    from .ensemble import _segment
    sample_times = list(args[0])
    rate = None if fn is stress_series else float(args[1])
    rngs = [Rng(seed + i).state() for i in range(n_traj)]
    phys_l, R_l, rng_l = batch_layout(fn, phys, R0s, rngs)
    ens = Ensemble(phys_l, [sim] * len(phys_l), R_l, rng_l, device=device, form=form)
    per = np.empty((n_traj, len(sample_times)))
    t = sim.time_start
    for s, ts in enumerate(sample_times):
        k = count_steps(_segment(sim, t, ts))
        ens.advance(t, k, CACHE_RESET_PER_CALL)
        per[:, s] = series_from_tau(fn, ens.observables()[:, _TAU_XY], n_traj, rate)
        t = ts
    status = ens.statuses()
    fatal = status[:n_traj] & ST_FATAL_MASK
    if fn is viscosity_series_vr:
        fatal = fatal | (status[n_traj:] & ST_FATAL_MASK)
    return [Failure(i, IntegratorError(int(fatal[i]), i)) if fatal[i] else per[i].tolist() for i in range(n_traj)]


def shear_viscosity_series(phys, sim, rate, n_traj, sample_times, *, variance_reduction=False, **kwargs):
    """(n_traj, n_samples) array of per-sample viscosity contributions
    (rheology.py:111-135). phys.flow must already be a shear flow at rate;
    the other keyword arguments go to run_ensemble."""
    from .ensemble import run_ensemble
    fn = viscosity_series_vr if variance_reduction else viscosity_series
    return np.asarray(run_ensemble(phys, sim, n_traj, fn, args=(list(sample_times), rate), **kwargs))


def equilibrium_stress_series(phys, sim, n_traj, sample_times, **kwargs):
    """(n_traj, n_samples) array of tau_xy(t) at zero flow, for Green-Kubo
    (rheology.py:138-147)."""
    from .ensemble import run_ensemble
    return np.asarray(run_ensemble(phys, sim, n_traj, stress_series, args=(list(sample_times),), **kwargs))


def shear_viscosity(phys, sim, rate, n_traj, sample_times, **kwargs):
    """Steady-state polymer shear viscosity as (mean, stderr): each
    trajectory's samples averaged, then the trajectories treated as
    independent (rheology.py:150-160)."""
    from .ensemble import mean_stderr
    series = shear_viscosity_series(phys, sim, rate, n_traj, sample_times, **kwargs)
    return mean_stderr([float(np.mean(s)) for s in series])
