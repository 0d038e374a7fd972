"""Seeded single-call integration cases shared by the golden-fixture generator
and the parity tests: every spring law, EV potential, bending, flow kind,
external-force kind and HI method the integrator supports, at sizes the CPU
oracle finishes in well under a second.
"""
from __future__ import annotations

import os

import numpy as np

from bdsim_b200 import initial
from bdsim_b200.params import DelSMethod, EV, Bending, Flow, PhysParams, SimParams, Spring


def _shear(rate):
    K = np.zeros((3, 3))
    K[0, 1] = rate
    return Flow.constant(K)


def _uniaxial(rate):
    return Flow.constant(np.diag([rate, -rate / 2.0, -rate / 2.0]))


def _sim(dt, n_steps, tol=1e-3, t0=0.0, com=True):
    s = SimParams()
    s.dt = dt
    s.time_start = t0
    s.time_end = t0 + (n_steps - 1) * dt
    s.implicit_loop_tol = tol
    s.update_center_of_mass = com
    return s


def build_case(name):
    """-> (R0 (N,3), PhysParams, SimParams, rng seed)."""
    p = PhysParams()
    if name == "rouse_hook":
        p.spring.type, p.spring.sqrtb = Spring.Hook, 1000.0
        R0 = initial.gaussian_chain(10, seed=11)
        sim = _sim(0.1, 11, tol=1e-6)
        seed = 5
    elif name == "fene_free_shear_gauss":
        p.spring.type, p.spring.sqrtb = Spring.FENE, 50.0 ** 0.5
        p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 1.0, 1.0
        p.flow = _shear(2.0)
        R0 = initial.gaussian_chain(6, seed=3)
        sim = _sim(0.01, 30, tol=1e-6)
        seed = 7
    elif name == "cfg1_ff_cholesky":
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 2.0, 1.0
        p.hstar, p.hi_method = 0.3, DelSMethod.Cholesky
        p.flow = _shear(1.0)
        R0 = initial.fene_fraenkel_chain(10, sigma=1.0, dQ=2.0, seed=0)
        sim = _sim(0.01, 40)
        seed = 0
    elif name == "cfg2_fene_cheb_gauss":
        p.spring.type, p.spring.sqrtb = Spring.FENE, 50.0 ** 0.5
        p.hstar, p.hi_method = 0.25, DelSMethod.Chebyshev
        p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 1.0, 0.5
        p.flow = _shear(1.0)
        R0 = initial.gaussian_chain(50, bond_std=1.0, seed=2)
        sim = _sim(1e-3, 20)
        seed = 2
    elif name == "cfg3_wlc_lj_uniax":
        p.spring.type, p.spring.sqrtb = Spring.WLC, 17.0
        p.hstar, p.hi_method = 0.2, DelSMethod.Chebyshev
        p.ev.type, p.ev.zstar, p.ev.dstar, p.ev.max_cutoff = EV.LJ, 0.3, 1.0, 2.5
        p.flow = _uniaxial(0.5)
        R0 = initial.gaussian_chain(24, seed=4)
        sim = _sim(5e-4, 20)
        seed = 4
    elif name == "cfg4_fene_b100_cheb":
        p.spring.type, p.spring.sqrtb = Spring.FENE, 10.0
        p.hstar, p.hi_method = 0.25, DelSMethod.Chebyshev
        p.flow = _uniaxial(2.0)
        R0 = initial.gaussian_chain(30, seed=6)
        sim = _sim(1e-3, 20)
        seed = 6
    elif name == "cfg5_ff_bend_sdk_cheb":
        N = 20
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 0.1, 1.0
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 5.0
        p.ev.type, p.ev.dstar, p.ev.max_cutoff = EV.SDK, 1.0, 1.5
        p.ev.phi = [0.5] * (N * N)
        p.hstar, p.hi_method = 0.3, DelSMethod.Chebyshev
        p.flow = _shear(0.1)
        R0 = initial.fene_fraenkel_bending_chain(N, 1.0, 0.1, 5.0, seed=8)
        sim = _sim(1e-4, 10)
        seed = 8
    elif name == "cfg5_ff_bend_sdk_cholesky":
        R0, p, sim, seed = build_case("cfg5_ff_bend_sdk_cheb")
        p.hi_method = DelSMethod.Cholesky
        return R0, p, sim, seed
    elif name == "ilc_timeflow_external":
        p.spring.type, p.spring.sqrtb = Spring.ILC, 8.0
        p.flow = Flow.time_varying([0.0, 0.05, 0.2], [np.zeros((3, 3)), _shear(3.0)._k0, _uniaxial(1.0)._k0])
        p.external.add_stretch(0, -1, (0.0, 0.0, 2.5))
        p.external.add_time_varying(3, [0.0, 0.1], [(0.0, 0.0, 0.0), (1.0, -2.0, 0.5)])
        p.hstar, p.hi_method = 0.15, DelSMethod.Chebyshev
        R0 = initial.gaussian_chain(12, seed=9)
        sim = _sim(0.01, 25)
        seed = 9
    elif name == "wlcbounded_free":
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.WLCbounded, 6.0, 1.5
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 1.0
        R0 = initial.fene_fraenkel_chain(8, sigma=2.0, dQ=1.5, seed=10)
        sim = _sim(0.01, 20)
        seed = 10
    elif name == "fraenkel_lj_equil_nocom":
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.Fraenkel, 5.0, 1.0
        p.ev.type, p.ev.zstar, p.ev.dstar = EV.LJ, 0.5, 0.8
        p.ev.contour_dist_for_EV = 2
        p.equilibration = True
        p.hstar, p.hi_method = 0.1, DelSMethod.Cholesky
        R0 = initial.fene_fraenkel_chain_aligned_x(7, sigma=1.0, dQ=0.5, seed=12)
        sim = _sim(0.005, 25, com=False)
        seed = 12
    elif name == "n2_dumbbell_hi":
        p.spring.type, p.spring.sqrtb = Spring.FENE, 5.0
        p.hstar, p.hi_method = 0.2, DelSMethod.Chebyshev
        R0 = np.array([[0.0, 0.0, 0.0], [0.3, -0.8, 0.5]])
        sim = _sim(0.01, 15)
        seed = 13
    elif name == "n3_bend_hi_chol":
        p.spring.type, p.spring.sqrtb = Spring.Hook, 100.0
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 2.0
        p.hstar, p.hi_method = 0.25, DelSMethod.Cholesky
        R0 = initial.gaussian_chain(3, seed=14)
        sim = _sim(0.01, 15)
        seed = 14
    elif name == "cheb_fallback_always":
        # fd_err_max < 0: no Chebyshev series satisfies the fluctuation-
        # dissipation check (its error is >= 0), so every step grows the
        # series to MAXCHEB terms and falls back to the Cholesky factor
        # (src/mobility.cpp:69-81). (With fd_err_max = 0 a series converged to
        # machine precision can still pass, on an error of exactly 0.)
        p.spring.type, p.spring.sqrtb = Spring.FENE, 50.0 ** 0.5
        p.hstar, p.hi_method, p.fd_err_max = 0.25, DelSMethod.Chebyshev, -1.0
        p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 1.0, 0.5
        p.flow = _shear(1.0)
        R0 = initial.gaussian_chain(12, seed=21)
        sim = _sim(1e-3, 8)
        seed = 21
    elif name == "corrector_cap_tol0":
        # implicit_loop_tol = 0: the increment reaches exactly 0 at the fixed
        # point, never below it, so every step runs the corrector to its
        # 100N cap and is accepted as non-converged (src/integrator.cpp:140-163)
        p.spring.type, p.spring.sqrtb = Spring.FENE, 5.0
        p.hstar, p.hi_method = 0.2, DelSMethod.Cholesky
        p.flow = _shear(2.0)
        R0 = initial.gaussian_chain(8, bond_std=0.8, seed=22)
        sim = _sim(1e-3, 5, tol=0.0)
        seed = 22
    elif name == "corrector_cap_stretched":
        # the serving regime: FENE b=100 in uniaxial extension at rate 5 at
        # full extension, where the reference's own corrector stops
        # converging on most steps. R0 is the reference's state after 718
        # steps from gaussian_chain(30, seed=31) with Rng(31) (prestates.npz).
        stretched_physics(p)
        R0 = prestate(name)
        sim = _sim(1e-3, 12, t0=0.718)
        seed = 42
    elif name == "wlcbounded_sigma095":
        # sigma = 0.95: the rtsafe bracket [2 sigma - 1, 1) of
        # solve_wlc_bounded (src/spring.cpp:101-119) is 0.1 wide
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.WLCbounded, 6.0, 5.7
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 1.0
        R0 = initial.fene_fraenkel_chain(8, sigma=5.7, dQ=0.25, seed=24)
        sim = _sim(0.01, 20)
        seed = 24
    else:
        raise KeyError(name)
    p.number_of_beads = len(R0)
    return np.ascontiguousarray(R0, dtype=np.float64), p, sim, seed


def stretched_physics(p):
    """FENE b=100, h*=0.25 Chebyshev, uniaxial extension at rate 5."""
    p.spring.type, p.spring.sqrtb = Spring.FENE, 10.0
    p.hstar, p.hi_method = 0.25, DelSMethod.Chebyshev
    p.flow = _uniaxial(5.0)


PRESTATES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "prestates.npz")


def prestate_spec(name):
    """How the reference produced a family's starting state, with the
    family's own physics: (beads, seed of gaussian_chain and of Rng, steps
    from t = 0, dt)."""
    return {"corrector_cap_stretched": (30, 31, 718, 1e-3)}[name]


def prestate(name):
    """A family's starting positions, made by the reference (see
    prestate_spec) and stored in prestates.npz."""
    with np.load(PRESTATES) as z:
        return z[f"{name}/R0"].copy()


# the families that take the reference's failure branches
FAILURE_CASES = ["cheb_fallback_always", "corrector_cap_tol0", "corrector_cap_stretched", "wlcbounded_sigma095"]

CASES = [
    "rouse_hook", "fene_free_shear_gauss", "cfg1_ff_cholesky", "cfg2_fene_cheb_gauss", "cfg3_wlc_lj_uniax",
    "cfg4_fene_b100_cheb", "cfg5_ff_bend_sdk_cheb", "cfg5_ff_bend_sdk_cholesky", "ilc_timeflow_external",
    "wlcbounded_free", "fraenkel_lj_equil_nocom", "n2_dumbbell_hi", "n3_bend_hi_chol",
] + FAILURE_CASES


def build_large_case(name, N, n_steps=2, seed=0):
    """Full-size chains of the large-chain configurations (a few steps, for
    parity at sizes where D is held in global memory):

    cfg5_*: FENE-Fraenkel springs (sigma=1, dQ=0.1 -> sqrtb 0.1), bending
    stiffness 5, SDK excluded volume (d*=1, uniform phi=0.5, cutoff 1.5),
    h*=0.3 HI by Chebyshev or Cholesky, shear 0.1, dt=1e-4, R0 from
    fene_fraenkel_bending_chain(N, 1.0, 0.1, 5.0, seed).
    cfg3_wlc_lj: Marko-Siggia WLC with Q0=20, LJ EV (0.3, 1.0, cutoff 2.5),
    h*=0.2 Chebyshev, uniaxial 0.5, dt=5e-4, gaussian_chain(N, seed).
    """
    p = PhysParams()
    if name in ("cfg5_cheb", "cfg5_cholesky"):
        p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 0.1, 1.0
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 5.0
        p.ev.type, p.ev.dstar, p.ev.max_cutoff = EV.SDK, 1.0, 1.5
        p.ev.phi = [0.5] * (N * N)
        p.hstar = 0.3
        p.hi_method = DelSMethod.Cholesky if name == "cfg5_cholesky" else DelSMethod.Chebyshev
        p.flow = _shear(0.1)
        R0 = initial.fene_fraenkel_bending_chain(N, 1.0, 0.1, 5.0, seed=seed)
        sim = _sim(1e-4, n_steps)
    elif name == "cfg3_wlc_lj":
        p.spring.type, p.spring.sqrtb = Spring.WLC, 20.0
        p.hstar, p.hi_method = 0.2, DelSMethod.Chebyshev
        p.ev.type, p.ev.zstar, p.ev.dstar, p.ev.max_cutoff = EV.LJ, 0.3, 1.0, 2.5
        p.flow = _uniaxial(0.5)
        R0 = initial.gaussian_chain(N, seed=seed)
        sim = _sim(5e-4, n_steps)
    else:
        raise KeyError(name)
    p.number_of_beads = len(R0)
    return np.ascontiguousarray(R0, dtype=np.float64), p, sim, seed + 1
