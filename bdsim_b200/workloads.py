"""Seeded synthetic workloads of the benchmark configurations.

bdsim publishes no dataset: its benchmarks integrate seeded synthetic chains.
Each builder here returns the per-chain (PhysParams, SimParams, R0, Rng seed)
of one configuration, generated from a seed so that every run (bench, tests,
CPU baseline) integrates the same chains.

  batched_cheb     4096 x N=50 FENE b=50, h*=0.25 Chebyshev, Gauss EV, shear 1
  uneven_wlc       N ~ U{20..200}, Marko-Siggia WLC Q0 ~ U[10,30], h*=0.2
                   Chebyshev, uniaxial 0.5, LJ (eps 0.3, sigma 1, cutoff 2.5)
  small_cholesky   N=10 FENE-Fraenkel (sigma 1, dQ 2), h*=0.3 Cholesky, shear 1
  stiff_large      N=500 FENE-Fraenkel (sigma 1, dQ 0.1) + bending C=5, SDK EV
                   (sigma 1, uniform phi 0.5), h*=0.3, shear 0.1, dt=1e-4
  serving_jobs     Poisson job stream (N ~ U{10..300}, n_traj ~ U{1..256},
                   n_steps log-uniform [1e3, 1e5], shear or uniaxial at
                   U[0.1, 5], FENE b=100, h*=0.25 Chebyshev, write_every 100)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import flows, initial
from .params import EV, Bending, DelSMethod, PhysParams, SimParams, Spring


def _sim(dt: float) -> SimParams:
    s = SimParams()
    s.dt = dt
    return s


def batched_cheb_phys(n_beads: int = 50):
    """FENE b=50, h*=0.25 Chebyshev+Lanczos, Gauss EV z*=1 d*=0.5, shear 1, dt=1e-3."""
    p = PhysParams()
    p.spring.type = Spring.FENE
    p.spring.sqrtb = 50.0 ** 0.5
    p.hstar = 0.25
    p.hi_method = DelSMethod.Chebyshev
    p.ev.type = EV.Gauss
    p.ev.zstar = 1.0
    p.ev.dstar = 0.5
    p.flow = flows.shear(1.0)
    p.number_of_beads = n_beads
    return p, _sim(1e-3)


def batched_cheb(n_chains: int, first_seed: int = 0, n_beads: int = 50):
    """Chains i = 0..n-1: R0 = gaussian_chain(N, bond_std=1, seed=first+i), Rng(first+i)."""
    p, s = batched_cheb_phys(n_beads)
    R0 = [initial.gaussian_chain(n_beads, bond_std=1.0, seed=first_seed + i) for i in range(n_chains)]
    return [p] * n_chains, [s] * n_chains, R0, [first_seed + i for i in range(n_chains)]


def uneven_wlc(n_chains: int, seed: int = 0, n_min: int = 20, n_max: int = 200, Ns=None):
    """N ~ U{n_min..n_max} (or the given Ns) and Q0 ~ U[10, 30] per chain (seeded), WLC springs
    with sqrtb = Q0, h*=0.2 Chebyshev, uniaxial extension 0.5, LJ EV z*=0.3
    d*=1 cut at 2.5, dt=5e-4. R0: Gaussian bonds (unit variance per
    component), each bond shortened to at most 0.9 Q0."""
    gen = np.random.default_rng(seed)
    Ns = gen.integers(n_min, n_max + 1, size=n_chains) if Ns is None else np.asarray(Ns, dtype=np.int64)
    Q0s = gen.uniform(10.0, 30.0, size=n_chains)
    s = _sim(5e-4)
    phys, R0 = [], []
    flow = flows.uniaxial_extension(0.5)
    for i in range(n_chains):
        p = PhysParams()
        p.spring.type = Spring.WLC
        p.spring.sqrtb = float(Q0s[i])
        p.hstar = 0.2
        p.hi_method = DelSMethod.Chebyshev
        p.ev.type = EV.LJ
        p.ev.zstar = 0.3
        p.ev.dstar = 1.0
        p.ev.max_cutoff = 2.5
        p.flow = flow
        p.number_of_beads = int(Ns[i])
        phys.append(p)
        b = np.random.default_rng(seed * 1000003 + i).normal(size=(int(Ns[i]) - 1, 3))
        L = np.linalg.norm(b, axis=1)
        cap = 0.9 * Q0s[i]
        b[L > cap] *= (cap / L[L > cap])[:, None]
        R = np.zeros((int(Ns[i]), 3))
        R[1:] = np.cumsum(b, axis=0)
        R0.append(R - R.mean(axis=0))
    return phys, [s] * n_chains, R0, [seed * 100003 + i for i in range(n_chains)]


def small_cholesky(n_chains: int = 16, first_seed: int = 0):
    """N=10 FENE-Fraenkel (natural length 1, sqrtb 2), h*=0.3 Cholesky, shear 1, dt=0.01."""
    p = PhysParams()
    p.spring.type = Spring.FENEFraenkel
    p.spring.natural_length = 1.0
    p.spring.sqrtb = 2.0
    p.hstar = 0.3
    p.hi_method = DelSMethod.Cholesky
    p.flow = flows.shear(1.0)
    p.number_of_beads = 10
    s = _sim(0.01)
    R0 = [initial.fene_fraenkel_chain(10, sigma=1.0, dQ=2.0, seed=first_seed + i) for i in range(n_chains)]
    return [p] * n_chains, [s] * n_chains, R0, [first_seed + i for i in range(n_chains)]


def stiff_large_phys(n_beads: int = 500, method=DelSMethod.Chebyshev):
    """FENE-Fraenkel (natural length 1, sqrtb 0.1) + OneMinusCosTheta C=5, SDK EV
    d*=1 with a uniform phi = 0.5 table (the reference's SDK tail weight; its
    SDK core has no epsilon), h*=0.3, shear 0.1, dt=1e-4."""
    p = PhysParams()
    p.spring.type = Spring.FENEFraenkel
    p.spring.natural_length = 1.0
    p.spring.sqrtb = 0.1
    p.bend.type = Bending.OneMinusCosTheta
    p.bend.stiffness = 5.0
    p.ev.type = EV.SDK
    p.ev.dstar = 1.0
    p.ev.phi = np.full(n_beads * n_beads, 0.5)
    p.hstar = 0.3
    p.hi_method = method
    p.flow = flows.shear(0.1)
    p.number_of_beads = n_beads
    return p, _sim(1e-4)


def stiff_large(n_chains: int, first_seed: int = 0, n_beads: int = 500, method=DelSMethod.Chebyshev):
    p, s = stiff_large_phys(n_beads, method)
    R0 = [initial.fene_fraenkel_bending_chain(n_beads, 1.0, 0.1, 5.0, seed=first_seed + i) for i in range(n_chains)]
    return [p] * n_chains, [s] * n_chains, R0, [first_seed + i for i in range(n_chains)]


@dataclass
class JobSpec:
    """One ensemble job of the serving workload."""
    arrival: float  # seconds after the start of the stream
    n_beads: int
    n_traj: int
    n_steps: int
    flow: str  # "shear" | "uniaxial"
    rate: float
    seed: int
    write_every: int = 100
    phys: PhysParams = field(default=None, repr=False)
    sim: SimParams = field(default=None, repr=False)


def serving_phys(n_beads: int, flow: str, rate: float):
    p = PhysParams()
    p.spring.type = Spring.FENE
    p.spring.sqrtb = 10.0
    p.hstar = 0.25
    p.hi_method = DelSMethod.Chebyshev
    p.flow = flows.shear(rate) if flow == "shear" else flows.uniaxial_extension(rate)
    p.number_of_beads = n_beads
    return p, _sim(1e-3)


def serving_jobs(rate: float = 200.0, duration: float = 60.0, seed: int = 0, n_beads=(10, 300),
                 n_traj=(1, 256), n_steps=(1e3, 1e5), flow_rate=(0.1, 5.0), write_every: int = 100):
    """Poisson arrivals at `rate` jobs/s over `duration` s, each job drawn as
    the serving configuration states."""
    gen = np.random.default_rng(seed)
    t, jobs = 0.0, []
    while True:
        t += gen.exponential(1.0 / rate)
        if t >= duration:
            break
        N = int(gen.integers(n_beads[0], n_beads[1] + 1))
        nt = int(gen.integers(n_traj[0], n_traj[1] + 1))
        ns = int(round(math.exp(gen.uniform(math.log(n_steps[0]), math.log(n_steps[1])))))
        fl = "shear" if gen.random() < 0.5 else "uniaxial"
        fr = float(gen.uniform(*flow_rate))
        p, s = serving_phys(N, fl, fr)
        jobs.append(JobSpec(arrival=t, n_beads=N, n_traj=nt, n_steps=ns, flow=fl, rate=fr,
                            seed=int(gen.integers(0, 2 ** 31 - 1)), write_every=write_every, phys=p, sim=s))
    return jobs
