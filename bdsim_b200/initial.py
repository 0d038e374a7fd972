"""Initial chain configurations, numerically identical to bdsim's generators
(python/bdsim/initial.py of the bdsim project) for the same seed.

Identity matters: `simulate(..., seed=s)` must start trajectory i from the
same R0 as the reference does, so each constructor makes the same numpy
Generator draws in the same order (PCG64 via default_rng(seed)).
"""
from __future__ import annotations

import numpy as np


def gaussian_chain(n: int, bond_std: float = 1.0, seed=None) -> np.ndarray:
    """Random walk of n beads with isotropic Gaussian bonds, centre of mass at
    the origin (initial.py:5-16)."""
    gen = np.random.default_rng(seed)
    steps = gen.normal(scale=bond_std, size=(n - 1, 3))
    R = np.zeros((n, 3))
    R[1:] = np.cumsum(steps, axis=0)
    return R - R.mean(axis=0)


def inverse_cdf_sample(x, pdf, u):
    """Samples with density proportional to pdf on grid x for uniforms u, by
    the trapezoidal CDF (initial.py:98-103)."""
    seg = 0.5 * (pdf[:-1] + pdf[1:]) * np.diff(x)
    cdf = np.concatenate(([0.0], np.cumsum(seg)))
    cdf /= cdf[-1]
    return np.interp(u, cdf, x)


def _fene_fraenkel_lengths(n_bonds, sigma, dQ, gen, nsteps=10000):
    """Bond lengths from psi(Q) ~ Q^2 (1 - (Q-sigma)^2/dQ^2)^(dQ^2/2) on
    [max(0, sigma-dQ), sigma+dQ] (initial.py:29-41)."""
    alpha = dQ * dQ
    Q = np.linspace(max(0.0, sigma - dQ), sigma + dQ, nsteps)
    Q[0] += 1e-7
    Q[-1] -= 1e-7
    psi = Q * Q * (1.0 - (Q - sigma) ** 2 / alpha) ** (alpha / 2.0)
    seg = 0.5 * (psi[:-1] + psi[1:]) * np.diff(Q)
    cdf = np.concatenate(([0.0], np.cumsum(seg)))
    cdf /= cdf[-1]
    return np.interp(gen.random(n_bonds), cdf, Q)


def _unit_vectors_marsaglia(n, gen):
    """n isotropic unit vectors by Marsaglia's rejection method, drawn in
    batches of 2*(remaining)+8 pairs (initial.py:44-60)."""
    out = np.empty((n, 3))
    done = 0
    while done < n:
        pairs = gen.uniform(-1.0, 1.0, size=(2 * (n - done) + 8, 2))
        s = pairs[:, 0] ** 2 + pairs[:, 1] ** 2
        ok = pairs[s < 1.0]
        sk = ok[:, 0] ** 2 + ok[:, 1] ** 2
        k = min(len(ok), n - done)
        w = np.sqrt(1.0 - sk[:k])
        out[done:done + k, 0] = 2.0 * ok[:k, 0] * w
        out[done:done + k, 1] = 2.0 * ok[:k, 1] * w
        out[done:done + k, 2] = 1.0 - 2.0 * sk[:k]
        done += k
    return out


def fene_fraenkel_chain(n: int, sigma: float, dQ: float, seed=None) -> np.ndarray:
    """FENE-Fraenkel equilibrium bond lengths, random directions, bead 0 at the
    origin (initial.py:63-74)."""
    gen = np.random.default_rng(seed)
    lengths = _fene_fraenkel_lengths(n - 1, sigma, dQ, gen)
    bonds = _unit_vectors_marsaglia(n - 1, gen) * lengths[:, None]
    R = np.zeros((n, 3))
    R[1:] = np.cumsum(bonds, axis=0)
    return R


def fene_fraenkel_chain_aligned_x(n: int, sigma: float, dQ: float, seed=None) -> np.ndarray:
    """FENE-Fraenkel bond lengths, all bonds along x (initial.py:77-83)."""
    gen = np.random.default_rng(seed)
    lengths = _fene_fraenkel_lengths(n - 1, sigma, dQ, gen)
    R = np.zeros((n, 3))
    R[1:, 0] = np.cumsum(lengths)
    return R


def isotropic_directions(n, gen):
    """n isotropic unit vectors from uniform cos(theta) and azimuth (initial.py:106-111)."""
    c = gen.uniform(-1.0, 1.0, n)
    s = np.sqrt(1.0 - c ** 2)
    phi = gen.uniform(0.0, 2.0 * np.pi, n)
    return np.stack([s * np.cos(phi), s * np.sin(phi), c], axis=1)


def one_minus_cos_theta_angles(n, stiffness, gen):
    """Bond angles for the C(1-cos theta) potential, cos(theta) ~ exp(C u) on
    [-1, 1], sampled analytically (initial.py:114-125)."""
    C = stiffness
    if C == 0.0:
        return np.arccos(gen.uniform(-1.0, 1.0, n))
    y = gen.random(n)
    u = np.log(np.exp(-C) + y * (np.exp(C) - np.exp(-C))) / C
    return np.arccos(np.clip(u, -1.0, 1.0))


def _rotation_taking_z_to(u):
    """Rodrigues rotation with R @ e_z == u (initial.py:128-138)."""
    c = u[2]
    if c > 1.0 - 1e-12:
        return np.eye(3)
    if c < -1.0 + 1e-12:
        return np.diag([1.0, -1.0, -1.0])
    v = np.array([-u[1], u[0], 0.0])
    vx = np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])
    return np.eye(3) + vx + vx @ vx * ((1.0 - c) / (v @ v))


def equilibrium_chain(lengths, angles=None, seed=None):
    """Chain from bond lengths (n-1) and included angles (n-2; None => right
    angles), random azimuths, bead 0 at the origin (initial.py:141-164)."""
    lengths = np.asarray(lengths, dtype=float)
    nb = len(lengths)
    gen = np.random.default_rng(seed)
    u = np.empty((nb, 3))
    u[0] = isotropic_directions(1, gen)[0]
    for i in range(1, nb):
        theta = np.pi / 2 if angles is None else float(angles[i - 1])
        az = gen.uniform(0.0, 2.0 * np.pi)
        local = np.array([np.sin(theta) * np.cos(az), np.sin(theta) * np.sin(az), np.cos(theta)])
        u[i] = _rotation_taking_z_to(u[i - 1]) @ local
    R = np.zeros((nb + 1, 3))
    R[1:] = np.cumsum(u * lengths[:, None], axis=0)
    return R


def fene_fraenkel_bending_chain(n, sigma, dQ, stiffness, seed=None):
    """FENE-Fraenkel lengths plus OneMinusCosTheta angles (initial.py:167-173);
    the assembly draws from a fresh generator with the same seed."""
    gen = np.random.default_rng(seed)
    lengths = _fene_fraenkel_lengths(n - 1, sigma, dQ, gen)
    angles = one_minus_cos_theta_angles(n - 2, stiffness, gen) if n > 2 else None
    return equilibrium_chain(lengths, angles, seed=seed)
