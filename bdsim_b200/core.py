"""The compiled-core functions of bdsim (bindings/module.cpp:45-76, 308-316),
computed on the GPU.

`integrate(R, phys, sim, rng)` is the drop-in for `_bdsim.integrate`: the same
arguments, R copied in and a new (N, 3) array returned, `rng` advanced in
place, and an exception when the integrator gives up on the chain (the
reference raises on a non-positive-definite diffusion tensor and aborts on
rtsafe / WLCbounded / ExactSqrt failures; here those are status bits turned
into `IntegratorError`). `integrate_many` is the batched form.
"""
from __future__ import annotations

import copy
import threading

import numpy as np

from . import _abi
from ._abi import ST_FATAL_MASK, STATUS_NAMES
from .engine import Context, form_code
from .params import PhysParams, SimParams, rng_state, set_rng_state

_local = threading.local()


class IntegratorError(RuntimeError):
    """The integrator gave up on a chain (status bits in `.status`)."""

    def __init__(self, status: int, index: int = 0):
        self.status = int(status)
        self.index = index
        names = [msg for bit, msg in STATUS_NAMES.items() if status & bit and bit & ST_FATAL_MASK]
        super().__init__("; ".join(names) or f"status {status}")


def _ctx(device: int = 0) -> Context:
    cache = getattr(_local, "ctx", None)
    if cache is None:
        cache = _local.ctx = {}
    if device not in cache:
        cache[device] = Context(device)
    return cache[device]


def integrate_many(Rs, phys, sims, rngs, *, form="plain", device: int = 0, raise_on_failure=False):
    """Integrate many chains, chain i over sims[i]'s [time_start, time_end]
    with a cold spectral cache (one reference integrate call each).

    phys/sims: one object for all chains, or a list. rngs: Rng objects,
    advanced in place. Returns (list of new (N,3) arrays, status array,
    counters list)."""
    n = len(Rs)
    phys_l = phys if isinstance(phys, (list, tuple)) else [phys] * n
    sims_l = sims if isinstance(sims, (list, tuple)) else [sims] * n
    Ns = [len(r) for r in Rs]
    R = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64).reshape(-1, 3) for r in Rs]))
    rng = np.ascontiguousarray(np.array([rng_state(g) for g in rngs], dtype=np.int32).reshape(n, 3))
    ctx = _ctx(device)
    ctx.set_chains(phys_l, sims_l, Ns)
    status, counters = ctx.integrate_host(R, rng, form_code(form))
    for g, st in zip(rngs, rng):
        set_rng_state(g, st)
    off = np.concatenate([[0], np.cumsum(Ns)])
    out = [R[off[i]:off[i + 1]].copy() for i in range(n)]
    if raise_on_failure:
        bad = np.nonzero(status & ST_FATAL_MASK)[0]
        if bad.size:
            raise IntegratorError(int(status[bad[0]]), int(bad[0]))
    return out, status, counters


def integrate(R, phys: PhysParams, sim: SimParams, rng, *, form="plain", device: int = 0):
    """Integrate one chain; returns the evolved (N,3) positions (bindings/module.cpp:45-50)."""
    R = np.ascontiguousarray(R, dtype=np.float64)
    if R.ndim != 2 or R.shape[1] != 3:
        raise ValueError("R must be an (N, 3) float64 array")
    out, status, _ = integrate_many([R], phys, sim, [rng], form=form, device=device)
    if status[0] & ST_FATAL_MASK:
        raise IntegratorError(int(status[0]))
    return out[0]


def forces_many(Rs, phys, which: int, t: float = 0.0, *, device: int = 0):
    """Force components (`which` ORs _abi.F_* bits) per chain, FP64 on the GPU."""
    import torch
    n = len(Rs)
    phys_l = phys if isinstance(phys, (list, tuple)) else [phys] * n
    Ns = [len(r) for r in Rs]
    R = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64).reshape(-1, 3) for r in Rs]))
    ctx = _ctx(device)
    ctx.set_chains(phys_l, [SimParams()] * n, Ns)
    Rd = torch.from_numpy(R).to(torch.device("cuda", device))
    Fd = torch.empty_like(Rd)
    ctx.forces(Rd, Fd, which, t)
    F = Fd.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(Ns)])
    return [F[off[i]:off[i + 1]].copy() for i in range(n)]


def total_force_many(Rs, phys, *, device: int = 0):
    """Spring + EV + bending force per chain (no external)."""
    return forces_many(Rs, phys, _abi.F_SPRING | _abi.F_EV | _abi.F_BEND, device=device)


def total_force(R, phys: PhysParams, *, device: int = 0):
    """Intramolecular force (spring + bending + EV), excluding external forces
    (bindings/module.cpp:67-76)."""
    return total_force_many([np.asarray(R, dtype=np.float64)], phys, device=device)[0]


def spring_force(R, spring, *, device: int = 0):
    """Net spring force per bead (bindings/module.cpp:52-55)."""
    p = PhysParams()
    p.spring = copy.deepcopy(spring)
    return forces_many([np.asarray(R, dtype=np.float64)], p, _abi.F_SPRING, device=device)[0]


def bending_force(R, bend, *, device: int = 0):
    """Bending force per bead (bindings/module.cpp:56-60)."""
    p = PhysParams()
    p.bend = copy.deepcopy(bend)
    return forces_many([np.asarray(R, dtype=np.float64)], p, _abi.F_BEND, device=device)[0]


def ev_force(R, ev, equilibration: bool = False, *, device: int = 0):
    """Excluded-volume force per bead (bindings/module.cpp:61-66)."""
    p = PhysParams()
    p.ev = copy.deepcopy(ev)
    p.equilibration = bool(equilibration)
    return forces_many([np.asarray(R, dtype=np.float64)], p, _abi.F_EV, device=device)[0]


def external_force(phys: PhysParams, nbeads: int, t: float = 0.0, *, device: int = 0):
    """Applied external force on each bead at time t (bindings/module.cpp:128-132)."""
    R = np.zeros((int(nbeads), 3))
    return forces_many([R], phys, _abi.F_EXTERNAL, t, device=device)[0]
