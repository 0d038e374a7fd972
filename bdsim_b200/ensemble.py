"""The run layer of bdsim (python/bdsim/ensemble.py of the bdsim project) with
backend="cuda": every trajectory of an ensemble is a chain of one device
batch, advanced on the GPU chunk by chunk.

Semantics kept from the reference:
  * trajectory i is seeded seed+i and starts from INITIALIZERS[method](N, seed+i)
    (ensemble.py:157-161, 197-199);
  * a chunk of k steps is one integrate call over [t0, t0+(k-1)dt], and each
    call starts the spectral (Lanczos) cache cold (ensemble.py:106-123);
  * snapshots at step 0, every write_every steps and the last step;
  * a trajectory whose integration fails becomes a Failure, dropped and
    reported, with MAX_FAILED_FRACTION enforced (ensemble.py:230, 244-284).
"""
from __future__ import annotations

import os
import sys
import threading
from dataclasses import dataclass, field

import numpy as np

from . import rheology, storage
from ._abi import CACHE_PERSIST, CACHE_RESET_PER_CALL, ST_FATAL_MASK, count_steps
from .core import IntegratorError, integrate
from .engine import Ensemble
from .initial import (fene_fraenkel_bending_chain, fene_fraenkel_chain, fene_fraenkel_chain_aligned_x,
                      gaussian_chain)
from .failures import Failure
from .params import PhysParams, Rng, SimParams


def _init_gaussian(n, seed, kw): return gaussian_chain(n, seed=seed, **kw)
def _init_fene_fraenkel(n, seed, kw): return fene_fraenkel_chain(n, seed=seed, **kw)
def _init_fene_fraenkel_x(n, seed, kw): return fene_fraenkel_chain_aligned_x(n, seed=seed, **kw)
def _init_fene_fraenkel_bending(n, seed, kw): return fene_fraenkel_bending_chain(n, seed=seed, **kw)


INITIALIZERS = {
    "gaussian": _init_gaussian,
    "fene_fraenkel": _init_fene_fraenkel,
    "fene_fraenkel_x": _init_fene_fraenkel_x,
    "fene_fraenkel_bending": _init_fene_fraenkel_bending,
}

MAX_FAILED_FRACTION = 0.1


@dataclass
class Initial:
    """Initial-configuration method (a key of INITIALIZERS) and its kwargs."""
    method: str = "gaussian"
    kwargs: dict = field(default_factory=dict)


@dataclass
class Output:
    """Run directory, snapshot interval (0 => start and end only), forces flag."""
    directory: str = None
    write_every: int = 0
    write_forces: bool = False
    compression: str = "gzip"


def _segment(sim: SimParams, t0: float, t1: float) -> SimParams:
    s = SimParams()
    s.dt = sim.dt
    s.implicit_loop_tol = sim.implicit_loop_tol
    s.update_center_of_mass = sim.update_center_of_mass
    s.time_start = t0
    s.time_end = t1
    return s


def n_steps_of(sim: SimParams) -> int:
    """Integrator steps implied by sim's time span and dt (ensemble.py:95-97)."""
    return int(round((sim.time_end - sim.time_start) / sim.dt))


def mean_stderr(values):
    arr = np.asarray(values, dtype=float)
    n = arr.size
    mean = float(arr.mean())
    stderr = float(arr.std(ddof=1) / np.sqrt(n)) if n > 1 else float("nan")
    return mean, stderr


def _phys_summary(phys: PhysParams) -> dict:
    return {"n_beads": int(phys.number_of_beads), "spring_type": str(phys.spring.type),
            "sqrtb": float(phys.spring.sqrtb), "natural_length": float(phys.spring.natural_length),
            "hstar": float(phys.hstar), "hi_method": str(phys.hi_method)}


def _drop_failures(results, what, max_fraction=None):
    ok = [r for r in results if not isinstance(r, Failure)]
    bad = [r for r in results if isinstance(r, Failure)]
    if not bad:
        return ok, bad
    n = len(results)
    frac = len(bad) / n
    seen, lines = set(), []
    for f in bad:
        key = f.message.split("(")[0]
        if key not in seen:
            seen.add(key)
            lines.append(f"    trajectory {f.index}: {f.message.splitlines()[0]}")
    print(f"bdsim: {len(bad)} of {n} {what} failed and were dropped ({100 * frac:.0f}%). Distinct causes:",
          file=sys.stderr)
    for line in lines[:3]:
        print(line, file=sys.stderr)
    limit = MAX_FAILED_FRACTION if max_fraction is None else max_fraction
    if frac > limit:
        raise RuntimeError(f"{len(bad)} of {n} {what} failed ({100 * frac:.0f}%), above the {100 * limit:.0f}% "
                           "limit. Reduce dt or tighten implicit_loop_tol, or raise max_failed_fraction.")
    if not ok:
        raise RuntimeError(f"every one of the {n} {what} failed")
    return ok, bad


def _check_backend(backend):
    if backend != "cuda":
        raise ValueError(f"bdsim_b200 runs ensembles on the GPU: use backend='cuda' (got {backend!r})")


def _start(phys, sim, n_traj, seed, initial, form, device):
    initial = initial or Initial()
    R0s = [INITIALIZERS[initial.method](phys.number_of_beads, seed + i, dict(initial.kwargs)) for i in range(n_traj)]
    rngs = [Rng(seed + i).state() for i in range(n_traj)]
    return Ensemble([phys] * n_traj, [sim] * n_traj, R0s, rngs, device=device, form=form), R0s


def simulate(phys: PhysParams, sim: SimParams, *, n_traj: int = 1, seed: int = 0, n_steps: int = None,
             initial: Initial = None, output: Output = None, backend: str = "cuda", n_workers: int = None,
             on_error: str = "skip", max_failed_fraction: float = None, form="plain", device: int = 0):
    """Run n_traj chains on the GPU and write their snapshots (ensemble.py:179-227)."""
    _check_backend(backend)
    initial = initial or Initial()
    output = output or Output()
    if output.directory is None:
        raise ValueError("output.directory must be set (the run folder to write into)")
    n_steps = int(n_steps) if n_steps is not None else n_steps_of(sim)
    os.makedirs(output.directory, exist_ok=True)
    ens, R0s = _start(phys, sim, n_traj, seed, initial, form, device)
    torch = ens.torch
    w = output.write_every if (output.write_every and output.write_every > 0) else n_steps
    n_snap = 1 + (n_steps + w - 1) // w
    # each snapshot: device -> pinned host copy on the launch stream (after the
    # chunk's kernel, before the next), then spooled to disk by the writer's
    # thread while the device runs the next chunk; two pinned buffers rotate
    writer = storage.RunWriter(output.directory, ens.offsets, n_snap, bool(output.write_forces))
    total = int(ens.offsets[-1])
    pin_R = [torch.empty((total, 3), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    pin_F = [torch.empty((total, 3), dtype=torch.float64, pin_memory=True) for _ in range(2)] \
        if output.write_forces else None
    free = [threading.Semaphore(1) for _ in range(2)]

    def snapshot(k, step, time_):
        slot = k % 2
        free[slot].acquire()
        pin_R[slot].copy_(ens.R, non_blocking=True)
        if pin_F is not None:
            pin_F[slot].copy_(ens.total_force_device(), non_blocking=True)
        ready = torch.cuda.Event()
        ready.record()
        writer.put(k, step, time_, pin_R[slot].numpy(), None if pin_F is None else pin_F[slot].numpy(),
                   ready=ready, release=free[slot].release)

    snapshot(0, 0, sim.time_start)
    step, k = 0, 0
    while step < n_steps:
        chunk = min(w, n_steps - step)
        t0 = sim.time_start + step * sim.dt
        ens.advance(t0, count_steps(_segment(sim, t0, t0 + (chunk - 1) * sim.dt)), CACHE_RESET_PER_CALL)
        step += chunk
        k += 1
        snapshot(k, step, sim.time_start + step * sim.dt)
    status = ens.statuses()
    keep = [not (status[i] & ST_FATAL_MASK) for i in range(n_traj)]

    def attrs(i):
        return {"index": i, "seed": seed + i, "n_steps": n_steps, "write_every": output.write_every or n_steps,
                "dt": float(sim.dt), **{f"phys_{k}": v for k, v in _phys_summary(phys).items()}}

    written = iter(writer.finish(keep, attrs, compression=output.compression))
    results = [next(written) if keep[i] else Failure(i, IntegratorError(int(status[i]), i)) for i in range(n_traj)]
    if on_error == "raise":
        bad = [r for r in results if isinstance(r, Failure)]
        if bad:
            raise bad[0].error
    files, failed = _drop_failures(results, "trajectories", max_failed_fraction)
    storage.write_manifest(output.directory, {
        "n_trajectories": len(files), "n_trajectories_requested": n_traj, "n_trajectories_failed": len(failed),
        "seed": seed, "n_steps": n_steps, "dt": float(sim.dt), "write_every": output.write_every or n_steps,
        "write_forces": bool(output.write_forces), "initial": {"method": initial.method, "kwargs": initial.kwargs},
        "phys": _phys_summary(phys), "files": list(files), "backend": "cuda", "form": str(form),
        "counters": ens.counter_totals()})
    return storage.read_run(output.directory)


def trajectory_samples(R0, phys: PhysParams, sim: SimParams, rng, sample_times, *, form="plain", device=0):
    """Configurations of one chain at each sample time (ensemble.py:126-138)."""
    R = np.asarray(R0, dtype=np.float64)
    out, t = [], sim.time_start
    for ts in sample_times:
        R = integrate(R, phys, _segment(sim, t, ts), rng, form=form, device=device)
        out.append((ts, R.copy()))
        t = ts
    return out


def final_state(R0, phys, sim, rng):
    """per_trajectory reducer: the final (N,3) configuration (ensemble.py:309-318)."""
    return np.asarray(integrate(R0, phys, sim, rng), dtype=np.float64)


def sampled_states(R0, phys, sim, rng, sample_times):
    """per_trajectory reducer: the configuration at each sample time (ensemble.py:321-327)."""
    return [R for _t, R in trajectory_samples(R0, phys, sim, rng, sample_times)]


# The reference's own reducers, by (module, name): run_ensemble batches these
# when the reference's run layer hands them over with backend="cuda".
_REFERENCE_REDUCERS = {
    ("bdsim.ensemble", "final_state"): "final_state",
    ("bdsim.ensemble", "sampled_states"): "sampled_states",
    ("bdsim.rheology", "stress_series"): "stress_series",
    ("bdsim.rheology", "viscosity_series"): "viscosity_series",
    ("bdsim.rheology", "viscosity_series_vr"): "viscosity_series_vr",
}


def batched_reducer(fn):
    """This package's batched equivalent of a per_trajectory reducer: the
    function itself when it is one of ours, ours for the reference's
    final_state / sampled_states / rheology series, else None."""
    if fn is final_state or fn is sampled_states or fn in rheology.BATCHED:
        return fn
    name = _REFERENCE_REDUCERS.get((getattr(fn, "__module__", None), getattr(fn, "__qualname__", None)))
    if name is None:
        return None
    return {"final_state": final_state, "sampled_states": sampled_states}.get(name) or getattr(rheology, name)


def run_ensemble(phys: PhysParams, sim: SimParams, n_traj: int, per_trajectory, *, args=(), seed: int = 0,
                 initial: Initial = None, backend="cuda", n_workers=None, on_error="skip",
                 max_failed_fraction=None, form="plain", device: int = 0):
    """Run n_traj chains, reducing each with per_trajectory (ensemble.py:330-379).

    final_state, sampled_states and the rheology series (stress_series,
    viscosity_series, viscosity_series_vr) run batched: all trajectories
    (and the control chains of the variance-reduced series) advance together
    in one device batch per integrate segment. Any other function is called
    once per trajectory as per_trajectory(R0, phys, sim, rng, *args); the
    integrate calls it makes run on the GPU one chain at a time.
    """
    _check_backend(backend)
    initial = initial or Initial()
    per_trajectory = batched_reducer(per_trajectory) or per_trajectory
    if per_trajectory is final_state or per_trajectory is sampled_states:
        ens, _ = _start(phys, sim, n_traj, seed, initial, form, device)
        if per_trajectory is final_state:
            segs = [(sim.time_start, sim.time_end)]
        else:
            times = list(args[0])
            segs = list(zip([sim.time_start] + times[:-1], times))
        per = [[] for _ in range(n_traj)]
        for t0, t1 in segs:
            k = count_steps(_segment(sim, t0, t1))
            ens.advance(t0, k, CACHE_RESET_PER_CALL)
            for i, R in enumerate(ens.positions()):
                per[i].append(R)
        status = ens.statuses()
        out = []
        for i in range(n_traj):
            if status[i] & ST_FATAL_MASK:
                out.append(Failure(i, IntegratorError(int(status[i]), i)))
            else:
                out.append(per[i][-1] if per_trajectory is final_state else per[i])
    elif per_trajectory in rheology.BATCHED:
        R0s = [INITIALIZERS[initial.method](phys.number_of_beads, seed + i, dict(initial.kwargs))
               for i in range(n_traj)]
        out = rheology.run_batched(per_trajectory, phys, sim, n_traj, args, R0s, seed, form, device)
    else:
        out = []
        for i in range(n_traj):
            R0 = INITIALIZERS[initial.method](phys.number_of_beads, seed + i, dict(initial.kwargs))
            try:
                out.append(per_trajectory(R0, phys, sim, Rng(seed + i), *args))
            except Exception as exc:
                if on_error == "raise":
                    raise
                out.append(Failure(i, exc))
    if on_error == "raise":
        bad = [r for r in out if isinstance(r, Failure)]
        if bad:
            raise bad[0].error
    out, _ = _drop_failures(out, "trajectories", max_failed_fraction)
    return out
