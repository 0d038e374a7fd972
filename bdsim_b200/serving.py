"""Serving: continuous batching of ensemble jobs on one GPU.

bdsim runs one ensemble per `simulate` call (python/bdsim/ensemble.py:179-227).
A `Server` instead keeps a pool of chain slots resident on the device and
admits jobs -- each the arguments of a `simulate` call -- while others run:

  * admission: a job of n_traj chains of N beads needs n_traj consecutive
    slots, n_traj*N consecutive beads of the pool (the pool is the HBM budget:
    positions, warm-start vectors and the snapshot buffers) and room under the
    active-chain cap; queued jobs are admitted in arrival order with a short
    first-fit lookahead (policy "fifo") or smallest estimated work first
    (policy "sjf": n_traj * n_steps * N^2, the pair work of its D.x products),
    and arrivals beyond the queue limit are rejected;
  * each server iteration is ONE time-sliced launch (bdcu_run_slice) over the
    chains of every running job (buckets by bead count, device work lists),
    so jobs of different N, n_traj and n_steps share the GPU: every chain
    takes up to `slice_steps` steps of its current chunk (write_every steps,
    the job's snapshot interval), and none starts a new step after
    `slice_budget_s` -- a job whose steps are slow (a corrector at its
    100N-iteration cap takes ~1 s per step at N=300) cannot hold the others'
    snapshots back;
  * the launch reports each chain's completed steps and time; a chunk in
    progress continues in the next launch from there with its warm spectral
    cache, so a chunk cut into slices gives the same chains, bit for bit, as
    one integrate call over it;
  * when all of a job's chains have finished a chunk, its positions are
    copied to the host and delivered (at its last chunk with its statuses),
    and a finished job's slots are freed for the next admission;
  * latency of a job = arrival to delivery of its last snapshot.

A job's chains follow exactly the trajectory of `simulate` with the same
arguments: trajectory i is seeded seed+i and starts from the same initial
configuration, a chunk of k steps is one integrate span [t0, t0+(k-1)dt] with
a cold spectral cache (CACHE_RESET_PER_CALL, the default), and the RNG stream
carries across chunks.
"""
from __future__ import annotations

import bisect
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from ._abi import CACHE_PERSIST, CACHE_RESET_PER_CALL, COUNTER_FIELDS, ST_FATAL_MASK, count_steps
from .engine import Context, _torch, form_code
from . import _abi, storage
from .ensemble import INITIALIZERS, Initial, Output, _phys_summary, _segment, n_steps_of
from .params import PhysParams, Rng, SimParams

BYTES_PER_BEAD = 4 * 24  # R, warm-start cache, two snapshot buffers (FP64 xyz each)


class Intervals:
    """First-fit allocator of [0, capacity) in integer units."""

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        self._free = [(0, self.capacity)]  # sorted, coalesced (start, length)

    def alloc(self, n: int):
        n = int(n)
        for i, (s, L) in enumerate(self._free):
            if L >= n:
                if L == n:
                    self._free.pop(i)
                else:
                    self._free[i] = (s + n, L - n)
                return s
        return None

    def free(self, start: int, n: int):
        if n <= 0:
            return
        i = bisect.bisect_left(self._free, (start, 0))
        self._free.insert(i, (int(start), int(n)))
        merged = []
        for s, L in self._free:
            if merged and merged[-1][0] + merged[-1][1] == s:
                merged[-1] = (merged[-1][0], merged[-1][1] + L)
            else:
                merged.append((s, L))
        self._free = merged

    def used(self) -> int:
        return self.capacity - sum(L for _, L in self._free)

    def high_water(self) -> int:
        """End of the last allocated unit (0 when empty)."""
        if not self._free:
            return self.capacity
        s, L = self._free[-1]
        return s if s + L == self.capacity else self.capacity


@dataclass
class Job:
    """The arguments of one `simulate` call, plus its arrival time."""
    phys: PhysParams
    sim: SimParams
    n_traj: int = 1
    seed: int = 0
    n_steps: int = None
    initial: Initial = None
    write_every: int = 0
    keep_snapshots: bool = True
    name: str = ""
    # the run directory of `simulate` (python/bdsim/storage.py layout): each
    # chunk's positions are spooled to disk by a writer thread as they arrive,
    # and traj_NNNNN + manifest.json are written when the job completes
    # (positions only: write_forces is not served)
    output: Output = None


@dataclass
class JobState:
    job: Job
    t_arrival: float
    state: str = "queued"  # queued | running | done | rejected
    t_admit: float = None
    t_done: float = None
    n_steps: int = 0
    step: int = 0  # steps of the chunks completed
    chunk_end: int = -1  # step count at the end of the chunk in progress (-1: none)
    t_chunk_end: float = 0.0
    slot0: int = -1
    bead0: int = -1
    arena0: int = -1
    arena_n: int = 0
    n_beads: int = 0
    steps: list = field(default_factory=list)
    times: list = field(default_factory=list)
    positions: list = field(default_factory=list)  # per snapshot: (n_traj, N, 3)
    status: np.ndarray = None
    counters: dict = None
    writer: object = None  # storage.RunWriter of a job with an output directory
    files: list = None     # the trajectory files it wrote
    write_error: object = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrival

    def trajectories(self) -> np.ndarray:
        """(n_traj, n_snap, N, 3) positions, the layout of `simulate`'s files."""
        return np.stack(self.positions, axis=1)


class Server:
    """Continuous batching of ensemble jobs on one GPU (see the module text).

    form: "mixed" or "plain"; max_chains: slots of the pool; bead_capacity:
    beads of the pool (default: hbm_budget_bytes / BYTES_PER_BEAD);
    max_active_chains: cap on running chains (None: the pool); queue_limit:
    queued jobs beyond which arrivals are rejected (None: unbounded)."""

    def __init__(self, device: int = 0, form="mixed", max_chains: int = 65536, bead_capacity: int = None,
                 hbm_budget_bytes: int = 1 << 30, arena_capacity: int = 1 << 20, max_active_chains: int = None,
                 queue_limit: int = None, lookahead: int = 16, cache_mode: int = CACHE_RESET_PER_CALL,
                 on_snapshot=None, clock=time.monotonic, slice_steps: int = 10, slice_budget_s: float = 1.0,
                 policy: str = "fifo"):
        torch = _torch()
        self.torch = torch
        self.form = form_code(form)
        self.cache_mode = cache_mode
        if policy not in ("fifo", "sjf"):
            raise ValueError("policy is 'fifo' or 'sjf'")
        self.policy = policy
        self.slice_steps = int(slice_steps)
        self.budget_ns = int(slice_budget_s * 1e9)
        self.clock = clock
        self.on_snapshot = on_snapshot
        self.max_chains = int(max_chains)
        self.bead_capacity = int(bead_capacity or max(1024, hbm_budget_bytes // BYTES_PER_BEAD))
        self.max_active = int(max_active_chains or max_chains)
        self.queue_limit = queue_limit
        self.lookahead = int(lookahead)
        dev = torch.device("cuda", device)
        self.dev = dev
        self.ctx = Context(device)
        self.ctx.reserve(self.max_chains, self.bead_capacity, arena_capacity)
        nb, nc = self.bead_capacity, self.max_chains
        self.R = torch.zeros((nb, 3), dtype=torch.float64, device=dev)
        self.cache = torch.zeros(3 * nb, dtype=torch.float64, device=dev)
        self.rng = torch.zeros((nc, 3), dtype=torch.int32, device=dev)
        self.valid = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.status = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.counters = torch.zeros((nc, len(COUNTER_FIELDS)), dtype=torch.int64, device=dev)
        self.t0 = torch.zeros(nc, dtype=torch.float64, device=dev)
        self.k = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.steps_done = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.t_end = torch.zeros(nc, dtype=torch.float64, device=dev)
        # host view of every slot: steps left in its chunk, time of its next step
        self.rem = np.zeros(nc, dtype=np.int32)
        self.tnext = np.zeros(nc, dtype=np.float64)
        self.t_host = torch.zeros(nc, dtype=torch.float64, pin_memory=True)
        self.k_host = torch.zeros(nc, dtype=torch.int32, pin_memory=True)
        self.done_host = torch.zeros(nc, dtype=torch.int32, pin_memory=True)
        self.tend_host = torch.zeros(nc, dtype=torch.float64, pin_memory=True)
        self.status_host = torch.zeros(nc, dtype=torch.int32, pin_memory=True)
        self.slots = Intervals(nc)
        self.beads = Intervals(nb)
        self.arena = Intervals(arena_capacity)
        self.queue: list[JobState] = []
        self.running: list[JobState] = []
        self.done: list[JobState] = []
        self.rejected: list[JobState] = []
        self._iter = 0
        self._selected = None
        self.active_chains = 0
        self.chain_steps = 0
        self.t_first = None
        # where the time goes: device time of the slice launches, slices run,
        # chains selected per slice, counters of retired jobs' chains
        self.device_ms = 0.0
        self.n_slices = 0
        self.selected_chains = 0
        self.retired_counters = np.zeros(len(COUNTER_FIELDS), dtype=np.int64)
        self.finalizing = []  # threads writing finished jobs' run directories

    # ------------------------------------------------------------------ API

    def submit(self, job: Job, arrival: float = None) -> JobState:
        """Queue a job (arrival: a time of `clock`, default now)."""
        js = JobState(job=job, t_arrival=self.clock() if arrival is None else arrival)
        if self.t_first is None:
            self.t_first = js.t_arrival
        js.n_steps = int(job.n_steps) if job.n_steps is not None else n_steps_of(job.sim)
        js.n_beads = int(job.phys.number_of_beads)
        if self.queue_limit is not None and len(self.queue) >= self.queue_limit:
            js.state = "rejected"
            self.rejected.append(js)
            return js
        if job.n_traj > min(self.max_chains, self.max_active) or job.n_traj * js.n_beads > self.bead_capacity:
            js.state = "rejected"
            self.rejected.append(js)
            return js
        self.queue.append(js)
        return js

    def busy(self) -> bool:
        return bool(self.queue or self.running)

    def step(self):
        """One server iteration: admit, one time-sliced launch over the
        running jobs, deliver the chunks it completed."""
        self._admit()
        work = self._launch_slice()
        if work is not None:
            self._finish_slice(*work)

    def run_until_idle(self, max_iters: int = 10 ** 9):
        it = 0
        while self.busy() and it < max_iters:
            self.step()
            it += 1
        self.flush()

    def flush(self):
        """Wait until the run directories of finished jobs are written (their
        errors are raised here)."""
        while self.finalizing:
            self.finalizing.pop(0).join()
        errs = [js.write_error for js in self.done if getattr(js, "write_error", None) is not None]
        if errs:
            raise errs[0]

    def run_stream(self, jobs, arrivals, horizon: float = None, drain: bool = True, drain_limit: float = None):
        """Replay an arrival stream in real time: jobs[i] arrives arrivals[i]
        seconds after the start. Stops admitting at `horizon` seconds (if
        given) and, with drain, runs the admitted work to completion, or for
        at most `drain_limit` seconds past the horizon (jobs still running
        then are reported as censored)."""
        order = np.argsort(arrivals, kind="stable")
        t0 = self.clock()
        i = 0
        while True:
            now = self.clock() - t0
            while i < len(order) and arrivals[order[i]] <= now and (horizon is None or arrivals[order[i]] <= horizon):
                self.submit(jobs[order[i]], arrival=t0 + arrivals[order[i]])
                i += 1
            more = i < len(order) and (horizon is None or arrivals[order[i]] <= horizon)
            if not self.busy():
                if not more:
                    break
                time.sleep(max(0.0, min(0.05, arrivals[order[i]] - now)))
                continue
            if horizon is not None and now > horizon and (not drain or
                                                         (drain_limit is not None and now > horizon + drain_limit)):
                break
            self.step()
        self.flush()
        return self.stats(t0)

    def stats(self, t0: float = None) -> dict:
        """Latency and throughput of the jobs so far.

        p50/p99_latency_s cover completed jobs (n_latency_samples of them).
        Jobs still running or queued have waited at least now - arrival: with
        those as censored samples, p50/p99_latency_lower_bound_s are lower
        bounds of the percentiles over every admitted job
        (n_admitted_samples). The breakdown says where the wall time went:
        the share of it the GPU spent in slice launches, slices and chains per
        slice, and corrector iterations and D.x products per chain-step."""
        now = self.clock()
        lat = np.array([j.latency for j in self.done], dtype=np.float64)
        svc = np.array([j.t_done - j.t_admit for j in self.done], dtype=np.float64)
        cens = np.array([now - j.t_arrival for j in self.running + self.queue], dtype=np.float64)
        both = np.concatenate([lat, cens])
        t0 = self.t_first if t0 is None else t0
        # throughput over the whole replay: up to the last completion, or up
        # to now when nothing has completed yet
        wall = ((max(j.t_done for j in self.done) if self.done else now) - t0) if t0 is not None else 0.0
        span = (now - t0) if t0 is not None else 0.0
        pct = (lambda a, q: float(np.percentile(a, q)) if a.size else None)
        cnt = self.retired_counters.copy()
        if self.running:  # retired jobs' rows were zeroed when they left: the pool holds running jobs only
            cnt = cnt + self.counters.sum(dim=0).cpu().numpy().astype(np.int64)
        c = dict(zip(COUNTER_FIELDS, (int(v) for v in cnt)))
        steps = max(c["steps"], 1)
        return {"jobs_completed": len(self.done), "jobs_rejected": len(self.rejected),
                "jobs_queued": len(self.queue), "jobs_running": len(self.running),
                "p50_latency_s": pct(lat, 50), "p99_latency_s": pct(lat, 99), "n_latency_samples": int(lat.size),
                "p50_latency_lower_bound_s": pct(both, 50), "p99_latency_lower_bound_s": pct(both, 99),
                "n_admitted_samples": int(both.size),
                "p50_service_s": pct(svc, 50), "p99_service_s": pct(svc, 99),
                "chain_steps": int(self.chain_steps), "wall_s": wall,
                "chain_steps_per_s": (self.chain_steps / wall) if wall > 0 else None,
                "breakdown": {
                    "gpu_busy_frac": (self.device_ms * 1e-3 / span) if span > 0 else None,
                    "slices": self.n_slices,
                    "chains_per_slice": (self.selected_chains / self.n_slices) if self.n_slices else None,
                    "corrector_iters_per_step": c["corrector_iters"] / steps,
                    "dx_per_step": c["dx_products"] / steps,
                    "nonconverged_step_frac": c["nonconverged"] / steps,
                    "chain_steps_per_device_s": (self.chain_steps / (self.device_ms * 1e-3)) if self.device_ms else None}}

    # ------------------------------------------------------------ internals

    def _admit(self):
        torch = self.torch
        if self.policy == "sjf" and len(self.queue) > 1:
            self.queue.sort(key=lambda q: (int(q.job.n_traj) * q.n_steps * q.n_beads ** 2, q.t_arrival))
        i, looked = 0, 0
        limit = self.lookahead if self.policy == "fifo" else len(self.queue)
        while i < len(self.queue) and looked < limit:
            js = self.queue[i]
            job = js.job
            n, N = int(job.n_traj), js.n_beads
            ok = self.active_chains + n <= self.max_active
            s0 = self.slots.alloc(n) if ok else None
            b0 = self.beads.alloc(n * N) if s0 is not None else None
            if s0 is None or b0 is None:
                if s0 is not None:
                    self.slots.free(s0, n)
                i += 1
                looked += 1
                continue
            self.queue.pop(i)
            init = job.initial or Initial()
            R0s = [INITIALIZERS[init.method](N, job.seed + t, dict(init.kwargs)) for t in range(n)]
            R0 = np.ascontiguousarray(np.concatenate(R0s).reshape(-1, 3), dtype=np.float64)
            rng = np.array([Rng(job.seed + t).state() for t in range(n)], dtype=np.int32)
            self.R[b0:b0 + n * N].copy_(torch.from_numpy(R0).pin_memory(), non_blocking=True)
            self.rng[s0:s0 + n].copy_(torch.from_numpy(rng).pin_memory(), non_blocking=True)
            self.valid[s0:s0 + n].zero_()
            self.status[s0:s0 + n].zero_()
            self.counters[s0:s0 + n].zero_()
            packed = self.ctx.pack_slots([job.phys] * n, [job.sim] * n, [N] * n)
            a0 = 0
            if packed[2] is not None:
                a0 = self.arena.alloc(packed[2].size)
                if a0 is None:
                    raise RuntimeError("serving arena exhausted (raise arena_capacity)")
            used = self.ctx.fill_slots(list(range(s0, s0 + n)), None, None, None, [b0 + t * N for t in range(n)],
                                       arena_base=a0, packed=packed)
            js.slot0, js.bead0, js.arena0, js.arena_n = s0, b0, a0, used
            js.state, js.t_admit = "running", self.clock()
            js.steps.append(0)
            js.times.append(float(job.sim.time_start))
            if job.output is not None:
                if job.output.directory is None or job.output.write_forces:
                    raise ValueError("a served job's output needs a directory and no forces")
                w = job.write_every if (job.write_every and job.write_every > 0) else js.n_steps
                js.writer = storage.RunWriter(job.output.directory, np.arange(n + 1) * N,
                                              1 + (js.n_steps + w - 1) // w, max_pending=4)
                js.writer.put(0, 0, float(job.sim.time_start), R0.copy())
            if job.keep_snapshots:
                js.positions.append(R0.reshape(n, N, 3).copy())
            if self.on_snapshot is not None:
                self.on_snapshot(js, 0, float(job.sim.time_start), R0.reshape(n, N, 3))
            self.active_chains += n
            self.running.append(js)

    def _launch_slice(self):
        torch = self.torch
        work = [js for js in self.running if js.state == "running"]
        if not work:
            return None
        self._iter += 1
        rem, tnext = self.rem, self.tnext
        fresh = []
        for js in work:
            if js.chunk_end < 0:  # start the job's next chunk: one integrate span
                job, n, sim = js.job, int(js.job.n_traj), js.job.sim
                w = job.write_every if (job.write_every and job.write_every > 0) else js.n_steps
                chunk = min(w, js.n_steps - js.step)
                t0 = sim.time_start + js.step * sim.dt
                k = count_steps(_segment(sim, t0, t0 + (chunk - 1) * sim.dt))
                rem[js.slot0:js.slot0 + n] = k
                tnext[js.slot0:js.slot0 + n] = t0
                js.chunk_end = js.step + chunk
                js.t_chunk_end = sim.time_start + js.chunk_end * sim.dt
                fresh.append((js.slot0, n))
        sel = [s for js in work for s in range(js.slot0, js.slot0 + int(js.job.n_traj)) if rem[s] > 0]
        if not sel:
            return work, []
        hi_slot = max(js.slot0 + int(js.job.n_traj) for js in work)
        kh = self.k_host.numpy()
        kh[:hi_slot] = np.minimum(rem[:hi_slot], self.slice_steps)
        self.t_host.numpy()[:hi_slot] = tnext[:hi_slot]
        self.t0[:hi_slot].copy_(self.t_host[:hi_slot], non_blocking=True)
        self.k[:hi_slot].copy_(self.k_host[:hi_slot], non_blocking=True)
        if self.cache_mode == CACHE_RESET_PER_CALL:
            for s0, n in fresh:  # a new chunk starts with a cold spectral cache (a new integrate call)
                self.valid[s0:s0 + n].zero_()
        key = tuple(sel)
        if key != self._selected:
            self.ctx.select(sel)
            self._selected = key
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record()
        self.ctx.run_slice(self.R, self.rng, self.cache, self.valid, self.t0, self.k, self.status, self.counters,
                           self.form, CACHE_PERSIST, self.budget_ns, self.steps_done, self.t_end)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        self._slice_events = (e0, e1)
        self.n_slices += 1
        self.selected_chains += len(sel)
        self.done_host[:hi_slot].copy_(self.steps_done[:hi_slot], non_blocking=True)
        self.tend_host[:hi_slot].copy_(self.t_end[:hi_slot], non_blocking=True)
        self.status_host[:hi_slot].copy_(self.status[:hi_slot], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        return work, sel, ev

    def _finish_slice(self, work, sel, ev=None):
        torch = self.torch
        if ev is not None:
            ev.synchronize()
            e0, e1 = self._slice_events
            self.device_ms += e0.elapsed_time(e1)
        sel = np.asarray(sel, dtype=np.int64)
        if sel.size:
            done = self.done_host.numpy()[sel]
            self.rem[sel] -= done
            moved = done > 0
            self.tnext[sel[moved]] = self.tend_host.numpy()[sel[moved]]
            self.chain_steps += int(done.sum())
            fatal = (self.status_host.numpy()[sel] & ST_FATAL_MASK) != 0
            self.rem[sel[fatal]] = 0  # a failed chain is stopped for good
        now = self.clock()
        for js in work:
            n = int(js.job.n_traj)
            if js.chunk_end < 0 or self.rem[js.slot0:js.slot0 + n].any():
                continue
            # chunk complete for every chain: deliver its snapshot
            js.step = js.chunk_end
            js.chunk_end = -1
            N = js.n_beads
            if js.writer is not None:
                # device -> pinned host copy on the stream; the writer thread
                # waits for it and spools the chunk while the server goes on
                pinned = torch.empty((n * N, 3), dtype=torch.float64, pin_memory=True)
                pinned.copy_(self.R[js.bead0:js.bead0 + n * N], non_blocking=True)
                ready = torch.cuda.Event()
                ready.record()
                js.writer.put(len(js.steps), js.step, js.t_chunk_end, pinned.numpy(), ready=ready)
            rows = None
            if js.job.keep_snapshots or self.on_snapshot is not None:
                rows = self.R[js.bead0:js.bead0 + n * N].cpu().numpy().reshape(n, N, 3)
            js.steps.append(js.step)
            js.times.append(js.t_chunk_end)
            if js.job.keep_snapshots:
                js.positions.append(rows.copy())
            if self.on_snapshot is not None:
                self.on_snapshot(js, js.step, js.t_chunk_end, rows)
            st = self.status_host.numpy()[js.slot0:js.slot0 + n]
            if js.step >= js.n_steps or bool(((st & ST_FATAL_MASK) != 0).all()):
                js.status = st.copy()
                if js.writer is not None:  # the run directory is assembled off the serving loop
                    th = threading.Thread(target=self._write_run, args=(js,), daemon=True)
                    th.start()
                    self.finalizing.append(th)
                js.state, js.t_done = "done", now
                self._retire(js)

    def _write_run(self, js: JobState):
        """The job's run directory, as `simulate` writes it (its chunks are on
        the spool already)."""
        job = js.job
        keep = (js.status & ST_FATAL_MASK) == 0
        w = job.write_every if (job.write_every and job.write_every > 0) else js.n_steps

        def attrs(i):
            return {"index": i, "seed": job.seed + i, "n_steps": js.n_steps, "write_every": w,
                    "dt": float(job.sim.dt), **{f"phys_{k}": v for k, v in _phys_summary(job.phys).items()}}

        # (every chain failed before the end: the snapshots that ran)
        try:
            js.files = js.writer.finish(keep, attrs, compression=job.output.compression, n_used=len(js.steps))
        except Exception as exc:  # raised by flush()
            js.write_error = exc
            return
        init = job.initial or Initial()
        storage.write_manifest(job.output.directory, {
            "n_trajectories": len(js.files), "n_trajectories_requested": int(job.n_traj),
            "n_trajectories_failed": int((~keep).sum()), "seed": job.seed, "n_steps": js.n_steps,
            "dt": float(job.sim.dt), "write_every": w, "write_forces": False,
            "initial": {"method": init.method, "kwargs": init.kwargs}, "phys": _phys_summary(job.phys),
            "files": list(js.files), "backend": "cuda (served)"})
        js.writer = None

    def _retire(self, js: JobState):
        n = int(js.job.n_traj)
        rows = self.counters[js.slot0:js.slot0 + n].sum(dim=0).cpu().numpy()
        js.counters = dict(zip(COUNTER_FIELDS, (int(v) for v in rows)))
        self.retired_counters += rows.astype(np.int64)
        self.counters[js.slot0:js.slot0 + n].zero_()
        self.running.remove(js)
        self.done.append(js)
        self.slots.free(js.slot0, n)
        self.beads.free(js.bead0, n * js.n_beads)
        if js.arena_n:
            self.arena.free(js.arena0, js.arena_n)
        self.active_chains -= n

    def failed(self, js: JobState) -> np.ndarray:
        return (js.status & ST_FATAL_MASK) != 0


class NativeQueue:
    """The C ABI's serving queue (bdcu_queue_*, include/bdsim_cuda.h): the
    policy of `Server` -- admission by slots, beads, arena and the active-chain
    cap, FIFO with lookahead or shortest-job-first, one time-sliced launch per
    iteration, a snapshot per chunk -- run by the native library, optionally
    on its own worker thread, so that a C or C++ host serves the same way.
    This class only packs `Job`s (initial positions from the job's
    initializer, RNG states seed+i, one parameter record) and unpacks events.

    Events (`poll`): dicts with kind "snapshot" (positions (n_traj, N, 3)),
    "done" (status per chain, summed counters) or "rejected", and the job id,
    tag, step, time and the queue-clock times of arrival, admission and
    delivery."""

    _KINDS = {_abi.QEV_SNAPSHOT: "snapshot", _abi.QEV_DONE: "done", _abi.QEV_REJECTED: "rejected"}

    def __init__(self, device: int = 0, form="mixed", max_chains: int = 65536, bead_capacity: int = None,
                 hbm_budget_bytes: int = 1 << 30, arena_capacity: int = 1 << 20, max_active_chains: int = None,
                 queue_limit: int = None, lookahead: int = 16, cache_mode: int = CACHE_RESET_PER_CALL,
                 slice_steps: int = 10, slice_budget_s: float = 1.0, policy: str = "fifo", worker: bool = False):
        import ctypes
        self._ct = ctypes
        self.lib = _abi.load_library()
        if policy not in ("fifo", "sjf"):
            raise ValueError("policy is 'fifo' or 'sjf'")
        cfg = _abi.BdcuQueueConfig()
        cfg.form = form_code(form)
        cfg.policy = _abi.QUEUE_FIFO if policy == "fifo" else _abi.QUEUE_SJF
        cfg.max_chains = int(max_chains)
        cfg.max_active_chains = int(max_active_chains or 0)
        cfg.bead_capacity = int(bead_capacity or max(1024, hbm_budget_bytes // BYTES_PER_BEAD))
        cfg.arena_capacity = int(arena_capacity)
        cfg.queue_limit = int(queue_limit or 0)
        cfg.lookahead = int(lookahead)
        cfg.slice_steps = int(slice_steps)
        cfg.cache_mode = int(cache_mode)
        cfg.slice_budget_ns = int(slice_budget_s * 1e9)
        cfg.worker = 1 if worker else 0
        self.cfg = cfg
        self.h = ctypes.c_void_p()
        rc = self.lib.bdcu_queue_create(int(device), ctypes.byref(cfg), ctypes.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"bdcu_queue_create failed ({rc}): {self.lib.bdcu_queue_last_error(None).decode()}")
        self._pos = np.zeros(0, dtype=np.float64)
        self._status = np.zeros(cfg.max_chains, dtype=np.int32)

    def _ck(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.lib.bdcu_queue_last_error(self.h).decode()}")

    def close(self):
        if self.h:
            self.lib.bdcu_queue_destroy(self.h)
            self.h = self._ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, job: Job, tag: int = 0, snapshots: bool = None):
        """Queue a job; returns (job id, accepted). snapshots: deliver every
        chunk (default: job.keep_snapshots) or only the final positions."""
        ct = self._ct
        N, n = int(job.phys.number_of_beads), int(job.n_traj)
        init = job.initial or Initial()
        R0 = np.ascontiguousarray(np.concatenate(
            [INITIALIZERS[init.method](N, job.seed + t, dict(init.kwargs)) for t in range(n)]).reshape(-1, 3),
            dtype=np.float64)
        rng = np.ascontiguousarray([Rng(job.seed + t).state() for t in range(n)], dtype=np.int32)
        prec, srec, arena = _abi.pack_batch([job.phys], [job.sim], [N])
        d = _abi.BdcuJob()
        d.n_traj = n
        d.snapshots = int(job.keep_snapshots if snapshots is None else snapshots)
        d.n_steps = int(job.n_steps) if job.n_steps is not None else n_steps_of(job.sim)
        d.write_every = int(job.write_every) if job.write_every and job.write_every > 0 else 0
        d.tag = int(tag)
        d.phys = prec[0]
        d.sim = srec[0]
        r = prec[0]
        uses = r.phi_offset >= 0 or r.flow_n_times > 0 or r.ext_n_entries > 0
        arena = np.ascontiguousarray(arena if uses else np.zeros(0), dtype=np.float64)
        d.arena = arena.ctypes.data_as(_abi.c_double_p) if arena.size else None
        d.arena_len = int(arena.size)
        d.R0 = R0.ctypes.data_as(_abi.c_double_p)
        d.rng = rng.ctypes.data_as(_abi.c_int32_p)
        jid, ok = ct.c_int64(0), ct.c_int(0)
        self._ck(self.lib.bdcu_queue_submit(self.h, ct.byref(d), ct.byref(jid), ct.byref(ok)), "bdcu_queue_submit")
        return int(jid.value), bool(ok.value)

    def step(self) -> bool:
        """One iteration (caller-driven queues); True while jobs remain."""
        busy = self._ct.c_int(0)
        self._ck(self.lib.bdcu_queue_step(self.h, self._ct.byref(busy)), "bdcu_queue_step")
        return bool(busy.value)

    def wait_idle(self, timeout_s: float = None) -> bool:
        """Run (or wait for the worker) until no job is queued or running;
        returns True if jobs remain at the timeout."""
        busy = self._ct.c_int(0)
        ms = -1 if timeout_s is None else int(timeout_s * 1000)
        self._ck(self.lib.bdcu_queue_wait_idle(self.h, ms, self._ct.byref(busy)), "bdcu_queue_wait_idle")
        return bool(busy.value)

    def poll(self):
        """The oldest undelivered event as a dict, or None."""
        ct = self._ct
        ev, got = _abi.BdcuQueueEvent(), ct.c_int(0)
        while True:
            rc = self.lib.bdcu_queue_poll(self.h, ct.byref(ev), self._pos.ctypes.data_as(_abi.c_double_p),
                                          self._pos.size, self._status.ctypes.data_as(_abi.c_int32_p),
                                          self._status.size, ct.byref(got))
            if rc == 5:  # BDCU_E_LIMIT: the positions buffer is too small for this event
                self._pos = np.zeros(3 * ev.n_traj * ev.n_beads, dtype=np.float64)
                continue
            self._ck(rc, "bdcu_queue_poll")
            break
        if not got.value:
            return None
        out = {"kind": self._KINDS[ev.kind], "job": ev.job, "tag": ev.tag, "n_traj": ev.n_traj,
               "n_beads": ev.n_beads, "step": ev.step, "time": ev.time, "t_arrival": ev.t_arrival,
               "t_admit": ev.t_admit, "t_done": ev.t_done}
        if ev.kind == _abi.QEV_SNAPSHOT:
            out["snapshot"] = ev.snapshot
            out["positions"] = self._pos[:3 * ev.n_traj * ev.n_beads].reshape(ev.n_traj, ev.n_beads, 3).copy()
        elif ev.kind == _abi.QEV_DONE:
            out["status"] = self._status[:ev.n_traj].copy()
            out["counters"] = {f: getattr(ev.counters, f) for f in COUNTER_FIELDS}
        return out

    def events(self) -> list:
        out = []
        while (e := self.poll()) is not None:
            out.append(e)
        return out

    def stats(self) -> dict:
        st = _abi.BdcuQueueStats()
        self._ck(self.lib.bdcu_queue_get_stats(self.h, self._ct.byref(st)), "bdcu_queue_get_stats")
        return st.as_dict()
