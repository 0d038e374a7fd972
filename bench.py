"""Benchmark of the B200 ensemble integrator (bdsim ChainIntegrator step).

Workload (the reference's headline configuration, seeded synthetic chains):
  4096 trajectories x N=50 beads, FENE springs b=50, RPY HI h*=0.25 with the
  Chebyshev square root and Lanczos bounds, Gaussian EV z*=1 d*=0.5, simple
  shear rate 1, dt=1e-3; initial chains from Gaussian bonds (unit variance),
  trajectory i seeded with i.

A bench "step" is one chunk of CHUNK=100 integrator steps of every chain (one
write_every block), i.e. one launch of the persistent integrator kernel. The
headline value is the FP32-mixed form; the FP64 plain form is measured in the
same run. `e2e` goes through the reference-facing host-buffer entry point
(bdcu_integrate_host: pinned R and RNG state copied in, integrated, copied
out every step). `ensemble` compares the final ensemble <Rg^2> and <tau_xy>
of the two forms; `latency` is the p50/p99 job latency of the serving
workload replayed against the continuous-batching server.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

For N>1 launch under torch.distributed.run: every rank integrates its own
shard of 4096 chains (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CHAINS = 4096
N_BEADS = 50
CHUNK = 100
DT = 1e-3
WORKLOAD = ("4096 chains x N=50, FENE b=50, RPY h*=0.25 Chebyshev+Lanczos, Gauss EV z*=1 d*=0.5, "
            "shear 1.0, dt=1e-3, gaussian_chain(50, bond_std=1, seed=i), Rng(i)")
WORKLOAD_SHORT = "4096 x N=50 FENE b=50, RPY h*=0.25 Chebyshev, Gauss EV, shear 1, dt=1e-3 (cfg2)"
METRIC = "chain-steps/sec at N=50 HI (FP32-mixed vs FP64 plain, 1 B200)"
# the lighter serving stream: the same job mix, shorter jobs, fewer arrivals
LIGHT = {"scale_steps": 0.01, "rate": 2.0, "horizon": 20.0, "drain_limit": 20.0}
SERVING_WORKLOAD = ("Poisson arrivals 200 jobs/s; N ~ U{10..300}, n_traj ~ U{1..256}, n_steps log-uniform "
                    "[1e3, 1e5], shear or uniaxial at U[0.1, 5], FENE b=100, h*=0.25 Chebyshev, write_every=100; "
                    "replayed in real time for the horizon; shortest-job-first admission under a 256-job queue "
                    "bound and 4096 active chains, 100-step / 1 s time slices; jobs not finished by the end of "
                    "the horizon are not counted")
# Flop accounting per chain-step (dense-equivalent, the same for both forms):
#   each D.x product on the 3N-vector counts 2*(3N)^2 flops; each EV pair
#   evaluation 20 flops (2 evaluations per step, at R and R~); RPY pair
#   assembly 30 flops per pair (once per step).
C_EV = 20.0
C_RPY = 30.0


def make_phys():
    from bdsim_b200.params import DelSMethod, EV, Flow, PhysParams, SimParams, Spring
    p = PhysParams()
    p.spring.type = Spring.FENE
    p.spring.sqrtb = 50.0 ** 0.5
    p.hstar = 0.25
    p.hi_method = DelSMethod.Chebyshev
    p.ev.type = EV.Gauss
    p.ev.zstar = 1.0
    p.ev.dstar = 0.5
    K = np.zeros((3, 3))
    K[0, 1] = 1.0
    p.flow = Flow.constant(K)
    p.number_of_beads = N_BEADS
    s = SimParams()
    s.dt = DT
    return p, s


def make_chains(first, count):
    from bdsim_b200 import initial
    return [initial.gaussian_chain(N_BEADS, bond_std=1.0, seed=first + i) for i in range(count)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        loaded = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(torch, buf):
    buf.add_(1.0)  # a 256 MiB write, larger than the 126 MB L2


def run_form(torch, form, Rs, phys, sim, steps, warmup, rank_seed0, stream, bounds_every=1, team_shape=None):
    """Warm up, then time `steps` chunks with CUDA events on the launch stream.
    Each chunk starts its spectral (Lanczos) cache cold, as each integrate call
    of the reference's chunked simulate does. bounds_every: the mixed form's
    spectral-bound refresh interval (1: every step, the reference's policy)."""
    import bdsim_b200 as B
    from bdsim_b200._abi import CACHE_RESET_PER_CALL
    n = len(Rs)
    with torch.cuda.stream(stream):
        ens = B.Ensemble([phys] * n, [sim] * n, Rs, [(1, -1, rank_seed0 + i) for i in range(n)], form=form)
        ens.ctx.set_bounds_refresh(bounds_every)
        if form == "mixed" and team_shape is not None:
            ens.ctx.set_team_shape(0, *team_shape)
        t = 0.0
        for _ in range(warmup):
            ens.advance(t, CHUNK, CACHE_RESET_PER_CALL)
            t += CHUNK * DT
        if form == "mixed" and team_shape is None:
            # the bucket's team shape, timed on copies of the warmed-up state
            # (warm spectral cache, as in every step of a chunk but the first)
            ens.autotune(probe_steps=5, t_start=t)
        stream.synchronize()
        c0 = ens.counter_totals()
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        times = []
        for _ in range(steps):
            flush_l2(torch, flush)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ens.advance(t, CHUNK, CACHE_RESET_PER_CALL)
            e1.record(stream)
            t += CHUNK * DT
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        stream.synchronize()
        c1 = ens.counter_totals()
        failed = int(ens.failed().sum())
        obs = observables(ens, phys)
    delta = {k: c1[k] - c0[k] for k in c1}
    shape = [(b["team_warps"], b["team_beads_per_thread"]) if b["kernel"] == 1 else (b["block"],) for b in ens.plan()]
    return {"ms": times, "counters": delta, "failed": failed, "obs": obs, "shape": shape}


def observables(ens, phys):
    """Per-chain Rg^2 and Kramers shear stress tau_xy of the final state,
    computed on the device (total force, then bdcu_observables;
    python/bdsim/properties.py:17-41)."""
    o = ens.observables()
    return {"rg2": o[:, 0], "tau_xy": o[:, 2]}


def compare_observables(m, p):
    """Ensemble means of the two forms, their standard errors, the
    difference in units of the combined standard error, and the paired
    (same chain, same noise) difference."""
    out = {}
    for k in ("rg2", "tau_xy"):
        a, b = m[k], p[k]
        se_a, se_b = a.std(ddof=1) / np.sqrt(a.size), b.std(ddof=1) / np.sqrt(b.size)
        d = a - b
        out[k] = {"mixed": float(a.mean()), "plain": float(b.mean()), "se_mixed": float(se_a),
                  "se_plain": float(se_b),
                  "diff_in_sigma": float((a.mean() - b.mean()) / np.sqrt(se_a ** 2 + se_b ** 2)),
                  "paired_mean_abs_rel_diff": float(np.mean(np.abs(d)) / max(np.mean(np.abs(b)), 1e-300))}
    return out


def run_e2e(torch, Rs, phys, sim, steps, warmup, seed0, form, team_shape=None):
    """Through the host-buffer entry point: pinned R/RNG in, integrate one
    chunk (a cold spectral cache per call, as a reference integrate call),
    R/RNG/status out -- every step. team_shape: (warps, beads per thread) of
    the N=50 bucket, as the device-resident leg's autotuner chose it."""
    from bdsim_b200 import _abi
    from bdsim_b200.engine import Context, form_code
    n = len(Rs)
    ctx = Context(torch.cuda.current_device())
    s = type(sim)()
    s.dt = sim.dt
    s.implicit_loop_tol = sim.implicit_loop_tol
    s.time_start = 0.0
    s.time_end = (CHUNK - 1) * DT
    ctx.set_chains([phys] * n, [s] * n, [N_BEADS] * n)
    if team_shape is not None:
        ctx.set_team_shape(0, *team_shape)
    R = torch.from_numpy(np.concatenate(Rs)).pin_memory()
    rng = torch.tensor([(1, -1, seed0 + i) for i in range(n)], dtype=torch.int32).pin_memory()
    status = torch.zeros(n, dtype=torch.int32).pin_memory()
    Rp, rp, sp = (ctypes.cast(ctypes.c_void_p(x.data_ptr()), tp) for x, tp in
                  ((R, _abi.c_double_p), (rng, _abi.c_int32_p), (status, _abi.c_int32_p)))
    ctx.use_stream()
    fc = form_code(form)

    def once():
        rc = ctx.lib.bdcu_integrate_host(ctx.h, Rp, rp, sp, None, fc)
        if rc:
            raise RuntimeError(ctx.lib.bdcu_last_error(ctx.h).decode())

    for _ in range(warmup):
        once()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        once()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    h2d = R.numel() * 8 + rng.numel() * 4 + n * (8 + 4)
    d2h = R.numel() * 8 + rng.numel() * 4 + n * 4
    return n * CHUNK * steps / wall, h2d, d2h


def run_serving(torch, horizon, scale_steps=1.0, rate=200.0, seed=0, form="mixed", queue_limit=256,
                max_active=4096, drain=False, policy="sjf", slice_steps=100, slice_budget_s=1.0, drain_limit=None):
    """The serving workload: Poisson job arrivals replayed in real time
    against the continuous-batching server for `horizon` seconds. Jobs: N ~
    U{10..300}, n_traj ~ U{1..256}, n_steps log-uniform [1e3, 1e5] (times
    scale_steps), shear or uniaxial at U[0.1, 5], FENE b=100, h*=0.25
    Chebyshev, write_every=100. Snapshots are copied to pinned host memory
    and delivered every chunk (not kept)."""
    from bdsim_b200 import serving, workloads
    specs = workloads.serving_jobs(rate=rate, duration=horizon, seed=seed)
    jobs, arrivals = [], []
    for sp in specs:
        ns = max(100, int(round(sp.n_steps * scale_steps)))
        jobs.append(serving.Job(phys=sp.phys, sim=sp.sim, n_traj=sp.n_traj, seed=sp.seed, n_steps=ns,
                                write_every=sp.write_every, keep_snapshots=False))
        arrivals.append(sp.arrival)
    # every completed chunk's positions are copied to the host (delivered) and dropped
    srv = serving.Server(device=torch.cuda.current_device(), form=form, max_chains=max_active,
                         hbm_budget_bytes=2 << 30, queue_limit=queue_limit, max_active_chains=max_active,
                         policy=policy, slice_steps=slice_steps, slice_budget_s=slice_budget_s,
                         on_snapshot=lambda js, step, t, rows: None)
    torch.cuda.synchronize()
    st = srv.run_stream(jobs, np.asarray(arrivals), horizon=horizon, drain=drain, drain_limit=drain_limit)
    torch.cuda.synchronize()
    st.update({"jobs_offered": len(jobs), "horizon_s": horizon, "rate_jobs_per_s": rate,
               "n_steps_scale": scale_steps, "queue_limit": queue_limit, "max_active_chains": max_active,
               "policy": policy, "slice_steps": slice_steps, "slice_budget_s": slice_budget_s,
               "offered_chain_steps": int(sum(j.n_traj * j.n_steps for j in jobs))})
    return st


OTHER_WORKLOADS = {
    "cfg3": ("uneven batch: 8192 chains, N ~ U{20..200} (seeded), Marko-Siggia WLC with Q0 ~ U[10,30], h*=0.2 "
             "Chebyshev, uniaxial extension 0.5, LJ EV (0.3, 1.0, cut 2.5), dt=5e-4, FP64 connector solve; "
             "block shapes autotuned per N bucket", 8192, 20),
    "cfg5-cheb": ("large stiff chains: 1024 x N=500 FENE-Fraenkel (sigma 1, dQ 0.1) + bending 5 + SDK EV (d*=1, "
                  "uniform phi 0.5), h*=0.3 Chebyshev (FP64 Lanczos bounds), shear 0.1, dt=1e-4", 1024, 5),
    "cfg5-chol": ("large stiff chains: 1024 x N=500 as cfg5-cheb with the Cholesky square root (blocked; FP64 "
                  "tensor-core trailing updates in the mixed form)", 1024, 1),
}


def other_workload(torch, name, steps, warmup, forms, n_chains=None):
    """One JSON line for a non-headline configuration: chain-steps/s of each
    form over `steps` timed chunks (CUDA events on the launch stream, L2
    flushed between chunks)."""
    import bdsim_b200 as B
    from bdsim_b200 import workloads
    from bdsim_b200._abi import CACHE_PERSIST
    from bdsim_b200.params import DelSMethod
    desc, n, chunk = OTHER_WORKLOADS[name]
    n = n_chains or n
    if name == "cfg3":
        phys, sims, Rs, seeds = workloads.uneven_wlc(n, seed=0)
    else:
        method = DelSMethod.Cholesky if name == "cfg5-chol" else DelSMethod.Chebyshev
        phys, sims, Rs, seeds = workloads.stiff_large(n, 0, 500, method)
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {}
    for form in forms:
        with torch.cuda.stream(stream):
            ens = B.Ensemble(phys, sims, Rs, [(1, -1, s) for s in seeds], form=form)
            tuned = ens.autotune() if name == "cfg3" else None
            dt = np.array([s.dt for s in sims])
            t = np.array([s.time_start for s in sims])
            for _ in range(warmup):
                ens.advance(t, chunk, CACHE_PERSIST)
                t = t + chunk * dt
            stream.synchronize()
            c0 = ens.counter_totals()
            ms = []
            for _ in range(steps):
                flush_l2(torch, flush)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ens.advance(t, chunk, CACHE_PERSIST)
                e1.record(stream)
                t = t + chunk * dt
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            c1 = ens.counter_totals()
            out[form] = {"value": n * chunk * steps / (sum(ms) * 1e-3), "ms_per_chunk": float(np.mean(ms)),
                         "failed": int(ens.failed().sum()), "plan": ens.plan(), "tuned": tuned,
                         "counters_per_step": {k: (c1[k] - c0[k]) / max(c1["steps"] - c0["steps"], 1) for k in c1}}
        del ens
    line = {"metric": "chain-steps/sec", "workload": name, "value": out.get("mixed", out[forms[0]])["value"],
            "unit": "chain-steps/s", "n_gpus": 1, "steps": steps, "warmup": warmup, "chunk_steps": chunk,
            "higher_is_better": True, "data": "synthetic", "config": {"workload": desc, "n_chains": n},
            "forms": out}
    if "mixed" in out and "plain" in out:
        line["mixed_over_plain"] = out["mixed"]["value"] / out["plain"]["value"]
    print(json.dumps(line))
    return 0


def cpu_reference(seconds_target=15.0, threads=None):
    """The reference C++ step (oracle/_ref, compiled from the reference
    sources; the C restatement when that library is absent) on the host
    cores, on a bounded sample of the workload."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    orc = O.ref() if kind == "reference" else O.port()
    threads = threads or (os.cpu_count() or 1)
    phys, sim = make_phys()
    # calibrate on one chain
    R1 = make_chains(0, 1)
    s = type(sim)()
    s.dt, s.time_start, s.time_end = DT, 0.0, 19 * DT
    t0 = time.perf_counter()
    orc.integrate_many(R1, [phys], [s], [(1, -1, 0)], 1)
    per_step = (time.perf_counter() - t0) / 20.0
    steps = CHUNK
    chains = max(threads, int(seconds_target / max(per_step * steps, 1e-9)))
    chains = int(np.ceil(chains / threads) * threads)
    chains = min(chains, N_CHAINS)
    Rs = make_chains(0, chains)
    s.time_end = (steps - 1) * DT
    t0 = time.perf_counter()
    _, _, status = orc.integrate_many(Rs, [phys] * chains, [s] * chains, [(1, -1, i) for i in range(chains)], threads)
    wall = time.perf_counter() - t0
    return {"value": chains * steps / wall, "unit": "chain-steps/s", "cores": threads, "kind": kind,
            "wall_s": wall,
            "sample": f"{chains} of the {N_CHAINS} chains x {steps} steps (one chunk, cold Lanczos start), "
                      f"{threads} threads, {wall:.1f} s wall"}


def flops_per_chain_step(counters):
    n = 3 * N_BEADS
    steps = max(counters["steps"], 1)
    dx = counters["dx_products"] / steps
    pairs = N_BEADS * (N_BEADS - 1) / 2
    return dx * 2.0 * n * n + 2 * pairs * C_EV + pairs * C_RPY, dx


def measure_peak(fp64):
    path = os.path.join(ROOT, "bdsim_b200", "libbdsim_peak.so")
    lib = ctypes.CDLL(path)
    lib.bdpk_fma_tflops.restype = ctypes.c_double
    lib.bdpk_fma_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    return max(lib.bdpk_fma_tflops(int(fp64), 200000) for _ in range(3))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer e2e leg (profiling runs)")
    ap.add_argument("--chains", type=int, default=None,
                    help="chains per GPU (default: the workload's; profiling runs use fewer)")
    ap.add_argument("--forms", default="plain,mixed", help="integrator forms to time")
    ap.add_argument("--workload", default="cfg2", choices=["cfg2"] + sorted(OTHER_WORKLOADS),
                    help="cfg2 (default): the headline line; others print their own line")
    ap.add_argument("--serving-seconds", type=float, default=60.0,
                    help="length of the serving replay (0: skip it)")
    ap.add_argument("--team-shape", default=None,
                    help="mixed form: pin the team shape 'warps,beads_per_thread' instead of autotuning (profiling)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        steps, warmup = args.steps, args.warmup
        vals, walls = [], []
        base = None
        for i in range(warmup + steps):
            r = cpu_reference(seconds_target=10.0)
            if i >= warmup:
                vals.append(r["value"])
                walls.append(r["wall_s"])
                base = r
        v = float(np.median(vals))
        # a step of this arm is one bounded sample of the workload (a subset of
        # the chains for one 100-step chunk); ms_per_step is its measured wall time
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "chain-steps/s", "n_gpus": args.gpus,
                "steps": steps, "warmup": warmup, "ms_per_step": float(np.median(walls)) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD_SHORT, "chunk_steps": CHUNK, "n_chains_per_gpu": N_CHAINS,
                           "step": base["sample"]},
                "cpu_baseline": {"value": v, "unit": "chain-steps/s", "cores": base["cores"], "kind": base["kind"],
                                 "sample": base["sample"]},
                "e2e": {"value": v, "unit": "chain-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    torch.cuda.set_device(local)
    if args.workload != "cfg2":
        if rank != 0:
            return 0
        return other_workload(torch, args.workload, args.steps, args.warmup,
                              [f for f in args.forms.split(",") if f], args.chains)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    phys, sim = make_phys()
    from bdsim_b200.sharding import reduce_max, shard_bounds
    n_chains = args.chains or N_CHAINS
    # weak scaling: world shards of n_chains each, the global chain index is
    # the seed, so the shards together are the single-GPU ensemble of
    # world * n_chains chains
    first, _ = shard_bounds(np.ones(world * n_chains), world)[rank]
    Rs = make_chains(first, n_chains)
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    results = {}
    clocks = None
    forms = [f for f in args.forms.split(",") if f]
    shape = tuple(int(v) for v in args.team_shape.split(",")) if args.team_shape else None
    for form in forms:
        barrier()
        sampler = ClockSampler(local) if form == "mixed" else None
        if sampler:
            sampler.start()
        r = run_form(torch, form, Rs, phys, sim, args.steps, args.warmup, first, stream, team_shape=shape)
        if sampler:
            clocks = sampler.stop()
        barrier()
        r["total_ms"] = reduce_max(sum(r["ms"]), dist, device="cuda")
        results[form] = r

    if set(forms) == {"plain", "mixed"}:
        # the persistent-bounds policy: spectral bounds kept for 4 steps
        barrier()
        r = run_form(torch, "mixed", Rs, phys, sim, args.steps, args.warmup, first, stream, bounds_every=4,
                     team_shape=shape)
        barrier()
        r["total_ms"] = reduce_max(sum(r["ms"]), dist, device="cuda")
        results["mixed_k4"] = r
    # (the same chunks of the same chains as the device-resident leg: a step's
    # cost depends on how far the chains have relaxed)
    # and the team shape the device leg ran with
    e2e_shape = next((sh for sh in results.get("mixed", {}).get("shape", []) if len(sh) == 2), None)
    e2e = None if args.no_e2e else run_e2e(torch, Rs, phys, sim, args.steps, max(3, args.warmup), first, "mixed",
                                           team_shape=e2e_shape)
    serving = light = None
    if args.serving_seconds > 0 and set(forms) == {"plain", "mixed"}:
        # the serving configuration as stated (overload), then a lighter stream
        # of the same job mix that one GPU serves to completion
        serving = run_serving(torch, args.serving_seconds, seed=rank)
        light = run_serving(torch, LIGHT["horizon"], scale_steps=LIGHT["scale_steps"], rate=LIGHT["rate"],
                            seed=rank + 1, drain=True, drain_limit=LIGHT["drain_limit"])

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    def rate(r):
        return world * n_chains * CHUNK * args.steps / (r["total_ms"] * 1e-3)

    if set(forms) != {"plain", "mixed"}:
        # profiling run: one line per form, no headline
        for f in forms:
            print(json.dumps({"form": f, "chain_steps_per_s": rate(results[f]), "ms": results[f]["ms"],
                              "counters": results[f]["counters"]}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    mixed, plain = results["mixed"], results["plain"]
    fl_m, dx_m = flops_per_chain_step(mixed["counters"])
    fl_p, dx_p = flops_per_chain_step(plain["counters"])
    launch_ms = float(np.mean(mixed["ms"]))
    peak32 = measure_peak(False)
    peak64 = measure_peak(True)
    # algorithmic work: the reference algorithm's products (counted by the
    # plain form, which performs exactly those); the mixed form merges one of
    # them by linearity, so its own count (dx_m) is lower
    achieved = n_chains * CHUNK * fl_p / (launch_ms * 1e-3) / 1e12
    achieved_p = n_chains * CHUNK * fl_p / (float(np.mean(plain["ms"])) * 1e-3) / 1e12
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get("mixed_bytes_per_launch")
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_reference()
            cpu.pop("wall_s", None)  # stated in the sample
        except Exception as exc:  # reported, not fatal
            cpu = {"error": str(exc)}
    ens_m = compare_observables(mixed["obs"], plain["obs"])
    ens_k4 = compare_observables(results["mixed_k4"]["obs"], plain["obs"])
    # detail lines first; the headline line (last, compact) repeats the key figures
    print(json.dumps({"detail": "ensemble_mixed_vs_plain", **ens_m,
                      "steps_per_chain": (args.warmup + args.steps) * CHUNK, "n_chains": n_chains,
                      "note": "final state of each form from the same initial chains and seeds"}))
    print(json.dumps({"detail": "mixed_bounds_every_4", "value": rate(results["mixed_k4"]), "unit": "chain-steps/s",
                      "dx_per_step": flops_per_chain_step(results["mixed_k4"]["counters"])[1],
                      "ensemble_vs_plain": ens_k4,
                      "policy": "spectral bounds kept for 4 steps, refreshed early when a step's Chebyshev check "
                                "fails on them (bdcu_set_bounds_refresh; not the reference's policy)"}))
    print(json.dumps({"detail": "roofline", "flops_per_chain_step": fl_p, "dx_per_step_algorithm": dx_p,
                      "dx_per_step_mixed": dx_m, "fp32_fma_peak_tflops": peak32, "fp64_fma_peak_tflops": peak64,
                      "plain_tflops_dense_equiv": achieved_p, "plain_frac_of_fp64_peak": achieved_p / peak64,
                      "mixed_team_shape_autotuned": mixed["shape"], "plain_block": plain["shape"],
                      "hbm_peak_gbs_measured": _peaks().get("hbm_gbs"),
                      "peak_source": "FMA-loop kernels (libbdsim_peak.so) timed in this run; the integrator runs "
                                     "on CUDA cores, neither HBM- nor tensor-bound"}))
    for name, st in (("serving_overload", serving), ("serving_light", light)):
        if st is not None:
            print(json.dumps({"detail": name, **st}))
    print(json.dumps({"detail": "serving_workload", "overload": SERVING_WORKLOAD,
                      "light": f"the same job mix with n_steps x{LIGHT['scale_steps']} (min 100), "
                               f"{LIGHT['rate']} jobs/s for {LIGHT['horizon']} s, drained for up to {LIGHT['drain_limit']} s "
                               "(jobs still running then are censored samples)"}))

    def lat(st):
        if st is None:
            return None
        return {"p50_s": _r(st["p50_latency_s"]), "p99_s": _r(st["p99_latency_s"]), "n": st["n_latency_samples"],
                "p50_lb_s": _r(st["p50_latency_lower_bound_s"]), "p99_lb_s": _r(st["p99_latency_lower_bound_s"]),
                "n_all": st["n_admitted_samples"], "chain_steps_per_s": _r(st["chain_steps_per_s"])}

    line = {
        "metric": METRIC,
        "value": rate(mixed),
        "unit": "chain-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mixed["total_ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64 (mixed)",
        "data": "synthetic",
        "plain_fp64": {"value": rate(plain), "ms_per_step": plain["total_ms"] / args.steps},
        "mixed_over_plain": rate(mixed) / rate(plain),
        "config": {"workload": WORKLOAD_SHORT, "form": "mixed", "chunk_steps": CHUNK, "n_chains_per_gpu": n_chains,
                   "cache": "cold per chunk", "l2": "flushed (256 MiB write) between timed chunks",
                   "parallelism": f"trajectory shards x{world}", "plain_fp64_value": rate(plain),
                   "mixed_over_plain": rate(mixed) / rate(plain)},
        "roofline": {"bound": "fp32-simt", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                     "frac": achieved / peak32, "traffic": traffic},
        "e2e": None if e2e is None else {
            "value": e2e[0], "unit": "chain-steps/s", "h2d_bytes_per_step": e2e[1], "d2h_bytes_per_step": e2e[2]},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "failed_chains": {"mixed": mixed["failed"], "plain": plain["failed"]},
        "ensemble_sigma": {"rg2": _r(ens_m["rg2"]["diff_in_sigma"]), "tau_xy": _r(ens_m["tau_xy"]["diff_in_sigma"])},
        "latency": {"overload": lat(serving), "light": lat(light)},
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _r(v, digits=4):
    """v to `digits` significant digits (None stays None)."""
    return None if v is None else float(f"{v:.{digits}g}")


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


if __name__ == "__main__":
    sys.exit(main())
