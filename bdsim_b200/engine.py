"""Device-side engine over the C ABI (include/bdsim_cuda.h).

`Context` wraps one bdcu_ctx. `Ensemble` keeps a batch of chains resident on
the GPU -- positions, RNG streams, spectral warm-start vectors, status and
counters in torch device tensors -- and advances them chunk by chunk, which is
how `simulate` / `run_ensemble` use it. PyTorch provides the device buffers
and the stream; every computation is a CUDA kernel of libbdsim_cuda.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import (BdcuCounters, CACHE_PERSIST, CACHE_RESET_PER_CALL, COUNTER_FIELDS, FORM_MIXED_FP32,
                   FORM_PLAIN_FP64, ST_FATAL_MASK, dptr)

FORMS = {"plain": FORM_PLAIN_FP64, "fp64": FORM_PLAIN_FP64, "mixed": FORM_MIXED_FP32, "fp32": FORM_MIXED_FP32,
         FORM_PLAIN_FP64: FORM_PLAIN_FP64, FORM_MIXED_FP32: FORM_MIXED_FP32}


def form_code(form) -> int:
    try:
        return FORMS[form]
    except KeyError:
        raise ValueError(f"unknown integrator form {form!r} (use 'plain' or 'mixed')") from None


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("bdsim_b200 needs a CUDA device (B200); none is visible. There is no CPU fallback.")
    return torch


class BdcuError(RuntimeError):
    pass


class Context:
    """One C-ABI context on `device`, bound to the current torch stream."""

    def __init__(self, device: int = 0):
        torch = _torch()
        self.lib = _abi.load_library()
        self.device = int(device)
        self.torch = torch
        h = ctypes.c_void_p()
        rc = self.lib.bdcu_create(self.device, ctypes.byref(h))
        if rc != 0:
            raise BdcuError(f"bdcu_create failed ({rc})")
        self.h = h
        self.n_chains = 0
        self.n_beads = []

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.bdcu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != 0:
            msg = self.lib.bdcu_last_error(self.h).decode(errors="replace")
            raise BdcuError(f"{what} failed ({rc}): {msg}")

    def use_stream(self, stream=None):
        torch = self.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._ck(self.lib.bdcu_set_stream(self.h, ctypes.c_void_p(s.cuda_stream)), "bdcu_set_stream")

    def set_bounds_refresh(self, every_steps: int):
        """FP32-mixed form: recompute the spectral bounds every `every_steps`
        steps (and on a failed Chebyshev check); 1 is the reference's policy."""
        self._ck(self.lib.bdcu_set_bounds_refresh(self.h, int(every_steps)), "bdcu_set_bounds_refresh")

    def set_chains(self, phys_list, sim_list, n_beads_list):
        prec, srec, arena = _abi.pack_batch(phys_list, sim_list, n_beads_list)
        self._arena = arena
        self._ck(self.lib.bdcu_set_chains(self.h, len(phys_list), prec, srec,
                                          arena.ctypes.data_as(_abi.c_double_p), arena.size),
                 "bdcu_set_chains")
        self.n_chains = len(phys_list)
        self.n_beads = list(n_beads_list)

    def run(self, R, rng, cache, cache_valid, t_start, n_steps, status, counters, form, cache_mode):
        self.use_stream()
        self._ck(self.lib.bdcu_run(self.h, dptr(R), dptr(rng), dptr(cache), dptr(cache_valid), dptr(t_start),
                                   dptr(n_steps), dptr(status), dptr(counters), int(form), int(cache_mode)),
                 "bdcu_run")

    def run_slice(self, R, rng, cache, cache_valid, t_start, n_steps, status, counters, form, cache_mode,
                  budget_ns, steps_done, t_end):
        """bdcu_run with a time budget: steps_done / t_end receive each chain's
        completed steps and time (see bdcu_run_slice)."""
        self.use_stream()
        self._ck(self.lib.bdcu_run_slice(self.h, dptr(R), dptr(rng), dptr(cache), dptr(cache_valid),
                                         dptr(t_start), dptr(n_steps), dptr(status), dptr(counters), int(form),
                                         int(cache_mode), int(budget_ns), dptr(steps_done), dptr(t_end)),
                 "bdcu_run_slice")

    def integrate_host(self, R_host: np.ndarray, rng_host: np.ndarray, form):
        """Host-buffer integrate over each chain's SimParams span (cold cache).
        R_host (total_beads, 3) float64 and rng_host (n, 3) int32 are updated
        in place. Returns (status int32[n], counters list of dicts)."""
        self.use_stream()
        status = np.zeros(self.n_chains, dtype=np.int32)
        cnt = (BdcuCounters * self.n_chains)()
        self._ck(self.lib.bdcu_integrate_host(self.h, R_host.ctypes.data_as(_abi.c_double_p),
                                              rng_host.ctypes.data_as(_abi.c_int32_p),
                                              status.ctypes.data_as(_abi.c_int32_p), cnt, int(form)),
                 "bdcu_integrate_host")
        return status, [{f: getattr(c, f) for f in COUNTER_FIELDS} for c in cnt]

    def total_force(self, R_dev, F_dev):
        self.use_stream()
        self._ck(self.lib.bdcu_total_force(self.h, dptr(R_dev), dptr(F_dev)), "bdcu_total_force")

    def forces(self, R_dev, F_dev, which: int, t: float = 0.0):
        self.use_stream()
        self._ck(self.lib.bdcu_forces(self.h, dptr(R_dev), float(t), int(which), dptr(F_dev)), "bdcu_forces")

    # ---- launch plans (buckets by bead count, autotuned shapes)

    def describe_plan(self, form) -> list:
        """The buckets bdcu_run would launch for `form` on the current selection."""
        out = (_abi.BdcuBucketInfo * _abi.MAX_BUCKETS)()
        n = ctypes.c_int(0)
        self._ck(self.lib.bdcu_describe_plan(self.h, form_code(form), out, _abi.MAX_BUCKETS, ctypes.byref(n)),
                 "bdcu_describe_plan")
        return [out[i].as_dict() for i in range(n.value)]

    def autotune(self, form, R, rng, cache, cache_valid, t_start, probe_steps: int = 3) -> list:
        """Time every launch shape of each bucket (block kernel: block size,
        Lanczos vectors and D in shared memory; team kernel: warps per chain
        x beads per thread) on copies of the given state and keep the
        fastest; returns the tuned plan. Probe from a warmed-up state (valid
        warm-start cache): probes from a cold cache are dominated by the
        first step's 30-step Lanczos run."""
        self.use_stream()
        self._ck(self.lib.bdcu_autotune(self.h, form_code(form), dptr(R), dptr(rng), dptr(cache),
                                        dptr(cache_valid), dptr(t_start), int(probe_steps)), "bdcu_autotune")
        return self.describe_plan(form)

    def set_team_shape(self, bucket: int, team_warps: int, beads_per_thread: int = 2):
        """Pin the FP32-mixed form's team shape for team bucket 0..3 (warps
        per chain, beads per thread); team_warps=0 restores the default."""
        self._ck(self.lib.bdcu_set_team_shape(self.h, int(bucket), int(team_warps), int(beads_per_thread)),
                 "bdcu_set_team_shape")

    def set_single_launch(self, on: bool = True):
        """All team-kernel chains in one persistent launch (the widest team
        bucket's shape) instead of one launch per bucket."""
        self._ck(self.lib.bdcu_set_single_launch(self.h, int(bool(on))), "bdcu_set_single_launch")

    # ---- slot pools (serving)

    def reserve(self, n_slots: int, bead_capacity: int, arena_len: int = 0):
        self.use_stream()
        self._ck(self.lib.bdcu_reserve(self.h, int(n_slots), int(bead_capacity), int(arena_len)), "bdcu_reserve")
        self.n_chains = int(n_slots)

    def update_chains(self, slots, phys_recs, sim_recs, bead_offs):
        """Fill pool slots: `phys_recs`/`sim_recs` are ctypes arrays of
        BdcuPhys/BdcuSim (offsets into the context arena already set)."""
        self.use_stream()
        slots = np.ascontiguousarray(slots, dtype=np.int32)
        offs = np.ascontiguousarray(bead_offs, dtype=np.int64)
        self._ck(self.lib.bdcu_update_chains(self.h, len(slots), slots.ctypes.data_as(_abi.c_int32_p), phys_recs,
                                             sim_recs, offs.ctypes.data_as(_abi.c_int64_p)), "bdcu_update_chains")

    @staticmethod
    def pack_slots(phys_list, sim_list, n_beads_list):
        """Pack chains for fill_slots: (phys records, sim records, arena
        doubles they need -- None when they need none)."""
        n = len(phys_list)
        same = n > 1 and all(p is phys_list[0] for p in phys_list) and all(s is sim_list[0] for s in sim_list) \
            and all(k == n_beads_list[0] for k in n_beads_list)
        if same:
            # one ensemble: pack one record and replicate it
            p1, s1, arena = _abi.pack_batch(phys_list[:1], sim_list[:1], n_beads_list[:1])
            prec = (_abi.BdcuPhys * n)()
            srec = (_abi.BdcuSim * n)()
            ctypes.memmove(prec, ctypes.byref(p1[0]), ctypes.sizeof(_abi.BdcuPhys))
            ctypes.memmove(srec, ctypes.byref(s1[0]), ctypes.sizeof(_abi.BdcuSim))
            for dst, size in ((prec, ctypes.sizeof(_abi.BdcuPhys)), (srec, ctypes.sizeof(_abi.BdcuSim))):
                filled = 1
                while filled < n:  # doubling copies
                    k = min(filled, n - filled)
                    ctypes.memmove(ctypes.addressof(dst) + filled * size, ctypes.addressof(dst), k * size)
                    filled += k
        else:
            prec, srec, arena = _abi.pack_batch(phys_list, sim_list, n_beads_list)
        uses = any(prec[i].phi_offset >= 0 or prec[i].flow_n_times > 0 or prec[i].ext_n_entries > 0
                   for i in range(min(n, 1) if same else n))
        return prec, srec, (arena if uses else None)

    def fill_slots(self, slots, phys_list, sim_list, n_beads_list, bead_offs, arena_base: int = 0,
                   packed=None) -> int:
        """Write the chains' tables into the context arena at arena_base and
        fill the pool slots. Returns the number of arena doubles used."""
        prec, srec, arena = packed if packed is not None else self.pack_slots(phys_list, sim_list, n_beads_list)
        if arena is not None:
            for i in range(len(slots)):
                r = prec[i]
                if r.phi_offset >= 0:
                    r.phi_offset += arena_base
                if r.flow_n_times > 0:
                    r.flow_offset += arena_base
                if r.ext_n_entries > 0:
                    r.ext_offset += arena_base
            self.write_arena(arena_base, arena)
        self.update_chains(slots, prec, srec, bead_offs)
        return 0 if arena is None else int(arena.size)

    def write_arena(self, offset: int, values: np.ndarray):
        self.use_stream()
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._ck(self.lib.bdcu_write_arena(self.h, int(offset), v.ctypes.data_as(_abi.c_double_p), v.size),
                 "bdcu_write_arena")

    def select(self, slots=None):
        """The chains the next runs advance (None: every chain)."""
        if slots is None:
            self._ck(self.lib.bdcu_select(self.h, 0, None), "bdcu_select")
            return
        s = np.ascontiguousarray(slots, dtype=np.int32)
        self._ck(self.lib.bdcu_select(self.h, len(s), s.ctypes.data_as(_abi.c_int32_p)), "bdcu_select")

    def ran1(self, rng_dev, n_per_chain: int, out_dev):
        self.use_stream()
        self._ck(self.lib.bdcu_ran1(self.h, int(rng_dev.shape[0]), dptr(rng_dev), int(n_per_chain),
                                    dptr(out_dev)), "bdcu_ran1")


class Ensemble:
    """A batch of independent chains resident on one GPU.

    phys_list/sim_list: one PhysParams/SimParams per chain (sim supplies dt,
    implicit_loop_tol and update_center_of_mass; the time span of each
    `advance` is given explicitly). R0_list: (N_i, 3) arrays. rng_states:
    (ix, iy, seed) per chain.
    """

    def __init__(self, phys_list, sim_list, R0_list, rng_states, device: int = 0, form="plain"):
        torch = _torch()
        self.torch = torch
        self.form = form_code(form)
        self.ctx = Context(device)
        self.n = len(R0_list)
        self.Ns = [int(len(r)) for r in R0_list]
        self.ctx.set_chains(phys_list, sim_list, self.Ns)
        self.sims = list(sim_list)
        self.offsets = np.zeros(self.n + 1, dtype=np.int64)
        self.offsets[1:] = np.cumsum(self.Ns)
        dev = torch.device("cuda", device)
        self.dev = dev
        R = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64).reshape(-1, 3) for r in R0_list]))
        self.R = torch.from_numpy(R).to(dev)
        self.rng = torch.tensor(np.asarray(rng_states, dtype=np.int32).reshape(self.n, 3), device=dev)
        self.cache = torch.zeros(3 * int(self.offsets[-1]), dtype=torch.float64, device=dev)
        self.cache_valid = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.status = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.counters = torch.zeros((self.n, len(COUNTER_FIELDS)), dtype=torch.int64, device=dev)
        self._t = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self._k = torch.zeros(self.n, dtype=torch.int32, device=dev)

    def advance(self, t_start, n_steps, cache_mode=CACHE_PERSIST):
        """Run n_steps[i] steps of chain i from time t_start[i] (asynchronous)."""
        torch = self.torch
        self._t.copy_(torch.as_tensor(np.broadcast_to(np.asarray(t_start, dtype=np.float64), (self.n,)).copy()))
        self._k.copy_(torch.as_tensor(np.broadcast_to(np.asarray(n_steps, dtype=np.int32), (self.n,)).copy()))
        self.ctx.run(self.R, self.rng, self.cache, self.cache_valid, self._t, self._k, self.status,
                     self.counters, self.form, cache_mode)

    def plan(self) -> list:
        """The launch plan of this ensemble's form: one dict per bucket."""
        return self.ctx.describe_plan(self.form)

    def autotune(self, probe_steps: int = 3, t_start=None) -> list:
        """Choose the launch shape of each bucket (block kernel, and the
        mixed form's team shape) by timing each on a copy of the current
        state (the state itself is not advanced), from time t_start (per
        chain or one value; default: each chain's SimParams.time_start).
        Call it after a first chunk so that the probes start warm."""
        t = [s.time_start for s in self.sims] if t_start is None else np.broadcast_to(t_start, (self.n,))
        self._t.copy_(self.torch.as_tensor(np.array(t, dtype=np.float64)))
        return self.ctx.autotune(self.form, self.R, self.rng, self.cache, self.cache_valid, self._t, probe_steps)

    def reset_cache(self):
        self.cache_valid.zero_()

    def positions(self):
        R = self.R.cpu().numpy()
        return [R[self.offsets[i]:self.offsets[i + 1]].copy() for i in range(self.n)]

    def total_force_device(self):
        """Total force per bead of every chain, a device tensor (total_beads, 3)
        (asynchronous on the current stream)."""
        F = self.torch.empty_like(self.R)
        self.ctx.total_force(self.R, F)
        return F

    def total_force(self):
        F = self.torch.empty_like(self.R)
        self.ctx.total_force(self.R, F)
        Fh = F.cpu().numpy()
        return [Fh[self.offsets[i]:self.offsets[i + 1]].copy() for i in range(self.n)]

    def observables(self):
        """(n, 10) per chain on the device: [Rg^2, tau_xx, tau_xy, ..., tau_zz]
        (Kramers stress with the total force, python/bdsim/properties.py)."""
        torch = self.torch
        F = torch.empty_like(self.R)
        self.ctx.total_force(self.R, F)
        out = torch.empty((self.n, 10), dtype=torch.float64, device=self.dev)
        self.ctx._ck(self.ctx.lib.bdcu_observables(self.ctx.h, dptr(self.R), dptr(F), dptr(out)), "bdcu_observables")
        return out.cpu().numpy()

    def rng_states(self):
        return [tuple(int(v) for v in row) for row in self.rng.cpu().numpy()]

    def statuses(self) -> np.ndarray:
        return self.status.cpu().numpy()

    def failed(self) -> np.ndarray:
        return (self.statuses() & ST_FATAL_MASK) != 0

    def counter_totals(self) -> dict:
        c = self.counters.sum(dim=0).cpu().numpy()
        return {f: int(v) for f, v in zip(COUNTER_FIELDS, c)}
