"""ctypes view of the C ABI in include/bdsim_cuda.h and the parameter packer.

`pack_batch` turns per-chain (PhysParams, SimParams) into the bdcu_phys /
bdcu_sim record arrays and the shared double arena the ABI takes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import PhysParams, SimParams, external_entries

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)

# status bits (bdsim_cuda.h)
ST_NONCONVERGED = 1
ST_NOT_PD = 2
ST_CHEB_FALLBACK = 4
ST_RTSAFE_FAIL = 8
ST_NONFINITE = 16
ST_BAD_PARAM = 32
ST_TIMEOUT = 64
ST_FATAL_MASK = ST_NOT_PD | ST_RTSAFE_FAIL | ST_NONFINITE | ST_BAD_PARAM | ST_TIMEOUT

FORM_PLAIN_FP64 = 0
FORM_MIXED_FP32 = 1
CACHE_RESET_PER_CALL = 0
CACHE_PERSIST = 1

STATUS_NAMES = {
    ST_NONCONVERGED: "corrector did not converge",
    ST_NOT_PD: "cholesky_lower: matrix is not positive definite",
    ST_CHEB_FALLBACK: "Chebyshev fluctuation-dissipation check failed (Cholesky fallback)",
    ST_RTSAFE_FAIL: "rtsafe failed (root not bracketed or max iterations)",
    ST_NONFINITE: "bead positions became non-finite",
    ST_BAD_PARAM: "invalid parameter (WLCbounded sigma > 1 or ExactSqrt)",
    ST_TIMEOUT: "a bounded wait inside the kernel gave up (tile staging)",
}


class BdcuPhys(ctypes.Structure):
    _fields_ = [
        ("n_beads", ctypes.c_int32),
        ("spring_type", ctypes.c_int32),
        ("sqrtb", ctypes.c_double),
        ("natural_length", ctypes.c_double),
        ("ev_type", ctypes.c_int32),
        ("contour_dist_for_ev", ctypes.c_int32),
        ("zstar", ctypes.c_double),
        ("dstar", ctypes.c_double),
        ("min_cutoff", ctypes.c_double),
        ("max_cutoff", ctypes.c_double),
        ("phi_offset", ctypes.c_int64),
        ("bend_type", ctypes.c_int32),
        ("equilibration", ctypes.c_int32),
        ("bend_stiffness", ctypes.c_double),
        ("hstar", ctypes.c_double),
        ("hi_method", ctypes.c_int32),
        ("flow_n_times", ctypes.c_int32),
        ("ncheb_multiplier", ctypes.c_double),
        ("fd_err_max", ctypes.c_double),
        ("flow_kappa", ctypes.c_double * 9),
        ("flow_offset", ctypes.c_int64),
        ("ext_n_entries", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
        ("ext_offset", ctypes.c_int64),
    ]


class BdcuSim(ctypes.Structure):
    _fields_ = [
        ("time_start", ctypes.c_double),
        ("time_end", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("implicit_loop_tol", ctypes.c_double),
        ("update_center_of_mass", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
    ]


class BdcuCounters(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "steps", "dx_products", "cheb_terms", "corrector_iters",
        "lanczos_cold", "lanczos_warm", "cheb_fallbacks", "nonconverged")]


COUNTER_FIELDS = [f[0] for f in BdcuCounters._fields_]


class BdcuBucketInfo(ctypes.Structure):
    """One bucket of a launch plan (bdcu_bucket_info)."""
    _fields_ = [(k, ctypes.c_int32) for k in (
        "bucket", "kernel", "team_warps", "n_chains", "min_beads", "max_beads", "block", "grid", "v_cap",
        "d_in_smem", "tuned", "team_beads_per_thread")] + [("smem_bytes", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BdcuQueueConfig(ctypes.Structure):
    """bdcu_queue_config: the serving queue's pool and policy."""
    _fields_ = [("form", ctypes.c_int32), ("policy", ctypes.c_int32), ("max_chains", ctypes.c_int32),
                ("max_active_chains", ctypes.c_int32), ("bead_capacity", ctypes.c_int64),
                ("arena_capacity", ctypes.c_int64), ("queue_limit", ctypes.c_int32), ("lookahead", ctypes.c_int32),
                ("slice_steps", ctypes.c_int32), ("cache_mode", ctypes.c_int32), ("slice_budget_ns", ctypes.c_int64),
                ("worker", ctypes.c_int32), ("reserved0", ctypes.c_int32)]


class BdcuJob(ctypes.Structure):
    """bdcu_job: one simulate call's chains for the serving queue."""
    _fields_ = [("n_traj", ctypes.c_int32), ("snapshots", ctypes.c_int32), ("n_steps", ctypes.c_int64),
                ("write_every", ctypes.c_int64), ("tag", ctypes.c_int64), ("phys", BdcuPhys), ("sim", BdcuSim),
                ("arena", ctypes.POINTER(ctypes.c_double)), ("arena_len", ctypes.c_int64),
                ("R0", ctypes.POINTER(ctypes.c_double)), ("rng", ctypes.POINTER(ctypes.c_int32))]


class BdcuQueueEvent(ctypes.Structure):
    """bdcu_queue_event: a snapshot, a completion or a rejection."""
    _fields_ = [("kind", ctypes.c_int32), ("n_traj", ctypes.c_int32), ("n_beads", ctypes.c_int32),
                ("snapshot", ctypes.c_int32), ("job", ctypes.c_int64), ("tag", ctypes.c_int64),
                ("step", ctypes.c_int64), ("time", ctypes.c_double), ("t_arrival", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("counters", BdcuCounters)]


class BdcuQueueStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "submitted", "rejected", "queued", "running", "done", "active_chains", "chain_steps", "slices",
        "selected_chains", "pending_events")] + [("device_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


QUEUE_FIFO, QUEUE_SJF = 0, 1
QEV_SNAPSHOT, QEV_DONE, QEV_REJECTED = 1, 2, 3


class _Arena:
    def __init__(self):
        self.chunks = []
        self.size = 0
        self._memo = {}

    def add(self, values, key=None):
        if key is not None and key in self._memo:
            return self._memo[key]
        arr = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        off = self.size
        self.chunks.append(arr)
        self.size += arr.size
        if key is not None:
            self._memo[key] = off
        return off

    def array(self):
        if not self.chunks:
            return np.zeros(1, dtype=np.float64)
        return np.concatenate(self.chunks)


def _code(v) -> int:
    """Integer code of an enum value: this package's IntEnums, or the
    reference's nanobind enums (enum.Enum subclasses whose int is `.value`)."""
    return int(getattr(v, "value", v))


def _fill_phys(rec: BdcuPhys, phys: PhysParams, n_beads: int, arena: _Arena):
    rec.n_beads = int(n_beads)
    rec.spring_type = _code(phys.spring.type)
    rec.sqrtb = float(phys.spring.sqrtb)
    rec.natural_length = float(phys.spring.natural_length)
    ev = phys.ev
    rec.ev_type = _code(ev.type)
    rec.contour_dist_for_ev = int(ev.contour_dist_for_EV)
    rec.zstar = float(ev.zstar)
    rec.dstar = float(ev.dstar)
    rec.min_cutoff = float(ev.min_cutoff)
    rec.max_cutoff = float(ev.max_cutoff)
    rec.phi_offset = -1
    if len(ev.phi) > 0:
        phi = np.asarray(ev.phi, dtype=np.float64).reshape(-1)
        if phi.size != n_beads * n_beads:
            raise ValueError(f"EVParams.phi must hold N*N={n_beads * n_beads} values, got {phi.size}")
        rec.phi_offset = arena.add(phi, key=("phi", phi.tobytes()))
    rec.bend_type = _code(phys.bend.type)
    rec.equilibration = int(bool(phys.equilibration))
    rec.bend_stiffness = float(phys.bend.stiffness)
    rec.hstar = float(phys.hstar)
    rec.hi_method = _code(phys.hi_method)
    rec.ncheb_multiplier = float(phys.ncheb_multiplier)
    rec.fd_err_max = float(phys.fd_err_max)
    # Flow and ExternalForce are read through their pickled state, whose layout
    # this package shares with the reference's nanobind objects
    # (bindings/module.cpp:83-99 and 140-148), so either package's objects pack.
    constant, k0, times, ks = phys.flow.__getstate__()
    for i, v in enumerate(np.asarray(k0, dtype=np.float64).reshape(-1)):
        rec.flow_kappa[i] = float(v)
    times = np.asarray(times, dtype=np.float64).reshape(-1)
    ks = np.asarray(ks, dtype=np.float64).reshape(-1)
    if constant or times.size == 0:
        rec.flow_n_times = 0
        rec.flow_offset = 0
    else:
        rec.flow_n_times = int(times.size)
        rec.flow_offset = arena.add(np.concatenate([times, ks]), key=("flow", times.tobytes(), ks.tobytes()))
    ents = list(external_entries(phys.external.__getstate__()))
    rec.ext_n_entries = len(ents)
    rec.ext_offset = 0
    if ents:
        buf = []
        for bead, is_const, val, times, vals in ents:
            n = len(times)
            buf += [float(bead), 1.0 if is_const else 0.0, *val, float(n), *times]
            for v in vals:
                buf += list(v)
        rec.ext_offset = arena.add(np.array(buf), key=("ext", tuple(buf)))


def _fill_sim(rec: BdcuSim, sim: SimParams):
    rec.time_start = float(sim.time_start)
    rec.time_end = float(sim.time_end)
    rec.dt = float(sim.dt)
    rec.implicit_loop_tol = float(sim.implicit_loop_tol)
    rec.update_center_of_mass = int(bool(sim.update_center_of_mass))


def pack_batch(phys_list, sim_list, n_beads_list):
    """-> (phys_array ctypes, sim_array ctypes, arena float64 ndarray)."""
    n = len(phys_list)
    if not (len(sim_list) == n == len(n_beads_list)):
        raise ValueError("phys, sim and n_beads lists must have equal length")
    arena = _Arena()
    phys_arr = (BdcuPhys * max(n, 1))()
    sim_arr = (BdcuSim * max(n, 1))()
    # chains that share a PhysParams object (and a bead count) share its
    # record and its arena tables (flow and force samples, the N x N SDK phi)
    first = {}
    for i in range(n):
        key = (id(phys_list[i]), int(n_beads_list[i]))
        j = first.get(key)
        if j is None:
            _fill_phys(phys_arr[i], phys_list[i], n_beads_list[i], arena)
            first[key] = i
        else:
            phys_arr[i] = phys_arr[j]
        _fill_sim(sim_arr[i], sim_list[i])
    return phys_arr, sim_arr, arena.array()


def count_steps(sim: SimParams) -> int:
    """Steps the reference loop `for (t = t0; t <= t1 + dt/2; t += dt)`
    takes (src/integrator.cpp:67), replayed in double arithmetic."""
    t, t1, dt = float(sim.time_start), float(sim.time_end), float(sim.dt)
    if not dt > 0.0:
        raise ValueError("dt must be positive")
    lim = t1 + dt / 2.0
    n = 0
    while t <= lim:
        n += 1
        t += dt
    return n


def dptr(a) -> ctypes.c_void_p:
    """Raw pointer of a numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


_LIB = None
LIB_NAME = "libbdsim_cuda.so"


def lib_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)


def load_library():
    """Load the CUDA integrator library. Raises if it was not built: there is
    no CPU fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError(
            f"bdsim_b200: the CUDA integrator library {path} is missing; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (or `make -C bdsim_b200/csrc`). "
            "There is no CPU fallback.")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.bdcu_version.restype = ctypes.c_char_p
    lib.bdcu_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    lib.bdcu_destroy.argtypes = [vp]
    lib.bdcu_set_stream.argtypes = [vp, vp]
    lib.bdcu_set_bounds_refresh.argtypes = [vp, ctypes.c_int]
    lib.bdcu_observables.argtypes = [vp, vp, vp, vp]
    lib.bdcu_last_error.argtypes = [vp]
    lib.bdcu_last_error.restype = ctypes.c_char_p
    lib.bdcu_set_chains.argtypes = [vp, ctypes.c_int, ctypes.POINTER(BdcuPhys), ctypes.POINTER(BdcuSim),
                                    c_double_p, ctypes.c_int64]
    lib.bdcu_count_steps.argtypes = [ctypes.POINTER(BdcuSim), c_int64_p]
    lib.bdcu_run.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]
    lib.bdcu_run_slice.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                   vp, vp]
    lib.bdcu_integrate_host.argtypes = [vp, c_double_p, c_int32_p, c_int32_p,
                                        ctypes.POINTER(BdcuCounters), ctypes.c_int]
    lib.bdcu_total_force.argtypes = [vp, vp, vp]
    lib.bdcu_forces.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int, vp]
    lib.bdcu_ran1.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp]
    lib.bdcu_run_static.argtypes = [vp, ctypes.c_int, ctypes.POINTER(BdcuPhys), ctypes.POINTER(BdcuSim), c_double_p,
                                    ctypes.c_int64, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]
    lib.bdcu_describe_plan.argtypes = [vp, ctypes.c_int, ctypes.POINTER(BdcuBucketInfo), ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int)]
    lib.bdcu_autotune.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int]
    lib.bdcu_reserve.argtypes = [vp, ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
    lib.bdcu_update_chains.argtypes = [vp, ctypes.c_int, c_int32_p, ctypes.POINTER(BdcuPhys),
                                       ctypes.POINTER(BdcuSim), c_int64_p]
    lib.bdcu_write_arena.argtypes = [vp, ctypes.c_int64, c_double_p, ctypes.c_int64]
    lib.bdcu_select.argtypes = [vp, ctypes.c_int, c_int32_p]
    lib.bdcu_set_team_shape.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.bdcu_set_single_launch.argtypes = [vp, ctypes.c_int]
    lib.bdcu_check_chains.argtypes = [ctypes.c_int, ctypes.POINTER(BdcuPhys), ctypes.POINTER(BdcuSim), c_double_p,
                                      ctypes.c_int64, ctypes.c_char_p, ctypes.c_int]
    qp = ctypes.POINTER(BdcuQueueEvent)
    lib.bdcu_queue_create.argtypes = [ctypes.c_int, ctypes.POINTER(BdcuQueueConfig), ctypes.POINTER(vp)]
    lib.bdcu_queue_destroy.argtypes = [vp]
    lib.bdcu_queue_last_error.argtypes = [vp]
    lib.bdcu_queue_last_error.restype = ctypes.c_char_p
    lib.bdcu_queue_submit.argtypes = [vp, ctypes.POINTER(BdcuJob), c_int64_p, ctypes.POINTER(ctypes.c_int)]
    lib.bdcu_queue_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    lib.bdcu_queue_wait_idle.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]
    lib.bdcu_queue_poll.argtypes = [vp, qp, c_double_p, ctypes.c_int64, c_int32_p, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int)]
    lib.bdcu_queue_get_stats.argtypes = [vp, ctypes.POINTER(BdcuQueueStats)]
    for name in ("bdcu_queue_create", "bdcu_queue_destroy", "bdcu_queue_submit", "bdcu_queue_step",
                 "bdcu_queue_wait_idle", "bdcu_queue_poll", "bdcu_queue_get_stats"):
        getattr(lib, name).restype = ctypes.c_int
    for name in ("bdcu_set_single_launch", "bdcu_set_team_shape", "bdcu_check_chains", "bdcu_create", "bdcu_destroy", "bdcu_set_stream", "bdcu_set_chains",
                 "bdcu_count_steps", "bdcu_run", "bdcu_integrate_host", "bdcu_total_force",
                 "bdcu_forces", "bdcu_ran1", "bdcu_run_static", "bdcu_describe_plan", "bdcu_autotune",
                 "bdcu_reserve", "bdcu_update_chains", "bdcu_write_arena", "bdcu_select"):
        getattr(lib, name).restype = ctypes.c_int
    _LIB = lib
    return lib


# Symbols include/bdsim_cuda.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = [
    "bdcu_version", "bdcu_create", "bdcu_destroy", "bdcu_set_stream", "bdcu_last_error",
    "bdcu_set_chains", "bdcu_count_steps", "bdcu_run", "bdcu_integrate_host",
    "bdcu_total_force", "bdcu_forces", "bdcu_ran1", "bdcu_describe_plan", "bdcu_autotune",
    "bdcu_reserve", "bdcu_update_chains", "bdcu_write_arena", "bdcu_select", "bdcu_run_static",
    "bdcu_check_chains", "bdcu_set_team_shape", "bdcu_set_single_launch",
    "bdcu_queue_create", "bdcu_queue_destroy", "bdcu_queue_last_error", "bdcu_queue_submit",
    "bdcu_queue_step", "bdcu_queue_wait_idle", "bdcu_queue_poll", "bdcu_queue_get_stats",
]


def check_records(n, phys_arr, sim_arr, arena):
    """bdcu_check_chains on packed records (no GPU needed) -> (status, message)."""
    lib = load_library()
    msg = ctypes.create_string_buffer(512)
    rc = lib.bdcu_check_chains(n, phys_arr, sim_arr, arena.ctypes.data_as(c_double_p), arena.size, msg, 512)
    return rc, msg.value.decode()

KERNEL_BLOCK, KERNEL_TEAM = 0, 1
MAX_BUCKETS = 8

F_SPRING, F_EV, F_BEND, F_EXTERNAL = 1, 2, 4, 8
