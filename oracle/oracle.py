"""ctypes access to the test oracles (TEST INFRASTRUCTURE ONLY).

  Port       oracle/libbd_oracle.so   the C restatement (bd_oracle.c)
  Reference  oracle/_ref/libbdref.so  the bdsim C++ core compiled from source

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module.
Parameters are packed with the product's public ABI layout
(bdsim_b200._abi.pack_batch), which both libraries read.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from bdsim_b200._abi import BdcuCounters, BdcuPhys, BdcuSim, pack_batch

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "libbd_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libbdref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_intp = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile the oracles with oracle/Makefile (the reference only where its
    sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _p(a):
    return a.ctypes.data_as(_dp)


class _Lib:
    def __init__(self, path, prefix):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        L, P = self.lib, prefix
        getattr(L, P + "ran1").argtypes = [_ip, ctypes.c_int, _dp]
        getattr(L, P + "solve_implicit_r").argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                       ctypes.c_double, _dp, _dp]
        getattr(L, P + "solve_connector").argtypes = [_dp, ctypes.c_double, ctypes.POINTER(BdcuPhys), _dp]
        getattr(L, P + "total_force").argtypes = [_dp, ctypes.c_int, ctypes.POINTER(BdcuPhys), _dp, _dp]
        getattr(L, P + "rpy_matrix").argtypes = [_dp, ctypes.c_int, ctypes.c_double, _dp]
        getattr(L, P + "cholesky").argtypes = [_dp, ctypes.c_int, _dp]
        getattr(L, P + "cholesky").restype = ctypes.c_int

    def fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def ran1(self, state, n):
        st = (ctypes.c_int32 * 3)(*state)
        out = np.zeros(n)
        self.fn("ran1")(st, n, _p(out))
        return out, (st[0], st[1], st[2])

    def solve_implicit_r(self, spring_type, dtby4, gama, natscl):
        a, b = ctypes.c_double(), ctypes.c_double()
        self.fn("solve_implicit_r")(int(spring_type), dtby4, gama, natscl, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def solve_connector(self, gamma, dt, phys):
        prec, _, arena = pack_batch([phys], [_dummy_sim()], [2])
        g = np.ascontiguousarray(gamma, dtype=np.float64)
        out = np.zeros(3)
        self.fn("solve_connector")(_p(g), dt, prec, _p(out))
        return out

    def total_force(self, R, phys):
        R = np.ascontiguousarray(R, dtype=np.float64)
        prec, _, arena = pack_batch([phys], [_dummy_sim()], [len(R)])
        F = np.zeros_like(R)
        self.fn("total_force")(_p(R), len(R), prec, _p(arena), _p(F))
        return F

    def rpy_matrix(self, R, hstar):
        R = np.ascontiguousarray(R, dtype=np.float64)
        n = 3 * len(R)
        D = np.zeros((n, n))
        self.fn("rpy_matrix")(_p(R), len(R), hstar, _p(D))
        return D

    def cholesky(self, D):
        D = np.ascontiguousarray(D, dtype=np.float64)
        L = np.zeros_like(D)
        st = self.fn("cholesky")(_p(D), D.shape[0], _p(L))
        return L, st


class PortOracle(_Lib):
    """The C restatement."""

    def __init__(self, path=PORT_PATH):
        super().__init__(path, "bdo_")
        L = self.lib
        L.bdo_spring_force.argtypes = [_dp, ctypes.c_int, ctypes.POINTER(BdcuPhys), _dp]
        L.bdo_bending_force.argtypes = [_dp, ctypes.c_int, ctypes.POINTER(BdcuPhys), _dp]
        L.bdo_ev_force.argtypes = [_dp, ctypes.c_int, ctypes.POINTER(BdcuPhys), _dp, _dp]
        L.bdo_external_force.argtypes = [ctypes.c_int, ctypes.POINTER(BdcuPhys), _dp, ctypes.c_double, _dp]
        L.bdo_kappa.argtypes = [ctypes.POINTER(BdcuPhys), _dp, ctypes.c_double, _dp]
        L.bdo_unit_bonds_and_cosines.argtypes = [_dp, ctypes.c_int, _dp, _dp]
        L.bdo_spectral_bounds.argtypes = [_dp, ctypes.c_int, _dp, _intp, _dp, _dp, _intp]
        L.bdo_chebyshev_sqrt_times.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                               _dp, _intp, _dp, _intp, _dp]
        L.bdo_integrate.argtypes = [_dp, ctypes.POINTER(BdcuPhys), ctypes.POINTER(BdcuSim), _dp, _ip,
                                    _dp, _intp, ctypes.POINTER(BdcuCounters)]
        L.bdo_integrate.restype = ctypes.c_int
        L.bdo_integrate_many.argtypes = [_dp, _i64p, ctypes.c_int, ctypes.POINTER(BdcuPhys),
                                         ctypes.POINTER(BdcuSim), _dp, _ip, _ip, ctypes.c_int]

    def _forces(self, name, R, phys, with_arena):
        R = np.ascontiguousarray(R, dtype=np.float64)
        prec, _, arena = pack_batch([phys], [_dummy_sim()], [len(R)])
        F = np.zeros_like(R)
        if with_arena:
            getattr(self.lib, name)(_p(R), len(R), prec, _p(arena), _p(F))
        else:
            getattr(self.lib, name)(_p(R), len(R), prec, _p(F))
        return F

    def spring_force(self, R, phys):
        return self._forces("bdo_spring_force", R, phys, False)

    def bending_force(self, R, phys):
        return self._forces("bdo_bending_force", R, phys, False)

    def ev_force(self, R, phys):
        return self._forces("bdo_ev_force", R, phys, True)

    def external_force(self, phys, nbeads, t):
        prec, _, arena = pack_batch([phys], [_dummy_sim()], [nbeads])
        F = np.zeros((nbeads, 3))
        self.lib.bdo_external_force(nbeads, prec, _p(arena), t, _p(F))
        return F

    def kappa(self, phys, t):
        prec, _, arena = pack_batch([phys], [_dummy_sim()], [2])
        K = np.zeros(9)
        self.lib.bdo_kappa(prec, _p(arena), t, _p(K))
        return K.reshape(3, 3)

    def unit_bonds_and_cosines(self, R):
        R = np.ascontiguousarray(R, dtype=np.float64)
        N = len(R)
        u = np.zeros((N - 1, 3))
        c = np.zeros(max(N - 2, 1))
        self.lib.bdo_unit_bonds_and_cosines(_p(R), N, _p(u), _p(c))
        return u, c[: N - 2]

    def spectral_bounds(self, D, cache=None):
        D = np.ascontiguousarray(D, dtype=np.float64)
        n = D.shape[0]
        lmin, lmax = ctypes.c_double(), ctypes.c_double()
        steps = ctypes.c_int()
        if cache is None:
            self.lib.bdo_spectral_bounds(_p(D), n, None, None, ctypes.byref(lmin), ctypes.byref(lmax),
                                         ctypes.byref(steps))
            return lmin.value, lmax.value
        vec, valid = cache
        v = ctypes.c_int(int(valid))
        self.lib.bdo_spectral_bounds(_p(D), n, _p(vec), ctypes.byref(v), ctypes.byref(lmin),
                                     ctypes.byref(lmax), ctypes.byref(steps))
        cache[1] = v.value
        return lmin.value, lmax.value

    def chebyshev_sqrt_times(self, D, x0, mult=1.0, fd_tol=0.0025):
        D = np.ascontiguousarray(D, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1)
        out = np.zeros_like(x0)
        nt, fd = ctypes.c_int(), ctypes.c_double()
        self.lib.bdo_chebyshev_sqrt_times(_p(D), D.shape[0], _p(x0), mult, fd_tol, None, None, _p(out),
                                          ctypes.byref(nt), ctypes.byref(fd))
        return out, nt.value, fd.value

    def integrate(self, R, phys, sim, rng_state, cache=None):
        """-> (R_new, rng_state_new, status, counters dict)."""
        R = np.array(R, dtype=np.float64, copy=True, order="C")
        prec, srec, arena = pack_batch([phys], [sim], [len(R)])
        st = (ctypes.c_int32 * 3)(*rng_state)
        cnt = BdcuCounters()
        if cache is None:
            status = self.lib.bdo_integrate(_p(R), prec, srec, _p(arena), st, None, None, ctypes.byref(cnt))
        else:
            vec, valid = cache
            v = ctypes.c_int(int(valid))
            status = self.lib.bdo_integrate(_p(R), prec, srec, _p(arena), st, _p(vec), ctypes.byref(v),
                                            ctypes.byref(cnt))
            cache[1] = v.value
        counters = {f: getattr(cnt, f) for f, _ in BdcuCounters._fields_}
        return R, (st[0], st[1], st[2]), status, counters

    def integrate_many(self, Rs, phys_list, sim_list, rng_states, n_threads):
        return _integrate_many(self.lib.bdo_integrate_many, Rs, phys_list, sim_list, rng_states, n_threads)


class RefOracle(_Lib):
    """The bdsim reference C++ compiled from source."""

    def __init__(self, path=REF_PATH):
        super().__init__(path, "ref_")
        L = self.lib
        L.ref_spectral_bounds.argtypes = [_dp, ctypes.c_int, _dp, _intp, _dp, _dp]
        L.ref_chebyshev_sqrt_times.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                               _dp, _intp, _dp]
        L.ref_integrate.argtypes = [_dp, ctypes.POINTER(BdcuPhys), ctypes.POINTER(BdcuSim), _dp, _ip]
        L.ref_integrate.restype = ctypes.c_int
        L.ref_integrate_many.argtypes = [_dp, _i64p, ctypes.c_int, ctypes.POINTER(BdcuPhys),
                                         ctypes.POINTER(BdcuSim), _dp, _ip, _ip, ctypes.c_int]

    def spectral_bounds(self, D, cache=None):
        D = np.ascontiguousarray(D, dtype=np.float64)
        n = D.shape[0]
        lmin, lmax = ctypes.c_double(), ctypes.c_double()
        if cache is None:
            self.lib.ref_spectral_bounds(_p(D), n, None, None, ctypes.byref(lmin), ctypes.byref(lmax))
            return lmin.value, lmax.value
        vec, valid = cache
        v = ctypes.c_int(int(valid))
        self.lib.ref_spectral_bounds(_p(D), n, _p(vec), ctypes.byref(v), ctypes.byref(lmin), ctypes.byref(lmax))
        cache[1] = v.value
        return lmin.value, lmax.value

    def chebyshev_sqrt_times(self, D, x0, mult=1.0, fd_tol=0.0025):
        D = np.ascontiguousarray(D, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1)
        out = np.zeros_like(x0)
        nt, fd = ctypes.c_int(), ctypes.c_double()
        self.lib.ref_chebyshev_sqrt_times(_p(D), D.shape[0], _p(x0), mult, fd_tol, _p(out), ctypes.byref(nt),
                                          ctypes.byref(fd))
        return out, nt.value, fd.value

    def integrate(self, R, phys, sim, rng_state):
        R = np.array(R, dtype=np.float64, copy=True, order="C")
        prec, srec, arena = pack_batch([phys], [sim], [len(R)])
        st = (ctypes.c_int32 * 3)(*rng_state)
        status = self.lib.ref_integrate(_p(R), prec, srec, _p(arena), st)
        return R, (st[0], st[1], st[2]), status

    def integrate_many(self, Rs, phys_list, sim_list, rng_states, n_threads):
        return _integrate_many(self.lib.ref_integrate_many, Rs, phys_list, sim_list, rng_states, n_threads)


def _integrate_many(fn, Rs, phys_list, sim_list, rng_states, n_threads):
    Ns = [len(R) for R in Rs]
    off = np.zeros(len(Rs) + 1, dtype=np.int64)
    off[1:] = np.cumsum(Ns)
    R = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64) for r in Rs]))
    prec, srec, arena = pack_batch(phys_list, sim_list, Ns)
    rng = np.ascontiguousarray(np.asarray(rng_states, dtype=np.int32).reshape(-1))
    status = np.zeros(len(Rs), dtype=np.int32)
    fn(_p(R), off.ctypes.data_as(_i64p), len(Rs), prec, srec, _p(arena), rng.ctypes.data_as(_ip),
       status.ctypes.data_as(_ip), int(n_threads))
    outs = [R[off[i]:off[i + 1]].copy() for i in range(len(Rs))]
    return outs, rng.reshape(-1, 3), status


def _dummy_sim():
    from bdsim_b200.params import SimParams
    return SimParams()


def port():
    return PortOracle()


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    return RefOracle()
