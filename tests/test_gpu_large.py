"""Parity of the CUDA integrator with the oracle at full chain sizes (N=100
to 500: D, the Cholesky factor and the cold Lanczos basis in global memory;
the blocked Cholesky with full and ragged panels and tiles; the team
kernel's widest teams), a few steps per call.

Tolerances as in test_gpu_parity: plain FP64 form <= 1e-10 per call
(max|R_gpu - R_oracle| / max(1, max|R_oracle|)), bit-exact RNG streams and
identical step/corrector/Lanczos counters; FP32-mixed form <= 1e-4 per call.
"""
import time

import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi
from bdsim_b200.params import Rng
from tests.golden.cases import build_large_case

pytestmark = pytest.mark.gpu

CALL_TOL = 1e-10
MIXED_TOL = 1e-4


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, float(np.max(np.abs(b)))))


CASES = [("cfg5_cholesky", 500), ("cfg5_cholesky", 250), ("cfg5_cholesky", 150), ("cfg5_cholesky", 100),
         ("cfg5_cheb", 500),
         ("cfg3_wlc_lj", 200)]


@pytest.fixture(scope="module")
def oracle_results(port):
    out = {}
    for name, N in CASES:
        R0, p, s, seed = build_large_case(name, N)
        t0 = time.perf_counter()
        out[(name, N)] = port.integrate(R0, p, s, (1, -1, seed))
        print(f"oracle {name} N={N}: {time.perf_counter() - t0:.2f} s")
    return out


@pytest.mark.parametrize("name,N", CASES)
def test_plain_full_size_matches_oracle(name, N, oracle_results):
    R0, p, s, seed = build_large_case(name, N)
    g = Rng(seed)
    t0 = time.perf_counter()
    out, status, cnt = B.integrate_many([R0], p, s, [g], form="plain")
    print(f"plain {name} N={N}: {time.perf_counter() - t0:.3f} s")
    Rw, st, pst, pcnt = oracle_results[(name, N)]
    assert int(status[0]) == int(pst)
    assert g.state() == st
    assert rel(out[0], Rw) <= CALL_TOL
    for k in ("steps", "corrector_iters", "lanczos_cold", "lanczos_warm", "cheb_fallbacks"):
        assert cnt[0][k] == pcnt[k], k


@pytest.mark.parametrize("name,N", CASES)
def test_mixed_full_size_close_to_oracle(name, N, oracle_results):
    R0, p, s, seed = build_large_case(name, N)
    g = Rng(seed)
    t0 = time.perf_counter()
    out, status, cnt = B.integrate_many([R0], p, s, [g], form="mixed")
    print(f"mixed {name} N={N}: {time.perf_counter() - t0:.3f} s")
    Rw, st, pst, _ = oracle_results[(name, N)]
    assert not (status[0] & _abi.ST_FATAL_MASK)
    assert g.state() == st  # the same noise stream
    assert rel(out[0], Rw) <= MIXED_TOL


def test_full_size_batch_of_both_kernels_matches_alone():
    # two N=500 Cholesky chains and two N=200 Chebyshev chains in one call:
    # each result equals its single-chain call bit for bit (plain form)
    cases = [build_large_case("cfg5_cholesky", 500, seed=3), build_large_case("cfg5_cholesky", 500, seed=4),
             build_large_case("cfg3_wlc_lj", 200, seed=5), build_large_case("cfg3_wlc_lj", 200, seed=6)]
    Rs = [c[0] for c in cases]
    gs = [Rng(c[3]) for c in cases]
    out, status, _ = B.integrate_many(Rs, [c[1] for c in cases], [c[2] for c in cases], gs, form="plain")
    for i, c in enumerate(cases):
        g = Rng(c[3])
        one, st1, _ = B.integrate_many([c[0]], c[1], c[2], [g], form="plain")
        assert int(st1[0]) == int(status[i])
        assert np.array_equal(one[0], out[i]), i
        assert g.state() == gs[i].state()
