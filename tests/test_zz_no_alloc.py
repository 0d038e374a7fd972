"""bdcu_run_static -- the integrator entry point for callers that cannot
allocate device memory (a host application whose pool already owns the GPU's
memory, or a loop that must not take cudaMalloc's implicit synchronisation) --
against bdcu_run on identical inputs, two calls in a row.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test. It also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi
from tests.golden.cases import build_case

pytestmark = pytest.mark.gpu

CALL_TOL = 1e-10  # the per-call tolerance of the plain-form parity tests


def _batch():
    names = ["cfg2_fene_cheb_gauss", "cfg1_ff_cholesky", "cfg3_wlc_lj_uniax", "rouse_hook"]
    R0s, phys, sims, seeds = [], [], [], []
    for k, name in enumerate(names):
        for rep in range(3):
            R0, p, s, seed = build_case(name)
            R0s.append(R0 + 0.01 * rep)
            phys.append(p)
            sims.append(s)
            seeds.append(100 * k + rep)
    return R0s, phys, sims, seeds


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_static_entry_point_matches_bdcu_run_twice(form):
    import torch
    R0s, phys, sims, seeds = _batch()
    n = len(R0s)
    steps = [_abi.count_steps(s) for s in sims]

    ens = B.Ensemble(phys, sims, R0s, [(1, -1, s) for s in seeds], form=form)
    lib = ens.ctx.lib

    # the caller's own device buffers for the static path
    dev = torch.device("cuda", 0)
    R = torch.from_numpy(np.concatenate(R0s)).to(dev)
    rng = torch.tensor([(1, -1, s) for s in seeds], dtype=torch.int32, device=dev)
    cache = torch.zeros_like(ens.cache)
    valid = torch.zeros(n, dtype=torch.int32, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    counters = torch.zeros((n, 8), dtype=torch.int64, device=dev)
    prec, srec, arena = _abi.pack_batch(phys, sims, [len(r) for r in R0s])
    ctx = B.Context(0)
    ctx.use_stream()

    t = np.array([s.time_start for s in sims])
    for call in range(2):
        t0 = torch.tensor(t, dtype=torch.float64, device=dev)
        k = torch.tensor(steps, dtype=torch.int32, device=dev)
        ens.advance(t, steps, _abi.CACHE_PERSIST)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        rc = lib.bdcu_run_static(ctx.h, n, prec, srec, arena.ctypes.data_as(_abi.c_double_p), arena.size,
                                 _abi.dptr(R), _abi.dptr(rng), _abi.dptr(cache), _abi.dptr(valid), _abi.dptr(t0),
                                 _abi.dptr(k), _abi.dptr(status), _abi.dptr(counters),
                                 _abi.FORM_PLAIN_FP64 if form == "plain" else _abi.FORM_MIXED_FP32,
                                 _abi.CACHE_PERSIST)
        assert rc == 0, lib.bdcu_last_error(ctx.h).decode()
        torch.cuda.synchronize()
        if call == 1:
            # the first call loads the module and takes the array's address;
            # the second must leave the device's free memory as it found it
            assert torch.cuda.mem_get_info(0)[0] == free_before
        want = ens.R.cpu().numpy()
        got = R.cpu().numpy()
        assert np.array_equal(ens.status.cpu().numpy(), status.cpu().numpy()), call
        assert np.array_equal(ens.rng.cpu().numpy(), rng.cpu().numpy()), call
        assert _rel(got, want) <= CALL_TOL, (call, _rel(got, want))
        assert _rel(cache.cpu().numpy(), ens.cache.cpu().numpy()) <= CALL_TOL, call
        assert np.array_equal(ens.counters.cpu().numpy(), counters.cpu().numpy()), call
        t = t + np.array(steps) * np.array([s.dt for s in sims])


def test_static_entry_point_rejects_a_batch_beyond_its_maximum():
    # N=500 with HI: one block's Cholesky scratch alone is 1500^2 doubles (18 MB)
    R0, p, s, seed = build_case("cfg2_fene_cheb_gauss")
    p.number_of_beads = 500
    R0 = B.gaussian_chain(500, seed=1)
    prec, srec, arena = _abi.pack_batch([p], [s], [500])
    ctx = B.Context(0)
    import torch
    dev = torch.device("cuda", 0)
    R = torch.from_numpy(R0).to(dev)
    z32 = torch.zeros(3, dtype=torch.int32, device=dev)
    zc = torch.zeros(1500, dtype=torch.float64, device=dev)
    z1 = torch.zeros(1, dtype=torch.int32, device=dev)
    t0 = torch.zeros(1, dtype=torch.float64, device=dev)
    cnt = torch.zeros((1, 8), dtype=torch.int64, device=dev)
    rc = ctx.lib.bdcu_run_static(ctx.h, 1, prec, srec, arena.ctypes.data_as(_abi.c_double_p), arena.size,
                                 _abi.dptr(R), _abi.dptr(z32), _abi.dptr(zc), _abi.dptr(z1), _abi.dptr(t0),
                                 _abi.dptr(z1), _abi.dptr(z1), _abi.dptr(cnt), 0, _abi.CACHE_RESET_PER_CALL)
    assert rc == 5  # BDCU_E_LIMIT
    assert "maximum" in ctx.lib.bdcu_last_error(ctx.h).decode()


def test_static_entry_point_rejects_a_record_outside_the_arena():
    """The record checks of bdcu_set_chains apply before anything is launched:
    an external-force list that starts before the arena is BDCU_E_ARG."""
    import torch
    R0, p, s, seed = build_case("ilc_timeflow_external")
    prec, srec, arena = _abi.pack_batch([p], [s], [len(R0)])
    prec[0].ext_offset = -1
    ctx = B.Context(0)
    dev = torch.device("cuda", 0)
    n = len(R0)
    R = torch.from_numpy(R0).to(dev)
    rng = torch.tensor([[1, -1, seed]], dtype=torch.int32, device=dev)
    zc = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    z1 = torch.zeros(1, dtype=torch.int32, device=dev)
    t0 = torch.zeros(1, dtype=torch.float64, device=dev)
    k = torch.ones(1, dtype=torch.int32, device=dev)
    cnt = torch.zeros((1, 8), dtype=torch.int64, device=dev)
    before = R.clone()
    rc = ctx.lib.bdcu_run_static(ctx.h, 1, prec, srec, arena.ctypes.data_as(_abi.c_double_p), arena.size,
                                 _abi.dptr(R), _abi.dptr(rng), _abi.dptr(zc), _abi.dptr(z1), _abi.dptr(t0),
                                 _abi.dptr(k), _abi.dptr(z1), _abi.dptr(cnt), 0, _abi.CACHE_RESET_PER_CALL)
    torch.cuda.synchronize()
    assert rc == 1  # BDCU_E_ARG
    assert "outside the arena" in ctx.lib.bdcu_last_error(ctx.h).decode()
    assert torch.equal(R, before)
