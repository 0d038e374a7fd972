"""bdcu_run_slice: a run cut into launches -- by step caps, and by a time
budget -- continues each chain from the steps and time the previous launch
reports, with its warm spectral cache, and ends bit for bit where one
uninterrupted bdcu_run ends (positions, RNG streams, warm-start vectors,
statuses, step and product counts)."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi
from tests.golden.cases import build_case

pytestmark = pytest.mark.gpu

NAMES = ["cfg2_fene_cheb_gauss", "cfg1_ff_cholesky", "cfg3_wlc_lj_uniax", "ilc_timeflow_external",
         "cfg5_ff_bend_sdk_cheb", "rouse_hook"]
K = 37  # steps of the run


def _ensemble(form):
    cases = [build_case(n) for n in NAMES]
    return B.Ensemble([c[1] for c in cases], [c[2] for c in cases], [c[0] for c in cases],
                      [(1, -1, c[3]) for c in cases], form=form), [c[2].time_start for c in cases]


def _sliced(form, cap, budget_ns, max_launches=2000):
    import torch
    ens, t0 = _ensemble(form)
    n = ens.n
    rem = np.full(n, K, dtype=np.int32)
    tnext = np.array(t0, dtype=np.float64)
    done = torch.zeros(n, dtype=torch.int32, device=ens.dev)
    tend = torch.zeros(n, dtype=torch.float64, device=ens.dev)
    launches = 0
    while rem.any():
        assert launches < max_launches
        launches += 1
        ens._t.copy_(torch.from_numpy(tnext.copy()))
        ens._k.copy_(torch.from_numpy(np.minimum(rem, cap).astype(np.int32)))
        ens.ctx.run_slice(ens.R, ens.rng, ens.cache, ens.cache_valid, ens._t, ens._k, ens.status, ens.counters,
                          ens.form, _abi.CACHE_PERSIST, budget_ns, done, tend)
        d = done.cpu().numpy()
        te = tend.cpu().numpy()
        assert (d <= np.minimum(rem, cap)).all()
        rem -= d
        tnext[d > 0] = te[d > 0]
    return ens, launches


@pytest.mark.parametrize("form", ["plain", "mixed"])
@pytest.mark.parametrize("cap,budget_ns", [(5, 0), (K, 300_000)])
def test_sliced_run_equals_one_run(form, cap, budget_ns):
    ref, t0 = _ensemble(form)
    ref.advance(np.array(t0), K, _abi.CACHE_PERSIST)
    got, launches = _sliced(form, cap, budget_ns)
    if budget_ns == 0:
        assert launches == -(-K // cap)
    assert np.array_equal(got.R.cpu().numpy(), ref.R.cpu().numpy())
    assert np.array_equal(got.rng.cpu().numpy(), ref.rng.cpu().numpy())
    assert np.array_equal(got.cache.cpu().numpy(), ref.cache.cpu().numpy())
    assert np.array_equal(got.status.cpu().numpy(), ref.status.cpu().numpy())
    gc, rc = got.counter_totals(), ref.counter_totals()
    for k in ("steps", "dx_products", "corrector_iters", "cheb_fallbacks", "nonconverged"):
        assert gc[k] == rc[k], k


def test_slice_rejects_bad_arguments():
    import torch
    ens, t0 = _ensemble("plain")
    d = torch.zeros(ens.n, dtype=torch.int32, device=ens.dev)
    te = torch.zeros(ens.n, dtype=torch.float64, device=ens.dev)
    lib, h = ens.ctx.lib, ens.ctx.h
    args = [_abi.dptr(x) for x in (ens.R, ens.rng, ens.cache, ens.cache_valid, ens._t, ens._k, ens.status,
                                   ens.counters)]
    assert lib.bdcu_run_slice(h, *args, 0, _abi.CACHE_PERSIST, -1, _abi.dptr(d), _abi.dptr(te)) == 1
    assert lib.bdcu_run_slice(h, *args, 0, _abi.CACHE_PERSIST, 0, None, _abi.dptr(te)) == 1
