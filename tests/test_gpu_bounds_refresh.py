"""The FP32-mixed form's spectral-bound refresh policy (bdcu_set_bounds_refresh):
with the bounds kept for K steps (and refreshed early whenever a step's
Chebyshev check fails on them) the ensemble statistics stay those of the FP64
plain form, fewer D.x products are spent, and K=1 is the default policy
bit for bit."""
import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import initial
from bdsim_b200.params import DelSMethod, EV, Flow, PhysParams, SimParams, Spring

pytestmark = pytest.mark.gpu


def _setup(n, N=20, dt=1e-2):
    p = PhysParams()
    p.spring.type, p.spring.sqrtb = Spring.FENE, 50.0 ** 0.5
    p.hstar, p.hi_method = 0.25, DelSMethod.Chebyshev
    p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 1.0, 0.5
    K = np.zeros((3, 3))
    K[0, 1] = 1.0
    p.flow = Flow.constant(K)
    s = SimParams()
    s.dt = dt
    R0s = [initial.gaussian_chain(N, seed=i) for i in range(n)]
    return [p] * n, [s] * n, R0s, [(1, -1, i) for i in range(n)]


def _obs(ens):
    Rs, Fs = ens.positions(), ens.total_force()
    rg2 = np.array([np.sum((R - R.mean(0)) ** 2) / len(R) for R in Rs])
    txy = np.array([((R - R.mean(0)).T @ F)[0, 1] for R, F in zip(Rs, Fs)])
    return rg2, txy


def test_kept_bounds_keep_the_ensemble_statistics():
    n = 256
    phys, sims, R0s, rngs = _setup(n)
    res, dx = {}, {}
    for form, every in (("plain", 1), ("mixed", 4)):
        ens = B.Ensemble(phys, sims, R0s, rngs, form=form)
        ens.ctx.set_bounds_refresh(every)
        ens.advance(0.0, 400)
        assert not ens.failed().any()
        res[form] = _obs(ens)
        c = ens.counter_totals()
        dx[form] = c["dx_products"] / c["steps"]
    for k in range(2):
        a, b = res["plain"][k], res["mixed"][k]
        err = np.sqrt(a.var(ddof=1) / n + b.var(ddof=1) / n)
        assert abs(a.mean() - b.mean()) <= 3 * err, (k, a.mean(), b.mean(), err)
    assert dx["mixed"] < dx["plain"] - 3.0, dx


def test_refresh_every_step_is_the_default():
    phys, sims, R0s, rngs = _setup(32, N=50, dt=1e-3)
    out = []
    for every in (None, 1):
        ens = B.Ensemble(phys, sims, R0s, rngs, form="mixed")
        if every is not None:
            ens.ctx.set_bounds_refresh(every)
        ens.advance(0.0, 50)
        out.append(ens.R.cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_refresh_rejects_bad_values():
    ens = B.Ensemble(*_setup(2), form="mixed")
    with pytest.raises(Exception):
        ens.ctx.set_bounds_refresh(0)
