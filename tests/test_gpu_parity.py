"""Parity of the CUDA integrator (through the C ABI) with the reference.

Tolerances, stated once:
  PLAIN_TOL = 1e-12  plain FP64 form, ONE step from the reference's state and
                     RNG state: max|R_gpu - R_ref| / max(1, max|R_ref|)
  CALL_TOL  = 1e-10  plain form, one multi-step call (<= 40 steps). Chains
                     amplify last-bit differences step by step: the reference
                     itself moves by up to 3.5e-11 over the 10-step stiff
                     FENE-Fraenkel case when one libm result (acos, cos)
                     changes by one ulp, and CUDA's libm differs from glibc's
                     by up to 2 ulp.
  MIXED_TOL = 1e-4   FP32-mixed form, per call of <= 40 steps, same norm
  COND = 100         where a step (or call) is ill conditioned -- the
                     corrector at its 100N cap, whose iteration no longer
                     contracts -- the reference's own result moves by `sens`
                     (up to ~1e-8, stored per step in the fixtures) when one
                     input coordinate moves by one ulp; the bound there is
                     max(PLAIN_TOL or CALL_TOL, COND * sens). A build of the
                     C restatement with FMA contraction everywhere (every
                     multiply-add rounded differently) stays within 4.2 x sens
                     of the reference on every step of every family.
RNG streams are compared bit for bit; per-step statuses and corrector
iteration counts exactly.
"""
import os

import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi
from bdsim_b200.params import DelSMethod, EV, PhysParams, Rng, SimParams, Spring
from tests.golden.cases import CASES, FAILURE_CASES, build_case

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-12
CALL_TOL = 1e-10
MIXED_TOL = 1e-4
COND = 100.0
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, float(np.max(np.abs(b)))))


@pytest.fixture(scope="module")
def fixtures():
    return np.load(os.path.join(GOLD, "ref_steps.npz"))


def test_ran1_bitexact(port):
    import torch
    ctx = B.Context(0)
    ctx.set_chains([PhysParams()], [SimParams()], [2])
    states = [(1, -1, 10), (1, -1, 0), (1, -1, -7), (1, -1, 123456), (-716706388, 2128629622, 11)]
    rng = torch.tensor(states, dtype=torch.int32, device="cuda")
    out = torch.zeros((len(states), 257), dtype=torch.float64, device="cuda")
    ctx.ran1(rng, 257, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for i, s in enumerate(states):
        want, st = port.ran1(s, 257)
        assert np.array_equal(got[i], want)
        assert tuple(rng[i].tolist()) == st


def _one_step_sim(sim, t):
    one = SimParams()
    one.dt, one.implicit_loop_tol = sim.dt, sim.implicit_loop_tol
    one.update_center_of_mass = sim.update_center_of_mass
    one.time_start = one.time_end = t
    return one


def test_plain_every_step_matches_reference(fixtures):
    """Every step of every case, from the reference's own state, RNG state and
    time, as independent chains of one batch (cold spectral cache: each
    reference step is its own integrate call)."""
    Rs, phys, sims, rngs, want, want_rng, tags, tols, stats, iters = [], [], [], [], [], [], [], [], [], []
    for name in CASES:
        _, p, s, _ = build_case(name)
        SR = fixtures[f"{name}/steps/R"]
        Srng = fixtures[f"{name}/steps/rng"]
        St = fixtures[f"{name}/steps/t"]
        for k in range(len(St)):
            tols.append(max(PLAIN_TOL, COND * float(fixtures[f"{name}/steps/sens"][k])))
            stats.append(int(fixtures[f"{name}/steps/status"][k]))
            iters.append(int(fixtures[f"{name}/steps/iters"][k]))
            Rs.append(SR[k])
            phys.append(p)
            sims.append(_one_step_sim(s, float(St[k])))
            g = Rng(0)
            g.set_state(tuple(int(v) for v in Srng[k]))
            rngs.append(g)
            want.append(SR[k + 1])
            want_rng.append(tuple(int(v) for v in Srng[k + 1]))
            tags.append((name, k))
    out, status, cnt = B.integrate_many(Rs, phys, sims, rngs, form="plain")
    worst, loose = 0.0, 0
    for i, tag in enumerate(tags):
        assert status[i] == stats[i], (tag, status[i], stats[i])
        assert cnt[i]["corrector_iters"] == iters[i], (tag, cnt[i]["corrector_iters"], iters[i])
        assert rngs[i].state() == want_rng[i], tag
        e = rel(out[i], want[i])
        if tols[i] == PLAIN_TOL:
            worst = max(worst, e)
        else:
            loose += 1
        assert e <= tols[i], (tag, e, tols[i])
    print(f"{len(tags)} reference steps, worst relative difference {worst:.2e} "
          f"({loose} ill-conditioned capped steps at {COND:g} x the reference's 1-ulp sensitivity)")


def test_plain_every_warm_step_matches_port(port):
    """Steps that warm-start Lanczos from the previous step's cache: the
    oracle walks each Chebyshev case with one persistent cache; every step is
    replayed on the GPU from the oracle's state AND cache vector."""
    Rs, phys, sims, states, caches, valid, t0s, want, want_cache = [], [], [], [], [], [], [], [], []
    for name in [c for c in CASES if "cheb" in c or c in ("ilc_timeflow_external", "n2_dumbbell_hi")]:
        R0, p, s, seed = build_case(name)
        n = _abi.count_steps(s)
        cache = [np.zeros(3 * len(R0)), 0]
        R, st = R0.copy(), (1, -1, seed)
        for k in range(n):
            t = s.time_start + k * s.dt
            c_in, v_in = cache[0].copy(), cache[1]
            R1, st1, status, _ = port.integrate(R, p, _one_step_sim(s, t), st, cache=cache)
            if v_in:  # only steps that start warm
                Rs.append(R)
                phys.append(p)
                sims.append(s)
                states.append(st)
                caches.append(c_in)
                valid.append(v_in)
                t0s.append(t)
                want.append(R1)
                want_cache.append(cache[0].copy())
            R, st = R1, st1
    import torch
    ens = B.Ensemble(phys, sims, Rs, states, form="plain")
    ens.cache.copy_(torch.from_numpy(np.concatenate(caches)))
    ens.cache_valid.copy_(torch.tensor(valid, dtype=torch.int32))
    ens.advance(np.array(t0s), 1, _abi.CACHE_PERSIST)
    got = ens.positions()
    gc = ens.cache.cpu().numpy()
    assert not ens.failed().any()
    for i in range(len(Rs)):
        assert rel(got[i], want[i]) <= PLAIN_TOL, i
        o = 3 * int(ens.offsets[i])
        assert rel(gc[o:o + len(want_cache[i])], want_cache[i]) <= 1e-9, i
    print(f"{len(Rs)} warm-start steps")


@pytest.mark.parametrize("name", CASES)
def test_plain_call_matches_reference(name, fixtures):
    R0, p, s, seed = build_case(name)
    g = Rng(seed)
    out, status, _ = B.integrate_many([R0], p, s, [g], form="plain")
    assert int(status[0]) & _abi.ST_FATAL_MASK == int(fixtures[f"{name}/status"])
    assert int(status[0]) == int(fixtures[f"{name}/port_status"])
    assert g.state() == tuple(int(v) for v in fixtures[f"{name}/rng"])
    assert rel(out[0], fixtures[f"{name}/R1"]) <= max(CALL_TOL, COND * float(fixtures[f"{name}/sens"]))


@pytest.mark.parametrize("name", CASES)
def test_plain_matches_port_with_counters(name, port):
    R0, p, s, seed = build_case(name)
    g = Rng(seed)
    out, status, cnt = B.integrate_many([R0], p, s, [g], form="plain")
    Rp, st, pst, pcnt = port.integrate(R0, p, s, (1, -1, seed))
    fx = np.load(os.path.join(GOLD, "ref_steps.npz"))
    assert rel(out[0], Rp) <= max(CALL_TOL, COND * float(fx[f"{name}/sens"]))
    assert g.state() == st
    assert int(status[0]) == pst
    for k in ("steps", "corrector_iters", "lanczos_cold", "lanczos_warm", "cheb_fallbacks", "nonconverged"):
        assert cnt[0][k] == pcnt[k], k


@pytest.mark.parametrize("name", [c for c in CASES if "cholesky" not in c and c != "corrector_cap_stretched"])
def test_mixed_close_to_reference(name, fixtures):
    R0, p, s, seed = build_case(name)
    g = Rng(seed)
    out, status, _ = B.integrate_many([R0], p, s, [g], form="mixed")
    assert int(status[0]) == int(fixtures[f"{name}/port_status"])
    assert g.state() == tuple(int(v) for v in fixtures[f"{name}/rng"])  # same noise stream
    assert rel(out[0], fixtures[f"{name}/R1"]) <= MIXED_TOL


@pytest.mark.parametrize("name", FAILURE_CASES)
def test_failure_branches_match_the_reference_in_both_forms(name, fixtures):
    """Chebyshev -> Cholesky fallbacks and capped corrector steps: the same
    statuses and the same counts as the reference (the C restatement, bitwise
    equal to it on these families), in the plain and the FP32-mixed form,
    from the reference's state at every step. In the stretched-chain regime
    the capped corrector's result is ill conditioned (the reference moves by
    up to ~1e-8 for a one-ulp input change), which no FP32 computation can
    follow: the mixed form is held to the statuses and iteration counts
    there, and to MIXED_TOL where the steps are well conditioned."""
    _, p, s, _ = build_case(name)
    SR, Srng, St = fixtures[f"{name}/steps/R"], fixtures[f"{name}/steps/rng"], fixtures[f"{name}/steps/t"]
    want_st, want_it = fixtures[f"{name}/steps/status"], fixtures[f"{name}/steps/iters"]
    sens = fixtures[f"{name}/steps/sens"]
    n = len(St)
    for form in ("plain", "mixed"):
        rngs = []
        for k in range(n):
            g = Rng(0)
            g.set_state(tuple(int(v) for v in Srng[k]))
            rngs.append(g)
        out, status, cnt = B.integrate_many([SR[k] for k in range(n)], p,
                                            [_one_step_sim(s, float(St[k])) for k in range(n)], rngs, form=form)
        for k in range(n):
            assert int(status[k]) == int(want_st[k]), (form, k, status[k], want_st[k])
            assert rngs[k].state() == tuple(int(v) for v in Srng[k + 1]), (form, k)
            for c in ("cheb_fallbacks", "nonconverged"):
                assert cnt[k][c] == (1 if c == "cheb_fallbacks" and want_st[k] & _abi.ST_CHEB_FALLBACK else
                                     1 if c == "nonconverged" and want_st[k] & _abi.ST_NONCONVERGED else 0)
            e = rel(out[k], SR[k + 1])
            if form == "plain":
                assert cnt[k]["corrector_iters"] == int(want_it[k]), (k, cnt[k]["corrector_iters"])
                assert e <= max(PLAIN_TOL, COND * float(sens[k])), (k, e)
            elif sens[k] < 1e-12:
                assert e <= MIXED_TOL, (form, k, e)
        if name != "wlcbounded_sigma095":
            assert sum(c["cheb_fallbacks"] + c["nonconverged"] for c in cnt) > 0


def test_forces_match_port(port):
    rng = np.random.default_rng(3)
    R = np.cumsum(rng.normal(size=(17, 3)), axis=0)
    p = PhysParams()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 3.0, 1.0
    p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 0.8, 0.7
    p.bend.type, p.bend.stiffness = 1, 2.0
    assert rel(B.total_force(R, p), port.total_force(R, p)) <= 1e-14
    assert rel(B.spring_force(R, p.spring), port.spring_force(R, p)) <= 1e-15
    q = PhysParams()
    q.bend = p.bend
    assert rel(B.bending_force(R, p.bend), port.bending_force(R, q)) <= 1e-15
    q = PhysParams()
    q.ev = p.ev
    assert rel(B.ev_force(R, p.ev), port.ev_force(R, q)) <= 1e-14
    for t in (-1.0, 0.05, 0.5, 3.0):
        R0, pe, s, seed = build_case("ilc_timeflow_external")
        assert rel(B.external_force(pe, len(R0), t), port.external_force(pe, len(R0), t)) <= 1e-15


def test_chunked_persistent_cache_equals_port(port):
    """Two chunks with the warm-start cache kept (BDCU_CACHE_PERSIST) == the
    oracle integrating the same chunks with one persistent cache."""
    R0, p, s, seed = build_case("cfg2_fene_cheb_gauss")
    ens = B.Ensemble([p], [s], [R0], [(1, -1, seed)], form="plain")
    ens.advance(0.0, 7)
    ens.advance(7 * s.dt, 5)
    got = ens.positions()[0]
    cache = [np.zeros(3 * len(R0)), 0]
    s1 = SimParams()
    s1.dt, s1.time_start, s1.time_end = s.dt, 0.0, 6 * s.dt
    R1, st, _, _ = port.integrate(R0, p, s1, (1, -1, seed), cache=cache)
    s2 = SimParams()
    s2.dt, s2.time_start, s2.time_end = s.dt, 7 * s.dt, 11 * s.dt
    R2, st, _, c2 = port.integrate(R1, p, s2, st, cache=cache)
    assert rel(got, R2) <= CALL_TOL
    assert ens.rng_states()[0] == st


def test_same_result_alone_and_in_a_mixed_batch():
    names = ["cfg2_fene_cheb_gauss", "cfg1_ff_cholesky", "cfg3_wlc_lj_uniax", "rouse_hook", "n3_bend_hi_chol"]
    cases = [build_case(n) for n in names]
    alone = []
    for R0, p, s, seed in cases:
        out, _, _ = B.integrate_many([R0], p, s, [Rng(seed)], form="plain")
        alone.append(out[0])
    out, status, _ = B.integrate_many([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases],
                                      [Rng(c[3]) for c in cases], form="plain")
    for a, b in zip(alone, out):
        assert rel(b, a) <= CALL_TOL


def test_failures_are_statuses_not_faults():
    from tests.golden.singular import R0_SINGULAR, SINGULAR_HSTAR
    good, pg, sg, seed = build_case("cfg1_ff_cholesky")
    ps = PhysParams()
    ps.spring.type, ps.spring.sqrtb = Spring.FENE, 50.0
    ps.hstar, ps.hi_method = SINGULAR_HSTAR, DelSMethod.Cholesky
    s = SimParams()
    s.dt, s.time_start, s.time_end = 1e-3, 0.0, 0.0
    nan = good.copy()
    nan[3, 1] = np.nan
    pb = PhysParams()
    pb.spring.type, pb.spring.sqrtb, pb.spring.natural_length = Spring.WLCbounded, 2.0, 3.0
    pe = PhysParams()
    pe.hstar, pe.hi_method = 0.2, DelSMethod.ExactSqrt
    outs, status, _ = B.integrate_many([good, R0_SINGULAR, nan, good, good], [pg, ps, pg, pb, pe],
                                       [sg, s, sg, sg, sg], [Rng(i + 1) for i in range(5)])
    assert status[0] == 0
    assert status[1] & _abi.ST_NOT_PD
    assert status[2] & (_abi.ST_NONFINITE | _abi.ST_NOT_PD)
    assert status[3] & _abi.ST_BAD_PARAM
    assert status[4] & _abi.ST_BAD_PARAM
    ref_good, _, _ = B.integrate_many([good], pg, sg, [Rng(1)])
    assert rel(outs[0], ref_good[0]) <= CALL_TOL
    with pytest.raises(B.IntegratorError):
        B.integrate(R0_SINGULAR, ps, s, Rng(3))


def test_mixed_ensemble_statistics_match_plain():
    """Ensemble-mean Rg^2 and shear stress of the FP32-mixed form agree with
    the FP64 plain form within 3 standard errors (N=20, 256 chains)."""
    n = 256
    p = PhysParams()
    p.spring.type, p.spring.sqrtb = Spring.FENE, 50.0 ** 0.5
    p.hstar, p.hi_method = 0.25, DelSMethod.Chebyshev
    p.ev.type, p.ev.zstar, p.ev.dstar = EV.Gauss, 1.0, 0.5
    from bdsim_b200.params import Flow
    K = np.zeros((3, 3))
    K[0, 1] = 1.0
    p.flow = Flow.constant(K)
    s = SimParams()
    s.dt = 1e-2
    from bdsim_b200 import initial
    R0s = [initial.gaussian_chain(20, seed=i) for i in range(n)]
    res = {}
    for form in ("plain", "mixed"):
        ens = B.Ensemble([p] * n, [s] * n, R0s, [(1, -1, i) for i in range(n)], form=form)
        ens.advance(0.0, 400)
        Rs = ens.positions()
        Fs = ens.total_force()
        rg2 = np.array([np.sum((R - R.mean(0)) ** 2) / len(R) for R in Rs])
        txy = np.array([((R - R.mean(0)).T @ F)[0, 1] for R, F in zip(Rs, Fs)])
        res[form] = (rg2, txy)
        assert not ens.failed().any()
    for k in range(2):
        a, b = res["plain"][k], res["mixed"][k]
        err = np.sqrt(a.var(ddof=1) / n + b.var(ddof=1) / n)
        assert abs(a.mean() - b.mean()) <= 3 * err, (k, a.mean(), b.mean(), err)
