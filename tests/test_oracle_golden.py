"""The C restatement (oracle/bd_oracle.c) against the known answers of the
reference's own tests, and against the reference C++ compiled from source."""
import json
import os

import numpy as np
import pytest

from bdsim_b200.params import Bending, DelSMethod, EV, PhysParams, Spring
from bdsim_b200 import _abi
from tests.golden.cases import CASES, FAILURE_CASES, build_case

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KNOWN = json.load(open(os.path.join(GOLD, "known_answers.json")))


def test_rng_seed10(port):
    k = KNOWN["rng_seed10"]
    x, _ = port.ran1((1, -1, k["seed"]), 10)
    assert np.max(np.abs(x - np.array(k["values"]))) < k["tol"]


def test_rng_save_restore_replay(port):
    _, st = port.ran1((1, -1, 10), 3)
    a, _ = port.ran1(st, 5)
    b, _ = port.ran1(st, 5)
    assert np.array_equal(a, b)


def test_wlc_bounded_solves(port):
    for c in KNOWN["wlcb_solves"]["cases"]:
        r, ff = port.solve_implicit_r(Spring.WLCbounded, c["dtby4"], c["gama"], c["sigma"])
        assert abs(r - c["length"]) < c["tol_len"]
        if c["force"] is not None:
            assert abs(ff - c["force"]) < c["tol_force"]


def test_wlcb_reduces_to_wlc_and_fene_equals_ff(port):
    a = port.solve_implicit_r(Spring.WLCbounded, 0.05, 1.0, 0.0)
    b = port.solve_implicit_r(Spring.WLC, 0.05, 1.0, 0.0)
    assert abs(a[0] - b[0]) < 1e-6 and abs(a[1] - b[1]) < 1e-6
    for i in range(1, 101, 7):
        for j in range(1, 101, 7):
            g = (j * 0.5) / (i * 0.1)
            f = port.solve_implicit_r(Spring.FENE, 0.05, g, 0.0)[0]
            ff = port.solve_implicit_r(Spring.FENEFraenkel, 0.05, g, 0.0)[0]
            assert abs(f - ff) < 1e-6


def test_bonds_bounded_for_huge_gamma(port):
    for g in (1.0, 1e2, 1e4, 1e6, 1e8, 1e10, 1e14, 1e20):
        r = port.solve_implicit_r(Spring.FENEFraenkel, 0.01 / 4.0, g, 0.5)[0]
        assert 0.0 <= r <= 1.5 and np.isfinite(r)
    for g in (1.0, 1e4, 1e10, 1e20):
        r = port.solve_implicit_r(Spring.FENE, 0.01 / 4.0, g, 0.0)[0]
        assert 0.0 < r < 1.0


def test_unit_bonds_and_cosines(port):
    k = KNOWN["geometry"]
    u, c = port.unit_bonds_and_cosines(np.array(k["R"]))
    assert np.max(np.abs(u[:, 0] - k["ux"])) < k["tol"]
    assert np.max(np.abs(u[:, 1] - k["uy"])) < k["tol"]
    assert np.max(np.abs(u[:, 2] - k["uz"])) < k["tol"]
    assert np.max(np.abs(c - k["cos"])) < k["tol"]


def test_bending_cases(port):
    for case in KNOWN["bending"]["cases"]:
        p = PhysParams()
        p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, case["C"]
        F = port.bending_force(np.array(case["R"], dtype=float), p)
        assert np.max(np.abs(F - np.array(case["F"]))) < KNOWN["bending"]["tol"], case["name"]


def test_rpy_block_and_cholesky_n4(port):
    k = KNOWN["hi_n4"]
    D = port.rpy_matrix(np.array(k["R"]), k["hstar"])
    assert np.max(np.abs(D[0:3, 3:6] - np.array(k["block01"]))) < k["tol_block"]
    assert np.max(np.abs(D[3:6, 3:6] - np.eye(3))) < 1e-12
    L, st = port.cholesky(D)
    assert st == 0
    bx = (L @ np.array(k["X0"]).reshape(-1)).reshape(-1, 3)
    assert np.max(np.abs(np.sqrt(k["delts"]) * bx - np.array(k["chol_bx0_sqrt_delts"]))) < k["tol_chol"]


def test_chebyshev_is_a_square_root(port):
    k = KNOWN["hi_n4"]
    D = port.rpy_matrix(np.array(k["R"]), k["hstar"])
    x0 = np.array(k["X0"]).reshape(-1)
    bx, _, fd = port.chebyshev_sqrt_times(D, x0, 1.0, 1e-6)
    assert fd < 1e-4
    bbx, _, _ = port.chebyshev_sqrt_times(D, bx, 1.0, 1e-6)
    assert np.max(np.abs(bbx - D @ x0)) < 1e-4


def test_rouse_two_chained_integrations(port):
    k = KNOWN["rouse"]
    p = PhysParams()
    p.spring.type, p.spring.sqrtb = Spring.Hook, k["sqrtb"]
    p.number_of_beads = 10
    from bdsim_b200.params import SimParams
    s = SimParams()
    s.time_start, s.time_end, s.dt, s.implicit_loop_tol = 0.0, k["t_end"], k["dt"], k["tol_corr"]
    R1, st, status, _ = port.integrate(np.array(k["R0"]), p, s, (1, -1, k["seed"]))
    assert status == 0 and np.max(np.abs(R1 - np.array(k["ans1"]))) < k["tol"]
    R2, st, status, _ = port.integrate(np.array(k["ans1"]), p, s, st)
    assert np.max(np.abs(R2 - np.array(k["ans2"]))) < k["tol"]


@pytest.mark.parametrize("name", CASES)
def test_port_matches_reference_fixtures_bitwise(port, name):
    fx = np.load(os.path.join(GOLD, "ref_steps.npz"))
    R0, p, s, seed = build_case(name)
    assert np.array_equal(R0, fx[f"{name}/R0"])
    R1, st, status, cnt = port.integrate(R0, p, s, (1, -1, seed))
    # the reference reports only the fatal bits (as exceptions); the port
    # adds the non-fatal ones (non-converged steps, Chebyshev fallbacks)
    assert int(fx[f"{name}/status"]) == status & _abi.ST_FATAL_MASK
    assert int(fx[f"{name}/port_status"]) == status
    assert np.array_equal(R1, fx[f"{name}/R1"]), np.max(np.abs(R1 - fx[f"{name}/R1"]))
    assert tuple(int(v) for v in fx[f"{name}/rng"]) == st
    assert [cnt[k] for k in _abi.COUNTER_FIELDS] == [int(v) for v in fx[f"{name}/port_counters"]]


@pytest.mark.parametrize("name", CASES)
def test_port_matches_reference_step_by_step_bitwise(port, name):
    fx = np.load(os.path.join(GOLD, "ref_steps.npz"))
    _, p, s, _ = build_case(name)
    SR, Srng, St = fx[f"{name}/steps/R"], fx[f"{name}/steps/rng"], fx[f"{name}/steps/t"]
    from bdsim_b200.params import SimParams
    for k in range(len(St)):
        one = SimParams()
        one.dt, one.implicit_loop_tol = s.dt, s.implicit_loop_tol
        one.update_center_of_mass = s.update_center_of_mass
        one.time_start = one.time_end = float(St[k])
        R1, st, status, cnt = port.integrate(SR[k], p, one, tuple(int(v) for v in Srng[k]))
        assert status == int(fx[f"{name}/steps/status"][k]), (k, status)
        assert cnt["corrector_iters"] == int(fx[f"{name}/steps/iters"][k]), k
        assert np.array_equal(R1, SR[k + 1]) and st == tuple(int(v) for v in Srng[k + 1]), k


@pytest.mark.parametrize("name", FAILURE_CASES)
def test_failure_families_take_the_failure_branches(name):
    """The fixtures of these families show the branches they exist for: the
    Chebyshev -> Cholesky fallback, the corrector's 100N cap (in the
    deterministic tol = 0 form and in the stretched-chain regime where the
    reference's own iteration stops contracting), and rtsafe on a narrow
    WLC-bounded bracket."""
    fx = np.load(os.path.join(GOLD, "ref_steps.npz"))
    cnt = dict(zip(_abi.COUNTER_FIELDS, (int(v) for v in fx[f"{name}/port_counters"])))
    steps = fx[f"{name}/steps/status"]
    if name == "cheb_fallback_always":
        assert cnt["cheb_fallbacks"] == cnt["steps"] > 0 and all(s & _abi.ST_CHEB_FALLBACK for s in steps)
    elif name == "corrector_cap_tol0":
        _, p, _, _ = build_case(name)
        assert cnt["nonconverged"] == cnt["steps"] > 0
        assert all(int(i) == 100 * p.number_of_beads + 1 for i in fx[f"{name}/steps/iters"])
    elif name == "corrector_cap_stretched":
        capped = [(int(s) & _abi.ST_NONCONVERGED) != 0 for s in steps]
        assert 0 < sum(capped) < len(capped)  # both branches
        # where the corrector is capped the reference's own result moves by
        # far more than an ulp when its input moves by one ulp
        sens = fx[f"{name}/steps/sens"]
        assert max(sens[capped]) > 1e-12 > max(sens[[not c for c in capped]])
    else:
        _, p, _, _ = build_case(name)
        assert p.spring.natural_length / p.spring.sqrtb == pytest.approx(0.95)
        assert cnt["corrector_iters"] > cnt["steps"]


def test_port_matches_live_reference_components(port, ref):
    rng = np.random.default_rng(1)
    R = np.cumsum(rng.normal(size=(12, 3)), axis=0)
    for hs in (0.1, 0.3):
        assert np.array_equal(port.rpy_matrix(R, hs), ref.rpy_matrix(R, hs))
    D = port.rpy_matrix(R, 0.25)
    L1, s1 = port.cholesky(D)
    L2, s2 = ref.cholesky(D)
    assert s1 == s2 == 0 and np.array_equal(L1, L2)
    x0 = rng.normal(size=36)
    a = port.chebyshev_sqrt_times(D, x0)
    b = ref.chebyshev_sqrt_times(D, x0)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1] and a[2] == b[2]
    p = PhysParams()
    p.spring.type, p.spring.sqrtb, p.spring.natural_length = Spring.FENEFraenkel, 3.0, 1.0
    p.ev.type, p.ev.zstar, p.ev.dstar = EV.LJ, 0.4, 0.9
    p.bend.type, p.bend.stiffness = Bending.OneMinusCosTheta, 1.5
    assert np.array_equal(port.total_force(R, p), ref.total_force(R, p))
    for t in (1, 2, 3, 4, 5, 6):
        for g in (0.0, 0.3, 1.7, 40.0):
            assert np.array_equal(port.solve_implicit_r(t, 0.01, g, 0.2), ref.solve_implicit_r(t, 0.01, g, 0.2),
                                  equal_nan=True)


def test_singular_configuration_is_not_pd(port):
    """R0_SINGULAR of the reference's Fortran cross-check
    (validation/compare_fortran_oracle.py:76-100) collapses onto two points;
    its RPY tensor is not positive definite."""
    from tests.golden.singular import R0_SINGULAR, SINGULAR_HSTAR
    D = port.rpy_matrix(R0_SINGULAR, SINGULAR_HSTAR)
    _, st = port.cholesky(D)
    assert st != 0
