"""Generate the golden fixtures of the parity tests.

  known_answers.json  the known-answer vectors of the bdsim reference's own
                      C++ tests (values as written in tests/test_*.cpp of the
                      bdsim project, which lifted them from the Fortran code),
                      each with its source file:line.
  ref_steps.npz       outputs of the reference C++ core (oracle/_ref, compiled
                      from the reference sources) for seeded integrations of
                      every configuration family the integrator supports:
                      one multi-step call per case, and the same span taken
                      one step per call (per-step states, RNG states, times).

Run where the reference sources exist:
    python tests/golden/make_golden.py [--ref REFERENCE_ROOT]
(the root defaults to $BDSIM_REF, else /root/reference). The GPU tests read only
these files, never the reference tree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The bdsim checkout to read: --ref PATH, else $BDSIM_REF, else /root/reference."""
    if "--ref" in sys.argv:
        return sys.argv[sys.argv.index("--ref") + 1]
    return os.environ.get("BDSIM_REF", "/root/reference")

ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bdsim_b200._abi import count_steps  # noqa: E402
from bdsim_b200.params import SimParams  # noqa: E402
from tests.golden.cases import CASES, build_case  # noqa: E402

KNOWN = {
    "rng_seed10": {
        "source": "tests/test_rng.cpp:16-20",
        "seed": 10,
        "values": [0.226473569869995, 0.357589989900589, 0.217218622565269, 0.688211202621460,
                   8.224623650312424e-002, 0.238840281963348, 0.956106066703796, 0.993510127067566,
                   0.167083948850632, 0.341053307056427],
        "tol": 1e-6,
    },
    "wlcb_solves": {
        "source": "tests/test_spring.cpp:25-40",
        "cases": [
            {"dtby4": 0.001 / 4.0, "gama": 5.0, "sigma": 0.8, "length": 0.999354532073543,
             "force": 1.601291769648808e4, "tol_len": 1e-6, "tol_force": 1e-2},
            {"dtby4": 0.001 / 4.0, "gama": 0.0, "sigma": 0.8, "length": 0.601489231399178,
             "force": -4.000000000000779e3, "tol_len": 1e-6, "tol_force": 1e-2},
            {"dtby4": 0.001 / 4.0, "gama": 1.0e5, "sigma": 0.8, "length": 0.999995917496677,
             "force": 3.999976329984242e8, "tol_len": 1e-6, "tol_force": 1e2},
            {"dtby4": 0.2 / 4.0, "gama": 2.0 * 2.220446049250313e-16, "sigma": 0.0, "length": 0.0,
             "force": None, "tol_len": 1e-6, "tol_force": None},
        ],
    },
    "geometry": {
        "source": "tests/test_config.cpp:17-40",
        "R": [[4.4300450016525000e-01, -3.3196056529376028e+00, 5.6132256569023198e-01],
              [1.9030176853078951e+00, -1.2695629199997360e+00, 6.8182316538962096e-01],
              [9.1311608108670805e-01, -7.1791445684858998e-02, 8.9166947220366999e-02],
              [4.4330671786225401e-01, 8.1458593138783497e-01, -1.2960528538904701e+00],
              [-1.5134472363696660e+00, 1.2352696315890850e+00, -8.9531485574350800e-01],
              [-1.4183050785054969e+00, 1.7319540232256150e+00, 1.8692574041718699e-01],
              [-4.4785729015092501e-01, 1.1633844528360100e+00, 9.9689781373572595e-01],
              [-2.7460991831883702e-01, 6.5784188432063095e-01, -1.9640797715447600e-01],
              [3.7236102056231302e-01, 3.0421928502129097e-01, -1.4997345046665300e-01],
              [-4.2058648163949502e-01, -1.2462951897582699e+00, 2.1612904801974000e-02]],
        "ux": [5.7944175608126003e-01, -5.9522532362554004e-01, -2.7468973561912702e-01,
               -9.5863447079962405e-01, 7.9645677196824999e-02, 7.0016073333826800e-01,
               1.3250236696976000e-01, 8.7574437340957700e-01, -4.5312745081482397e-01],
        "uy": [8.1360933812326097e-01, 7.2021694922843105e-01, 5.1825013808962705e-01,
               2.0609739688746501e-01, 4.1578586835775899e-01, -4.1021278232060898e-01,
               -3.8664705977290498e-01, -4.7866601579109902e-01, -8.8603680503118598e-01],
        "uz": [4.7823594888862002e-02, -3.5636268064846999e-01, -8.0991502240394098e-01,
               1.9632578636270501e-01, 9.0596836466724595e-01, 5.8438037331176895e-01,
               -9.1265939644337102e-01, 6.2854099056012996e-02, 9.8052503528402002e-02],
        "cos": [2.2403428410843801e-01, 8.2537830865396700e-01, 2.1112985007575100e-01,
                1.8720624513310299e-01, 4.1463422899762298e-01, -2.8195971820794202e-01,
                2.4374862584760501e-01, 3.3454893589510003e-02],
        "tol": 1e-6,
    },
    "bending": {
        "source": "tests/test_bending.cpp:31-73",
        "tol": 1e-6,
        "cases": [
            {"name": "3-bead 90deg", "C": 1.0, "R": [[0, 1, 0], [0, 0, 0], [1, 0, 0]],
             "F": [[-1, 0, 0], [1, 1, 0], [0, -1, 0]]},
            {"name": "3-bead random", "C": 1.0,
             "R": [[-3.0463813666787000e-02, -2.0816098199062599e-01, 7.8285534648953203e-01],
                   [1.1168640279183419e+00, 3.8970365089086001e-01, -4.9842591260299501e-01],
                   [-1.0864002142515550e+00, -1.8154266890023399e-01, -2.8442943388653802e-01]],
             "F": [[2.6795444632606003e-01, 1.0521229604980001e-03, 2.4043169403111900e-01],
                   [-2.2522472036063201e-01, -6.2136107095040000e-02, 3.6446114976283001e-02],
                   [-4.2729725965427998e-02, 6.1083984134540997e-02, -2.7687780900740200e-01]]},
            {"name": "4-bead random", "C": 1.0,
             "R": [[3.4134834606604614e-01, -4.9062758089567859e-01, -5.3069757124131800e-01],
                   [-5.9689886456173313e-01, 1.1835883708834525e+00, -4.0570939739629508e-01],
                   [-6.6797608011038512e-02, 2.3152014748196514e-01, 4.4833342082418248e-01],
                   [3.2234812650672562e-01, -9.2448093746973903e-01, 4.8807354781343082e-01]],
             "F": [[-1.0028333800544067e-02, 2.0204747869437264e-02, -3.4592206662609493e-01],
                   [1.4541591438301668e-01, 1.1254027277902146e-02, 2.9695704340823431e-01],
                   [-2.4178109393652047e-01, -8.3922618277541938e-02, -4.3532325503476693e-01],
                   [1.0639351335404786e-01, 5.2463843130202505e-02, 4.8428827825262755e-01]]},
            {"name": "5-bead random", "C": 2.0,
             "R": [[-5.1645947419192162e-01, 7.9748452989683460e-01, -4.1121562443647974e-01],
                   [-9.3988831202840872e-01, 1.1590716947448900e+00, -7.6310486638258535e-01],
                   [-6.7034760405534555e-01, -1.4053776613761966e+00, -2.9724073830375936e-01],
                   [1.1832133384385024e+00, -3.6608832152898463e-01, 6.1365584115473881e-01],
                   [9.4348205183717349e-01, -1.8509024173654354e-01, 8.5790538796808580e-01]],
             "F": [[1.0507847458911022e+00, 1.8075811550046665e+00, 5.9298653220518749e-01],
                   [-1.2494310241030562e+00, -1.8333141087409899e+00, -6.1970590685649796e-01],
                   [4.1982689539550588e-01, 3.4148812263349709e-01, -7.8361711242102261e-01],
                   [-4.2420142390715965e+00, -2.7289683808745142e+00, -1.3478360326510446e+00],
                   [4.0208336218880447e+00, 2.4132132119773404e+00, 2.1581725197233776e+00]]},
        ],
    },
    "hi_n4": {
        "source": "tests/test_hi.cpp:17-61",
        "hstar": 0.2,
        "delts": 0.1,
        "R": [[0.0, 0.0, 0.0],
              [-8.7001417024242400e+00, 5.3611027493752204e+00, 2.0995067416916502e+00],
              [-9.1605814460059198e-01, 1.1704273266182801e+01, -1.4985387607124800e+00],
              [-5.4793423363635396e+00, 4.8982010793314998e+00, 4.0063480623078496e+00]],
        "X0": [[-0.653795716820965, 2.25469853815588, 0.165603302292486],
               [-0.587509005201644, -0.745084985707505, -0.157459965970764],
               [-1.88644397151742, 3.16619, 1.23661201418787],
               [-0.958635132046656, -0.253142128732732, 1.43910244145363]],
        "block01": [[0.043185241172496, -0.010895545687992, -0.004266896699380],
                    [-0.010895545687992, 0.032217586367374, 0.002629298741189],
                    [-0.004266896699380, 0.002629298741189, 0.026533338541433]],
        "chol_bx0_sqrt_delts": [[-0.206748358961671, 0.712998281762464, 0.052368362328964],
                                [-0.202521038852097, -0.210272818508389, -0.045641895488899],
                                [-0.611043311268904, 1.022458498065220, 0.391180874642083],
                                [-0.351959054078799, -0.035305408161349, 0.461910033760980]],
        "tol_block": 1e-6,
        "tol_chol": 1e-5,
    },
    "rouse": {
        "source": "tests/test_integrator_rouse.cpp:29-97",
        "seed": 5, "dt": 0.1, "t_end": 1.0, "tol_corr": 1e-6, "sqrtb": 1000.0,
        "R0": [[0, 0, 0],
               [-6.586250662803650e-02, -4.911733418703079e-02, 2.791636288166050e-01],
               [-6.753685772418980e-01, 3.519757017493250e-01, -6.340299546718600e-01],
               [-2.844688922166820e00, -2.239686943590640e00, -7.809645235538480e-01],
               [-1.818384915590290e00, -2.201230965554710e00, 9.345296323299410e-01],
               [-3.210149317979810e00, -9.372534379363060e-01, -4.681020081043240e-01],
               [-1.490711003541950e00, -5.971195027232170e-01, -1.509506493806840e00],
               [-1.587433911859990e00, -1.017917685210700e00, -1.456502400338650e00],
               [-6.204553022980690e-01, -1.219155095517640e00, -7.125178799033161e-01],
               [-8.804024234414100e-01, -3.662307761609550e00, -7.348611745983360e-01]],
        "ans1": [[2.014655995894740e00, 3.266955094952210e00, 6.195918791485830e-01],
                 [6.898958025934120e-01, 8.753981552180370e-01, 4.785034222762240e-01],
                 [-3.793564324297950e-01, 1.489672909282450e00, -6.390832004693100e-01],
                 [-1.130337343526490e00, -6.146915212957660e-01, -5.621008935576799e-02],
                 [-6.222945452675470e-01, -1.038001996615710e00, 5.028959245456580e-01],
                 [-2.989398757279950e-01, -8.209160875818450e-01, 1.289920072746550e00],
                 [2.453406088052380e-01, 2.086869672299050e-01, 4.316992884969550e-01],
                 [-1.110128512089560e-01, -5.552336867493930e-01, -1.277926546344950e00],
                 [-6.424329445947624e-02, -1.036741598612170e00, -1.699024281591250e00],
                 [-1.915098093214250e-01, -2.620904430772130e00, 2.403765459336170e-01]],
        "ans2": [[2.358466969676050e00, 3.680650287690870e00, 7.391286505833830e-01],
                 [9.840637226840210e-02, 1.553897668605920e00, -4.535516789623883e-02],
                 [3.703216834718498e-03, 1.100513005729840e00, -5.311631291023066e-02],
                 [-1.762304275149680e00, -2.808383016377780e-02, 2.665681695031340e-01],
                 [-1.122405351207410e00, -4.065182692363470e-01, 9.790414477264030e-01],
                 [6.632472866300509e-02, -4.887170934587170e-01, 9.806758704379520e-01],
                 [-5.063576758472540e-01, -9.911910816941520e-01, 1.377974053682720e-01],
                 [2.248130548550660e-01, -9.103044958788740e-01, -1.223068999396410e00],
                 [-2.639644443515610e-01, -1.153796153975820e00, -1.197611287878650e00],
                 [1.905555228121980e00, -2.718416492074990e00, -5.090337805446200e-01]],
        "tol": 1e-6,
    },
}


def write_singular():
    """Extract R0_SINGULAR / SINGULAR_HSTAR from the reference's
    validation/compare_fortran_oracle.py into tests/golden/singular.py."""
    import re
    src = open(os.path.join(reference_root(), "validation", "compare_fortran_oracle.py")).read()
    m = re.search(r"R0_SINGULAR = np\.array\(\[(.*?)\]\)\s*\n\s*SINGULAR_HSTAR = ([0-9.eE+-]+)", src, re.S)
    rows = re.findall(r"\[([^\[\]]+)\]", m.group(1))
    arr = np.array([[float(v) for v in r.split(",")] for r in rows])
    with open(os.path.join(HERE, "singular.py"), "w") as f:
        f.write('"""R0_SINGULAR / SINGULAR_HSTAR of the reference\'s Fortran cross-check\n'
                '(validation/compare_fortran_oracle.py:76-100 of the bdsim project): a chain\n'
                'collapsed onto two points whose RPY tensor is not positive definite.\n'
                'Extracted from that file by tests/golden/make_golden.py."""\nimport numpy as np\n\n')
        f.write("R0_SINGULAR = np.array([\n")
        for r in arr:
            f.write("    [" + ", ".join(repr(float(v)) for v in r) + "],\n")
        f.write("])\n\nSINGULAR_HSTAR = " + repr(float(m.group(2))) + "\n")


COUNTERS = ["steps", "dx_products", "cheb_terms", "corrector_iters", "lanczos_cold", "lanczos_warm",
            "cheb_fallbacks", "nonconverged"]


def sensitivity(ref, R, phys, sim, rng, R_out):
    """How far the reference's own result moves when one input coordinate
    moves by one ulp: max over three coordinates of
    max|R_out' - R_out| / max(1, max|R_out|). About 1e-18 where the step is
    well conditioned; up to ~1e-8 where the corrector stops converging (its
    iteration no longer contracts), which bounds what any other rounding of
    the same step can reproduce."""
    N = len(R)
    worst = 0.0
    for i, d in ((min(1, N - 1), 0), (N // 2, 1), (N - 1, 2)):
        Rp = np.array(R, dtype=np.float64, copy=True)
        Rp[i, d] = np.nextafter(Rp[i, d], np.inf)
        Ro, _, _ = ref.integrate(Rp, phys, sim, rng)
        worst = max(worst, float(np.max(np.abs(Ro - R_out)) / max(1.0, float(np.max(np.abs(R_out))))))
    return worst


def write_prestates(ref):
    """Starting states of the families that begin mid-run, made by the
    reference from a fresh chain (tests/golden/cases.py:prestate_spec)."""
    from tests.golden.cases import PRESTATES, _sim, prestate_spec, stretched_physics
    from bdsim_b200.params import PhysParams
    from bdsim_b200 import initial
    out = {}
    for name in ("corrector_cap_stretched",):
        N, seed, steps, dt = prestate_spec(name)
        # the family's physics, from t = 0
        p = PhysParams()
        stretched_physics(p)
        p.number_of_beads = N
        R, _, status = ref.integrate(initial.gaussian_chain(N, seed=seed), p, _sim(dt, steps), (1, -1, seed))
        assert status == 0
        out[f"{name}/R0"] = R
    np.savez_compressed(PRESTATES, **out)


def main():
    write_singular()
    with open(os.path.join(HERE, "known_answers.json"), "w") as fh:
        json.dump(KNOWN, fh, indent=1)
    from oracle import oracle as O
    if not O.ref_available():
        O.build()
    ref = O.ref()
    port = O.port()
    write_prestates(ref)
    arrays = {}
    for name in CASES:
        R0, phys, sim, seed = build_case(name)
        R1, st1, status = ref.integrate(R0, phys, sim, (1, -1, seed))
        arrays[f"{name}/R0"] = R0
        arrays[f"{name}/R1"] = R1
        arrays[f"{name}/rng"] = np.array(st1, dtype=np.int64)
        arrays[f"{name}/status"] = np.array(status)
        # the non-fatal status bits and counters, which the reference only
        # prints: from the C restatement, bitwise equal to the reference here
        Rp, stp, sp, cp = port.integrate(R0, phys, sim, (1, -1, seed))
        assert np.array_equal(Rp, R1) and stp == st1, name
        arrays[f"{name}/port_status"] = np.array(sp)
        arrays[f"{name}/port_counters"] = np.array([cp[k] for k in COUNTERS], dtype=np.int64)
        arrays[f"{name}/sens"] = np.array(sensitivity(ref, R0, phys, sim, (1, -1, seed), R1))
        # the same span one reference step at a time: state k at time
        # t_k = t0 + k*dt -> state k+1 (each call a fresh model, cold cache)
        n = count_steps(sim)
        Rk, st = R0.copy(), (1, -1, seed)
        Rs, sts, ts = [Rk], [st], []
        sstat, siters, ssens = [], [], []
        for k in range(n):
            one = SimParams()
            one.dt, one.implicit_loop_tol = sim.dt, sim.implicit_loop_tol
            one.update_center_of_mass = sim.update_center_of_mass
            one.time_start = one.time_end = sim.time_start + k * sim.dt
            Rn, stn, stt = ref.integrate(Rk, phys, one, st)
            assert stt == 0
            Rpn, stpn, spn, cpn = port.integrate(Rk, phys, one, st)
            assert np.array_equal(Rpn, Rn) and stpn == stn, (name, k)
            sstat.append(spn)
            siters.append(cpn["corrector_iters"])
            ssens.append(sensitivity(ref, Rk, phys, one, st, Rn))
            Rk, st = Rn, stn
            Rs.append(Rk)
            sts.append(st)
            ts.append(one.time_start)
        arrays[f"{name}/steps/R"] = np.stack(Rs)
        arrays[f"{name}/steps/rng"] = np.array(sts, dtype=np.int64)
        arrays[f"{name}/steps/t"] = np.array(ts)
        arrays[f"{name}/steps/status"] = np.array(sstat, dtype=np.int64)
        arrays[f"{name}/steps/iters"] = np.array(siters, dtype=np.int64)
        arrays[f"{name}/steps/sens"] = np.array(ssens)
    np.savez_compressed(os.path.join(HERE, "ref_steps.npz"), **arrays)
    print(f"wrote {len(CASES)} reference cases")
    # the reference's initial-configuration generators (python/bdsim/initial.py),
    # loaded by path: they need only numpy
    import importlib.util
    spec = importlib.util.spec_from_file_location("bdsim_ref_initial",
                                                  os.path.join(reference_root(), "python", "bdsim", "initial.py"))
    ri = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ri)
    init = {}
    for seed in range(5):
        init[f"gaussian_chain/{seed}"] = ri.gaussian_chain(17, seed=seed)
        init[f"fene_fraenkel_chain/{seed}"] = ri.fene_fraenkel_chain(13, 1.0, 2.0, seed=seed)
        init[f"fene_fraenkel_chain_aligned_x/{seed}"] = ri.fene_fraenkel_chain_aligned_x(9, 1.0, 0.5, seed=seed)
        init[f"fene_fraenkel_bending_chain/{seed}"] = ri.fene_fraenkel_bending_chain(15, 1.0, 0.1, 5.0, seed=seed)
    np.savez_compressed(os.path.join(HERE, "initial_chains.npz"), **init)
    print(f"wrote {len(init)} initial chains")


if __name__ == "__main__":
    main()
