"""Host-side logic and the C ABI library, without a GPU."""
import ctypes
import glob
import os
import pickle
import re

import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi, initial
from bdsim_b200.params import DelSMethod, EV, Flow, PhysParams, Rng, SimParams, Spring

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(bdcu_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    path = _abi.lib_path()
    assert os.path.exists(path), "build libbdsim_cuda.so first (__graft_entry__.build())"
    lib = ctypes.CDLL(path)
    declared = _declared_symbols()
    assert declared, "no entry points found in include/*.h"
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(_abi.EXPORTED_SYMBOLS) <= declared


def test_library_version_and_count_steps():
    lib = _abi.load_library()
    assert b"sm_100a" in lib.bdcu_version()
    for t0, t1, dt in ((0.0, 1.0, 0.1), (0.3, 0.3, 0.01), (0.0, 9.99, 0.01), (1.0, 0.5, 0.1), (0.0, 0.19, 0.01)):
        s = SimParams()
        s.time_start, s.time_end, s.dt = t0, t1, dt
        rec = _abi.BdcuSim()
        _abi._fill_sim(rec, s)
        n = ctypes.c_int64()
        assert lib.bdcu_count_steps(ctypes.byref(rec), ctypes.byref(n)) == 0
        assert n.value == _abi.count_steps(s)
        # the reference loop replayed literally
        k, t = 0, t0
        while t <= t1 + dt / 2.0:
            k += 1
            t += dt
        assert n.value == k


def test_abi_struct_layout_matches_header(tmp_path):
    """ctypes records == the C compiler's layout of include/bdsim_cuda.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bdsim_cuda.h"', "int main(void) {"]
    for cname, cls in (("bdcu_phys", _abi.BdcuPhys), ("bdcu_sim", _abi.BdcuSim), ("bdcu_counters", _abi.BdcuCounters),
                       ("bdcu_bucket_info", _abi.BdcuBucketInfo), ("bdcu_queue_config", _abi.BdcuQueueConfig),
                       ("bdcu_job", _abi.BdcuJob), ("bdcu_queue_event", _abi.BdcuQueueEvent),
                       ("bdcu_queue_stats", _abi.BdcuQueueStats)):
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c_layout = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in (("bdcu_phys", _abi.BdcuPhys), ("bdcu_sim", _abi.BdcuSim), ("bdcu_counters", _abi.BdcuCounters),
                       ("bdcu_bucket_info", _abi.BdcuBucketInfo), ("bdcu_queue_config", _abi.BdcuQueueConfig),
                       ("bdcu_job", _abi.BdcuJob), ("bdcu_queue_event", _abi.BdcuQueueEvent),
                       ("bdcu_queue_stats", _abi.BdcuQueueStats)):
        assert c_layout[(cname, "size")] == ctypes.sizeof(cls)
        for fname, _ in cls._fields_:
            assert c_layout[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_params_pickle_roundtrip():
    p = PhysParams()
    p.spring.type, p.spring.sqrtb = Spring.FENE, 7.0
    p.ev.type, p.ev.zstar = EV.Gauss, 1.0
    p.hi_method = DelSMethod.Cholesky
    p.flow = Flow.time_varying([0, 1], [np.zeros((3, 3)), np.eye(3)])
    p.external.add_stretch(0, -1, (0, 0, 1))
    q = pickle.loads(pickle.dumps(p))
    assert q.spring.type == Spring.FENE and q.spring.sqrtb == 7.0 and q.hi_method == DelSMethod.Cholesky
    assert not q.flow.is_constant() and len(q.external.entries()) == 2
    r = Rng(42)
    assert pickle.loads(pickle.dumps(r)).state() == (1, -1, 42)
    s = SimParams()
    s.dt = 0.5
    assert pickle.loads(pickle.dumps(s)).dt == 0.5
    assert str(Spring.FENE) == "Spring.FENE"


def test_pack_batch_arena_layout():
    p = PhysParams()
    p.flow = Flow.time_varying([0.0, 2.0], [np.zeros((3, 3)), np.full((3, 3), 2.0)])
    p.external.add_constant(1, (1.0, 2.0, 3.0))
    p.external.add_time_varying(-1, [0.0, 1.0], [(0, 0, 0), (4, 5, 6)])
    p.ev.type = EV.SDK
    p.ev.phi = [0.5] * 9
    prec, srec, arena = _abi.pack_batch([p, p], [SimParams(), SimParams()], [3, 3])
    assert prec[0].flow_n_times == 2 and prec[0].flow_offset == prec[1].flow_offset
    f = prec[0].flow_offset
    assert list(arena[f:f + 2]) == [0.0, 2.0] and arena[f + 2 + 9] == 2.0
    e = prec[0].ext_offset
    assert list(arena[e:e + 6]) == [1.0, 1.0, 1.0, 2.0, 3.0, 0.0]
    assert list(arena[e + 6:e + 12]) == [-1.0, 0.0, 0.0, 0.0, 0.0, 2.0]
    assert arena[prec[0].phi_offset] == 0.5
    with pytest.raises(ValueError):
        p.ev.phi = [0.5] * 4
        _abi.pack_batch([p], [SimParams()], [3])


def test_initial_generators_match_reference_fixture():
    fx = np.load(os.path.join(ROOT, "tests", "golden", "initial_chains.npz"))
    for seed in range(5):
        assert np.array_equal(initial.gaussian_chain(17, seed=seed), fx[f"gaussian_chain/{seed}"])
        assert np.array_equal(initial.fene_fraenkel_chain(13, 1.0, 2.0, seed=seed), fx[f"fene_fraenkel_chain/{seed}"])
        assert np.array_equal(initial.fene_fraenkel_chain_aligned_x(9, 1.0, 0.5, seed=seed),
                              fx[f"fene_fraenkel_chain_aligned_x/{seed}"])
        assert np.array_equal(initial.fene_fraenkel_bending_chain(15, 1.0, 0.1, 5.0, seed=seed),
                              fx[f"fene_fraenkel_bending_chain/{seed}"])


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        B.integrate(np.zeros((4, 3)), PhysParams(), SimParams(), Rng(1))


def _external_case_records():
    from tests.golden.cases import build_case
    R0, phys, sim, _ = build_case("ilc_timeflow_external")
    prec, srec, arena = _abi.pack_batch([phys], [sim], [len(R0)])
    assert prec[0].ext_n_entries >= 2
    return prec, srec, arena


def test_check_chains_accepts_a_valid_record():
    prec, srec, arena = _external_case_records()
    rc, msg = _abi.check_records(1, prec, srec, arena)
    assert rc == 0, msg


def test_check_chains_rejects_a_negative_external_offset():
    """bdcu_run_static and bdcu_set_chains share these checks; a record that
    points before the arena never reaches a kernel."""
    prec, srec, arena = _external_case_records()
    prec[0].ext_offset = -1
    rc, msg = _abi.check_records(1, prec, srec, arena)
    assert rc == 1 and "external force list outside the arena" in msg


def test_check_chains_rejects_an_external_table_past_the_arena():
    prec, srec, arena = _external_case_records()
    # the second entry's sample count (header word 5) runs past the arena's end
    first = int(prec[0].ext_offset)
    nt0 = int(arena[first + 5])
    second = first + 6 + 4 * nt0
    bad = arena.copy()
    bad[second + 5] = float(arena.size)
    rc, msg = _abi.check_records(1, prec, srec, bad)
    assert rc == 1 and "external force list outside the arena" in msg
    # and a list whose entry count walks off the end
    prec[0].ext_n_entries = 1000
    rc, msg = _abi.check_records(1, prec, srec, arena)
    assert rc == 1


def test_check_chains_rejects_negative_flow_offset_and_bead_limit():
    from tests.golden.cases import build_case
    R0, phys, sim, _ = build_case("ilc_timeflow_external")
    prec, srec, arena = _abi.pack_batch([phys], [sim], [len(R0)])
    if prec[0].flow_n_times > 0:
        prec[0].flow_offset = -5
        rc, msg = _abi.check_records(1, prec, srec, arena)
        assert rc == 1 and "flow table" in msg
    prec, srec, arena = _abi.pack_batch([phys], [sim], [len(R0)])
    prec[0].n_beads = 5000
    rc, msg = _abi.check_records(1, prec, srec, arena)
    assert rc == 5 and "n_beads" in msg


def _queue_config(**kw):
    cfg = _abi.BdcuQueueConfig()
    cfg.form, cfg.policy, cfg.max_chains, cfg.bead_capacity = 1, _abi.QUEUE_FIFO, 8, 256
    cfg.arena_capacity, cfg.slice_steps, cfg.cache_mode = 64, 10, _abi.CACHE_RESET_PER_CALL
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


@pytest.mark.parametrize("bad", [dict(form=7), dict(policy=2), dict(max_chains=0), dict(bead_capacity=1),
                                 dict(arena_capacity=-1), dict(queue_limit=-1), dict(slice_steps=0),
                                 dict(cache_mode=9), dict(slice_budget_ns=-5), dict(worker=2)])
def test_queue_config_checks_come_before_the_gpu(bad):
    """bdcu_queue_create rejects a bad configuration with BDCU_E_ARG and a
    message before it touches CUDA."""
    lib = _abi.load_library()
    h = ctypes.c_void_p()
    cfg = _queue_config(**bad)
    assert lib.bdcu_queue_create(0, ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert not h.value
    assert lib.bdcu_queue_last_error(None).decode()


def test_queue_entry_points_reject_null_handles():
    lib = _abi.load_library()
    ev, got, busy = _abi.BdcuQueueEvent(), ctypes.c_int(), ctypes.c_int()
    jid, ok = ctypes.c_int64(), ctypes.c_int()
    st = _abi.BdcuQueueStats()
    assert lib.bdcu_queue_submit(None, None, ctypes.byref(jid), ctypes.byref(ok)) == 1
    assert lib.bdcu_queue_step(None, ctypes.byref(busy)) == 1
    assert lib.bdcu_queue_wait_idle(None, 0, ctypes.byref(busy)) == 1
    assert lib.bdcu_queue_poll(None, ctypes.byref(ev), None, 0, None, 0, ctypes.byref(got)) == 1
    assert lib.bdcu_queue_get_stats(None, ctypes.byref(st)) == 1
    assert lib.bdcu_queue_destroy(None) == 1
    assert lib.bdcu_queue_create(0, None, None) == 1


def test_queue_create_without_a_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _abi.load_library()
    h = ctypes.c_void_p()
    cfg = _queue_config()
    assert lib.bdcu_queue_create(0, ctypes.byref(cfg), ctypes.byref(h)) == 2  # BDCU_E_CUDA
    assert not h.value and lib.bdcu_queue_last_error(None).decode()
