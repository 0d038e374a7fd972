"""The reference's own parameter objects pass the C-ABI packer unchanged
(the backend="cuda" routing of the reference's simulate / run_ensemble hands
them over as they are), and its reducers map to the batched ones."""
import ctypes

import numpy as np
import pytest

import bdsim_b200 as B
from bdsim_b200 import _abi, ensemble, rheology
from bdsim_b200.params import rng_state, set_rng_state
from tests import refstandin as R
from tests.golden.cases import CASES, build_case


def _bytes(arr, n):
    return ctypes.string_at(ctypes.addressof(arr), ctypes.sizeof(arr._type_) * n)


@pytest.mark.parametrize("name", CASES)
def test_reference_objects_pack_like_ours(name):
    R0, phys, sim, _ = build_case(name)
    n = len(R0)
    p1, s1, a1 = _abi.pack_batch([phys], [sim], [n])
    p2, s2, a2 = _abi.pack_batch([R.phys_like(phys)], [R.sim_like(sim)], [n])
    assert _bytes(p1, 1) == _bytes(p2, 1)
    assert _bytes(s1, 1) == _bytes(s2, 1)
    assert np.array_equal(a1, a2)


def test_external_force_state_round_trips_in_the_reference_layout():
    _, phys, _, _ = build_case("ilc_timeflow_external")
    st = phys.external.__getstate__()
    assert len(st) == 6 and all(isinstance(x, list) for x in st)
    beads, is_const, consts, times, ntimes, values = st
    assert len(consts) == 3 * len(beads) and len(values) == 3 * len(times) == 3 * sum(ntimes)
    q = B.ExternalForce()
    q.__setstate__(st)
    assert q.entries() == phys.external.entries()


def test_reference_rng_state_is_read_and_written_through_its_pickled_state():
    g = R.Rng(42)
    assert rng_state(g) == (1, -1, 42)
    set_rng_state(g, (5, 6, 7))
    assert g.__getstate__() == (5, 6, 7)


def test_reference_reducers_map_to_the_batched_ones():
    assert ensemble.batched_reducer(R.reducer_named("bdsim.ensemble", "final_state")) is ensemble.final_state
    assert ensemble.batched_reducer(R.reducer_named("bdsim.ensemble", "sampled_states")) is ensemble.sampled_states
    for name in ("stress_series", "viscosity_series", "viscosity_series_vr"):
        assert ensemble.batched_reducer(R.reducer_named("bdsim.rheology", name)) is getattr(rheology, name)
    assert ensemble.batched_reducer(R.reducer_named("mypackage", "final_state")) is None
    assert ensemble.batched_reducer(ensemble.final_state) is ensemble.final_state


def test_control_chain_flow_keeps_the_callers_type():
    _, phys, _, _ = build_case("cfg2_fene_cheb_gauss")
    q = R.phys_like(phys)
    import copy
    ctl = rheology.control_phys(q)
    assert type(ctl.flow) is R.Flow and ctl.flow.__getstate__()[0] is True
    assert not any(ctl.flow.__getstate__()[1])
    assert q.flow.__getstate__() == phys.flow.__getstate__()  # the caller's object is untouched
