"""backend="cuda" routed from the reference's run layer: its own objects in,
the same results as this package's objects, bit for bit."""
import os

import numpy as np
import pytest

import bdsim_b200 as B
from tests import refstandin as R
from tests.golden.cases import build_case

pytestmark = pytest.mark.gpu


def _reference_simulate(phys, sim, *, n_traj=1, seed=0, n_steps=None, initial=None, output=None,
                        backend="serial", n_workers=None, on_error="skip", max_failed_fraction=None):
    """The first lines the routing adds to the reference's simulate."""
    if backend == "cuda":
        return B.simulate(phys, sim, n_traj=n_traj, seed=seed, n_steps=n_steps, initial=initial, output=output,
                          backend="cuda", on_error=on_error, max_failed_fraction=max_failed_fraction)
    raise AssertionError("the CPU path of the reference is not exercised here")


def _reference_run_ensemble(phys, sim, n_traj, per_trajectory, *, args=(), seed=0, initial=None,
                            backend="serial", n_workers=None, on_error="skip", max_failed_fraction=None):
    if backend == "cuda":
        return B.run_ensemble(phys, sim, n_traj, per_trajectory, args=args, seed=seed, initial=initial,
                              backend="cuda", on_error=on_error, max_failed_fraction=max_failed_fraction)
    raise AssertionError("the CPU path of the reference is not exercised here")


@pytest.mark.parametrize("name", ["cfg1_ff_cholesky", "cfg2_fene_cheb_gauss", "ilc_timeflow_external"])
def test_simulate_with_reference_objects_matches_ours(tmp_path, name):
    _, phys, sim, _ = build_case(name)
    n_steps = 12
    init = B.Initial("gaussian", {})
    a = _reference_simulate(R.phys_like(phys), R.sim_like(sim), n_traj=5, seed=3, n_steps=n_steps, initial=init,
                            output=B.Output(directory=str(tmp_path / "ref"), write_every=5), backend="cuda")
    b = B.simulate(phys, sim, n_traj=5, seed=3, n_steps=n_steps, initial=init,
                   output=B.Output(directory=str(tmp_path / "ours"), write_every=5))
    assert len(a) == len(b) == 5
    for ta, tb in zip(a, b):
        assert np.array_equal(ta.step, tb.step)
        assert np.array_equal(ta.time, tb.time)
        assert np.array_equal(ta.positions, tb.positions)
        assert list(ta.step) == [0, 5, 10, 12]


def test_run_ensemble_maps_the_reference_reducer_to_the_batched_path():
    _, phys, sim, _ = build_case("cfg2_fene_cheb_gauss")
    ref_final_state = R.reducer_named("bdsim.ensemble", "final_state")  # raises if it were called
    a = _reference_run_ensemble(R.phys_like(phys), R.sim_like(sim), 6, ref_final_state, seed=11, backend="cuda")
    b = B.run_ensemble(phys, sim, 6, B.final_state, seed=11)
    assert len(a) == len(b) == 6
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
