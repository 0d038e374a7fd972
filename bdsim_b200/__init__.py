"""bdsim_b200 -- B200-native ensemble integrator for bdsim's ChainIntegrator step.

The public names mirror bdsim's package (python/bdsim/__init__.py of the bdsim
project): the parameter types, the core functions (`integrate`,
`total_force`, ...), initial configurations, observables, and the run layer
(`simulate`, `run_ensemble`) whose backend="cuda" advances every trajectory of
an ensemble together on one GPU. Every integration runs in the CUDA library
libbdsim_cuda.so; there is no CPU fallback.
"""
from .params import (Spring, EV, Bending, DelSMethod, SpringParams, EVParams, BendingParams,
                     PhysParams, SimParams, Flow, Rng, ExternalForce)
from .core import (integrate, integrate_many, total_force, total_force_many, spring_force, bending_force,
                   ev_force, external_force, IntegratorError)
from .engine import Context, Ensemble
from . import flows, initial, properties, storage, failures, ensemble, rheology
from .initial import (gaussian_chain, fene_fraenkel_chain, fene_fraenkel_chain_aligned_x, equilibrium_chain,
                      fene_fraenkel_bending_chain, one_minus_cos_theta_angles, isotropic_directions)
from .properties import (end_to_end_sq, radius_of_gyration_sq, gyration_tensor, stretch, kramers_stress,
                         shear_viscosity as shear_viscosity_config, normal_stress_differences)
from .ensemble import (Initial, Output, INITIALIZERS, n_steps_of, simulate, run_ensemble, trajectory_samples,
                       final_state, sampled_states, mean_stderr, MAX_FAILED_FRACTION)
from .storage import read_run, read_trajectory, Run, Trajectory, map_property, ensemble_average
from .failures import Failure

__all__ = [
    "Spring", "EV", "Bending", "DelSMethod", "SpringParams", "EVParams", "BendingParams", "PhysParams",
    "SimParams", "Flow", "Rng", "ExternalForce", "integrate", "integrate_many", "total_force",
    "total_force_many", "spring_force", "bending_force", "ev_force", "external_force", "IntegratorError",
    "Context", "Ensemble", "flows", "initial", "properties", "storage", "failures", "ensemble", "rheology",
    "gaussian_chain", "fene_fraenkel_chain", "fene_fraenkel_chain_aligned_x", "equilibrium_chain",
    "fene_fraenkel_bending_chain", "one_minus_cos_theta_angles", "isotropic_directions",
    "end_to_end_sq", "radius_of_gyration_sq", "gyration_tensor", "stretch", "kramers_stress",
    "shear_viscosity_config", "normal_stress_differences", "Initial", "Output", "INITIALIZERS", "n_steps_of",
    "simulate", "run_ensemble", "trajectory_samples", "final_state", "sampled_states", "mean_stderr",
    "MAX_FAILED_FRACTION", "read_run", "read_trajectory", "Run", "Trajectory", "map_property",
    "ensemble_average", "Failure",
]
