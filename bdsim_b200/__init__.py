"""bdsim_b200 -- B200-native ensemble integrator for bdsim's ChainIntegrator step.

The public names mirror bdsim's package (python/bdsim/__init__.py of the bdsim
project): the parameter types, the core functions (`integrate`,
`total_force`, ...), and the run layer (`simulate`, `run_ensemble`) whose
backend="cuda" runs every trajectory of an ensemble on one GPU.
"""
from .params import (Spring, EV, Bending, DelSMethod, SpringParams, EVParams, BendingParams,
                     PhysParams, SimParams, Flow, Rng, ExternalForce)
from .core import (integrate, integrate_many, total_force, total_force_many, spring_force, bending_force,
                   ev_force, external_force, IntegratorError)
from .engine import Context, Ensemble
