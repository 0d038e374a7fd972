"""Velocity-gradient tensors of common flows as Flow objects
(python/bdsim/flows.py of the bdsim project)."""
import numpy as np

from .params import Flow


def equilibrium() -> Flow:
    """No flow (kappa = 0)."""
    return Flow()


def shear(rate: float) -> Flow:
    """Simple shear v = (rate*y, 0, 0): kappa[0][1] = rate."""
    K = np.zeros((3, 3))
    K[0, 1] = rate
    return Flow.constant(K)


def uniaxial_extension(rate: float) -> Flow:
    """Uniaxial extension diag(rate, -rate/2, -rate/2)."""
    return Flow.constant(np.diag([rate, -rate / 2.0, -rate / 2.0]))


def planar_extension(rate: float) -> Flow:
    """Planar extension diag(rate, -rate, 0)."""
    return Flow.constant(np.diag([rate, -rate, 0.0]))
