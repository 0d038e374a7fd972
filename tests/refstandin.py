"""Stand-ins with the Python surface of the reference's compiled objects.

bdsim's parameter types come from a nanobind module (bindings/module.cpp:167-317
of the bdsim project) that cannot be built here. These classes reproduce the
surface that module gives them, and nothing more:
  * enums are plain enum.Enum types (no int()); the integer is `.value`;
  * SpringParams, EVParams, BendingParams, PhysParams and SimParams are records
    of read-write attributes;
  * Flow, ExternalForce and Rng expose no attributes, only their methods and
    their pickled state in the module's layout (bindings/module.cpp:83-99,
    140-148, 302-306).
They are filled from this package's objects so both describe the same chain.
"""
from __future__ import annotations

import enum

import bdsim_b200 as B


class Spring(enum.Enum):
    Hook = 1
    FENE = 2
    ILC = 3
    WLC = 4
    Fraenkel = 5
    FENEFraenkel = 6
    WLCbounded = 7


class EV(enum.Enum):
    None_ = 0
    Gauss = 1
    LJ = 2
    SDK = 3
    SDKstickers = 4


class Bending(enum.Enum):
    None_ = 0
    OneMinusCosTheta = 1


class DelSMethod(enum.Enum):
    Chebyshev = 0
    Cholesky = 1
    ExactSqrt = 2


class _Record:
    pass


class Flow:
    def __init__(self, state=None):
        self._s = state if state is not None else (True, [0.0] * 9, [], [])

    def __getstate__(self):
        return self._s

    def __setstate__(self, s):
        self._s = s


class ExternalForce:
    def __init__(self, state=None):
        self._s = state if state is not None else ([], [], [], [], [], [])

    def __getstate__(self):
        return self._s

    def __setstate__(self, s):
        self._s = s

    def empty(self):
        return not self._s[0]


class Rng:
    def __init__(self, seed=123):
        self._s = (1, -1, int(seed))

    def __getstate__(self):
        return self._s

    def __setstate__(self, s):
        self._s = tuple(int(v) for v in s)


def phys_like(p: B.PhysParams):
    """A stand-in PhysParams equal to this package's `p`."""
    q = _Record()
    q.spring = _Record()
    q.spring.type = Spring(int(p.spring.type))
    q.spring.sqrtb = p.spring.sqrtb
    q.spring.natural_length = p.spring.natural_length
    q.ev = _Record()
    q.ev.type = EV(int(p.ev.type))
    for k in ("zstar", "dstar", "min_cutoff", "max_cutoff", "contour_dist_for_EV"):
        setattr(q.ev, k, getattr(p.ev, k))
    q.ev.phi = list(p.ev.phi)
    q.bend = _Record()
    q.bend.type = Bending(int(p.bend.type))
    q.bend.stiffness = p.bend.stiffness
    q.flow = Flow(p.flow.__getstate__())
    q.external = ExternalForce(p.external.__getstate__())
    q.number_of_beads = p.number_of_beads
    q.hstar = p.hstar
    q.hi_method = DelSMethod(int(p.hi_method))
    q.ncheb_multiplier = p.ncheb_multiplier
    q.fd_err_max = p.fd_err_max
    q.equilibration = p.equilibration
    return q


def sim_like(s: B.SimParams):
    q = _Record()
    for k in ("time_start", "time_end", "dt", "implicit_loop_tol", "update_center_of_mass"):
        setattr(q, k, getattr(s, k))
    return q


def reducer_named(module: str, name: str):
    """A function object that looks like the reference's `module.name`."""
    def fn(*a, **k):
        raise AssertionError("the reference's reducer must not run on the cuda backend")
    fn.__module__ = module
    fn.__qualname__ = name
    fn.__name__ = name
    return fn
