"""Parameter objects with the same names, fields, defaults and pickled state as
bdsim's compiled core (bindings/module.cpp:167-317 of the bdsim project).

They are plain Python here because the integrator they describe runs on the
GPU: `PhysParams`/`SimParams` are marshalled into the C ABI records of
include/bdsim_cuda.h by `bdsim_b200._abi.pack_batch`.
"""
from __future__ import annotations

import enum

import numpy as np


class _CoreEnum(enum.IntEnum):
    """Integer enum printing as `Type.Name`, like the nanobind enums."""

    def __str__(self):
        return f"{type(self).__name__}.{self.name}"

    __repr__ = __str__


class Spring(_CoreEnum):
    """Spring force laws (src/types.hpp:27-35)."""
    Hook = 1
    FENE = 2
    ILC = 3
    WLC = 4
    Fraenkel = 5
    FENEFraenkel = 6
    WLCbounded = 7


class EV(_CoreEnum):
    """Excluded-volume potentials (src/types.hpp:38-44)."""
    None_ = 0
    Gauss = 1
    LJ = 2
    SDK = 3
    SDKstickers = 4


class Bending(_CoreEnum):
    """Bending potentials (src/types.hpp:47-50)."""
    None_ = 0
    OneMinusCosTheta = 1


class DelSMethod(_CoreEnum):
    """Brownian square-root method under HI (src/types.hpp:53)."""
    Chebyshev = 0
    Cholesky = 1
    ExactSqrt = 2


class SpringParams:
    """SpringParams (src/spring.hpp:12-19)."""

    def __init__(self):
        self.type = Spring.Hook
        self.sqrtb = 10.0
        self.natural_length = 0.0

    def __getstate__(self):
        return (int(self.type), float(self.sqrtb), float(self.natural_length))

    def __setstate__(self, s):
        self.type, self.sqrtb, self.natural_length = Spring(s[0]), float(s[1]), float(s[2])


class EVParams:
    """EVParams (src/excluded_volume.hpp:17-25). `phi` is a row-major N*N list
    of SDK attractive strengths (empty => zeros)."""

    def __init__(self):
        self.type = EV.None_
        self.zstar = 0.0
        self.dstar = 0.0
        self.min_cutoff = 0.7
        self.max_cutoff = 1.5
        self.contour_dist_for_EV = 1
        self.phi = []

    def __getstate__(self):
        return (int(self.type), float(self.zstar), float(self.dstar), float(self.min_cutoff),
                float(self.max_cutoff), int(self.contour_dist_for_EV), list(map(float, self.phi)))

    def __setstate__(self, s):
        self.type = EV(s[0])
        self.zstar, self.dstar, self.min_cutoff, self.max_cutoff = map(float, s[1:5])
        self.contour_dist_for_EV = int(s[5])
        self.phi = list(s[6])


class BendingParams:
    """BendingParams (src/bending.hpp:9-12)."""

    def __init__(self):
        self.type = Bending.None_
        self.stiffness = 0.0

    def __getstate__(self):
        return (int(self.type), float(self.stiffness))

    def __setstate__(self, s):
        self.type, self.stiffness = Bending(s[0]), float(s[1])


class Flow:
    """Velocity-gradient tensor kappa, constant or tabulated and linearly
    interpolated with clamping (src/flow.hpp:17-43, src/flow.cpp:5-26)."""

    def __init__(self):
        self._constant = True
        self._k0 = np.zeros((3, 3))
        self._times = np.zeros(0)
        self._ks = np.zeros((0, 3, 3))

    @staticmethod
    def constant(kappa) -> "Flow":
        f = Flow()
        f._k0 = np.array(kappa, dtype=np.float64).reshape(3, 3).copy()
        return f

    @staticmethod
    def time_varying(times, kappas) -> "Flow":
        f = Flow()
        f._constant = False
        f._times = np.asarray(times, dtype=np.float64).copy()
        f._ks = np.asarray(kappas, dtype=np.float64).reshape(-1, 3, 3).copy()
        if len(f._times) != len(f._ks):
            raise ValueError("times and kappas must have the same length")
        return f

    def is_constant(self) -> bool:
        return self._constant or len(self._times) == 0

    def __getstate__(self):
        return (bool(self._constant), list(self._k0.reshape(-1)), list(self._times),
                list(self._ks.reshape(-1)))

    def __setstate__(self, s):
        self._constant = bool(s[0])
        self._k0 = np.array(s[1], dtype=np.float64).reshape(3, 3)
        self._times = np.array(s[2], dtype=np.float64)
        self._ks = np.array(s[3], dtype=np.float64).reshape(-1, 3, 3)


class ExternalForce:
    """User-applied bead forces, constant or time-interpolated
    (src/external_force.hpp:32-57). Negative bead indices count from the end."""

    def __init__(self):
        self._entries = []  # (bead, is_const, value(3), times, values(n,3))

    def add_constant(self, bead, force):
        self._entries.append((int(bead), True, tuple(map(float, force)), (), ()))

    def add_time_varying(self, bead, times, forces):
        times = tuple(map(float, times))
        vals = tuple(tuple(map(float, v)) for v in forces)
        if len(times) != len(vals):
            raise ValueError("times and forces must have the same length")
        self._entries.append((int(bead), False, (0.0, 0.0, 0.0), times, vals))

    def add_stretch(self, bead_minus, bead_plus, force):
        f = tuple(map(float, force))
        self.add_constant(bead_plus, f)
        self.add_constant(bead_minus, tuple(-x for x in f))

    def empty(self) -> bool:
        return not self._entries

    def entries(self):
        return list(self._entries)

    def __getstate__(self):
        """Parallel arrays (beads, is_const, consts, times, ntimes, values), the
        pickled layout of the reference's ExternalForce
        (bindings/module.cpp:83-99)."""
        beads, is_const, consts, times, ntimes, values = [], [], [], [], [], []
        for bead, const, val, ts, vs in self._entries:
            beads.append(int(bead))
            is_const.append(1 if const else 0)
            consts.extend(float(v) for v in val)
            ntimes.append(len(ts))
            times.extend(float(t) for t in ts)
            for v in vs:
                values.extend(float(x) for x in v)
        return (beads, is_const, consts, times, ntimes, values)

    def __setstate__(self, s):
        self._entries = list(external_entries(s))


def external_entries(state):
    """(bead, is_const, value(3), times, values) per entry, from an
    ExternalForce state tuple in the reference's layout."""
    beads, is_const, consts, times, ntimes, values = state
    ti = vi = 0
    for k, bead in enumerate(beads):
        n = int(ntimes[k])
        ts = tuple(float(t) for t in times[ti:ti + n])
        vs = tuple(tuple(float(x) for x in values[vi + 3 * j:vi + 3 * j + 3]) for j in range(n))
        ti += n
        vi += 3 * n
        yield (int(bead), bool(is_const[k]), tuple(float(x) for x in consts[3 * k:3 * k + 3]), ts, vs)


def rng_state(rng):
    """(ix, iy, seed) of an Rng: this package's or the reference's, whose only
    accessor is its pickled state (bindings/module.cpp:302-303)."""
    return tuple(int(v) for v in rng.__getstate__())


def set_rng_state(rng, state):
    """Write (ix, iy, seed) back into an Rng of either package."""
    rng.__setstate__(tuple(int(v) for v in state))


class PhysParams:
    """PhysParams (src/model.hpp:20-35)."""

    def __init__(self):
        self.spring = SpringParams()
        self.ev = EVParams()
        self.bend = BendingParams()
        self.flow = Flow()
        self.external = ExternalForce()
        self.number_of_beads = 10
        self.hstar = 0.0
        self.hi_method = DelSMethod.Chebyshev
        self.ncheb_multiplier = 1.0
        self.fd_err_max = 0.0025
        self.equilibration = False

    def __getstate__(self):
        return (self.spring, self.ev, self.bend, self.flow, int(self.number_of_beads),
                float(self.hstar), int(self.hi_method), float(self.ncheb_multiplier),
                float(self.fd_err_max), bool(self.equilibration), self.external)

    def __setstate__(self, s):
        (self.spring, self.ev, self.bend, self.flow, self.number_of_beads, self.hstar,
         hi, self.ncheb_multiplier, self.fd_err_max, self.equilibration, self.external) = s
        self.hi_method = DelSMethod(hi)


class SimParams:
    """SimParams (src/integrator.hpp:22-28)."""

    def __init__(self):
        self.time_start = 0.0
        self.time_end = 1.0
        self.dt = 0.01
        self.implicit_loop_tol = 1e-3
        self.update_center_of_mass = True

    def __getstate__(self):
        return (float(self.time_start), float(self.time_end), float(self.dt),
                float(self.implicit_loop_tol), bool(self.update_center_of_mass))

    def __setstate__(self, s):
        (self.time_start, self.time_end, self.dt, self.implicit_loop_tol,
         self.update_center_of_mass) = s


class Rng:
    """Numerical Recipes ran_1 stream state {ix, iy, seed} (src/rng.hpp:25-63).

    A fresh generator has ix=1, iy=-1, which triggers the lazy seeding of
    Rng::maybe_init (src/rng.cpp:31-39) on the first draw. Draws happen on
    the device; the state is uploaded and written back by the integrator.
    """

    def __init__(self, seed: int = 123):
        self.reset(seed)

    def reset(self, seed: int):
        self.ix, self.iy, self.seed = 1, -1, int(seed)

    def state(self):
        return (int(self.ix), int(self.iy), int(self.seed))

    def set_state(self, s):
        self.ix, self.iy, self.seed = (int(v) for v in s)

    def __getstate__(self):
        return self.state()

    def __setstate__(self, s):
        self.set_state(s)

    def __repr__(self):
        return f"Rng(ix={self.ix}, iy={self.iy}, seed={self.seed})"
