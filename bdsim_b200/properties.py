"""Per-configuration observables from an (N, 3) positions array
(python/bdsim/properties.py of the bdsim project). Host-side analysis helpers;
the device computes the forces they take (`total_force`)."""
import numpy as np


def end_to_end_sq(R: np.ndarray) -> float:
    """|R_N - R_1|^2."""
    d = R[-1] - R[0]
    return float(d @ d)


def gyration_tensor(R: np.ndarray) -> np.ndarray:
    """3x3 gyration tensor about the centre of mass."""
    X = R - R.mean(axis=0)
    return (X.T @ X) / len(R)


def radius_of_gyration_sq(R: np.ndarray) -> float:
    """Rg^2 = trace of the gyration tensor."""
    return float(np.trace(gyration_tensor(R)))


def stretch(R: np.ndarray) -> np.ndarray:
    """Extent (max - min) of the centred chain along each axis."""
    X = R - R.mean(axis=0)
    return X.max(axis=0) - X.min(axis=0)


def kramers_stress(R: np.ndarray, F: np.ndarray) -> np.ndarray:
    """Kramers-Kirkwood stress tau_ij = sum_mu (R_mu - R_c)_i F_mu,j."""
    return (R - R.mean(axis=0)).T @ F


def shear_viscosity(R: np.ndarray, F: np.ndarray, rate: float) -> float:
    """Polymer shear viscosity -tau_xy / rate."""
    return -kramers_stress(R, F)[0, 1] / rate


def normal_stress_differences(R: np.ndarray, F: np.ndarray):
    """(N1, N2) = (tau_xx - tau_yy, tau_yy - tau_zz)."""
    s = kramers_stress(R, F)
    return s[0, 0] - s[1, 1], s[1, 1] - s[2, 2]
