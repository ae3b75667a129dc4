"""Turbulon envelope shapes (steam/turbulons.py:1-48).

``SHAPES`` is the registry of valid shape names.  The envelopes are evaluated
on the device by ``steam_kernel_build`` (see simulate._turbulon_envelope); the
host functions below are the same formulas for callers that evaluate a shape
on their own radius array.  Shape codes are the C-ABI's ``shape`` argument.
"""

import numpy as np

SHAPES = {'mexican_hat', 'morlet_omega0_6'}
SHAPE_CODES = {'mexican_hat': 0, 'morlet_omega0_6': 1}


def mexican_hat(r_norm_sq, k):
    """(3 - rho) exp(-rho/2), rho = r^2 / (k/pi)^2 (steam/turbulons.py:23-37)."""
    ratio_sq = r_norm_sq / (k / np.pi) ** 2
    return (3.0 - ratio_sq) * np.exp(-ratio_sq / 2.0)


def morlet_omega0_6(r_norm_sq, k):
    """cos(6 r / k) exp(-rho/2) (steam/turbulons.py:40-48)."""
    ratio_sq = r_norm_sq / (k / np.pi) ** 2
    omega_0 = 6.0 / k
    return np.cos(omega_0 * np.sqrt(r_norm_sq)) * np.exp(-ratio_sq / 2.0)
