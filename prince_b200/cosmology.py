"""Flat Lambda-CDM expansion rate and the source-evolution shapes.

``H`` follows ``src/prince_cr/cosmology.py:10-21``; the evolution shapes
(star formation, GRB, AGN) follow ``cosmology.py:24-110``.  All functions
accept scalars or numpy arrays.
"""

from __future__ import annotations

import numpy as np

from . import constants as C


def H(z, H0=C.H_0s):
    """Expansion rate in 1/s: ``H0 * sqrt(Omega_m (1+z)^3 + Omega_Lambda)``."""
    return H0 * np.sqrt(C.Omega_m * (1 + z) ** 3 + C.Omega_Lambda)


def dldz(z):
    """Comoving path length per unit redshift, ``-1 / ((1+z) H(z) cm2sec)`` in cm.

    Same expression as ``UHECRPropagationSolver.dldz``
    (``src/prince_cr/solvers/propagation.py:360-361``).
    """
    return -1.0 / ((1.0 + z) * H(z) * C.PRINCE_UNITS.cm2sec)


def star_formation_rate(z, z_inhom=0.0):
    """Hopkins & Beacom star-formation history, normalised to 1 at z = 0."""
    if z < z_inhom:
        return 0.0
    if z <= 0.97:
        return (1.0 + z) ** 3.44
    if z <= 4.48:
        return 10.0 ** 1.09 * (1.0 + z) ** -0.26
    return 10.0 ** 6.66 * (1.0 + z) ** -7.8


def grb_rate_wp(z, z_inhom=0.0):
    """Wanderman & Piran GRB rate history, normalised to 1 at z = 0."""
    if z < z_inhom:
        return 0.0
    if z <= 3:
        return (1 + z) ** 2.1
    return (1 + 3) ** (2.1 + 1.4) * (1 + z) ** -1.4


def agn_rate(z, z_inhom=0.0):
    """AGN rate history, normalised to 1 at z = 0."""
    if z < z_inhom:
        return 0.0
    if z <= 1.7:
        return (1 + z) ** 5
    if z <= 2.7:
        return (1 + 1.7) ** 5
    return (1 + 1.7) ** 5 * 10 ** (2.7 - z)
