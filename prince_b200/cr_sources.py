"""Cosmic-ray source models: the injection term ``b(z)`` of the transport equation.

A source factorises into a fixed per-state injection grid ``g`` (set at
construction from the spectrum of each injected species) and a scalar
redshift dependence: ``injection_rate(z) = norm * evolution(z) * g``.  This
is the interface the reference solvers consume
(``src/prince_cr/cr_sources.py:14-162``); the spectral shapes keep the
reference's class names and parameter tuples (``cr_sources.py:165-317``).

Additions for the batched path: ``z_max`` switches a source off above a
redshift (the source injects nothing while ``z > z_max``), and
``evolution_array`` evaluates the redshift dependence on a whole z grid at
once so per-step coefficients for hundreds of columns are built without a
Python loop per step.
"""

from __future__ import annotations

from abc import ABCMeta, abstractmethod

import numpy as np

from .cosmology import agn_rate, grb_rate_wp, star_formation_rate


class CosmicRaySource(metaclass=ABCMeta):
    """Base class: precomputes ``injection_grid`` (length ``dim_states``).

    ``params`` maps PDG id to the spectral parameter tuple of the subclass;
    ``m`` is the evolution: ``"flat"``, a float (``(1+z)^m * SFR(z)``) or a
    tuple ``(keyword, m)`` with keyword in SFR, GRB, AGN, TDE, simple,
    simple_flat, simple_SFR (``cr_sources.py:90-162``).
    """

    def __init__(self, prince_run, pdgids=None, params=None, norm=1.0, m="flat",
                 z_max=None, *args, **kwargs):
        self.cr_grid = prince_run.cr_grid.grid
        self.dim_states = prince_run.dim_states
        self.norm = norm
        self.spec_man = prince_run.spec_man
        self.params = params
        self.pdgids = np.array(pdgids if pdgids is not None else list(params.keys()))
        self.pdgids.sort()
        self.source_evo_m = m
        self.z_max = None if z_max is None else float(z_max)
        self._compute_injection_grid()

    def _compute_injection_grid(self):
        self.injection_grid = np.zeros(self.dim_states)
        blocks = []
        for pid in self.pdgids:
            sref = self.spec_man.pdgid2sref[int(pid)]
            with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
                self.injection_grid[sref.sl] = self.injection_spectrum(
                    int(pid), self.cr_grid, self.params[int(pid)]
                )
            blocks.append(np.arange(sref.sl.start, sref.sl.stop))
        # states with a non-zero injection (only the injected species' blocks are written)
        idx = np.unique(np.concatenate(blocks)) if blocks else np.zeros(0, dtype=np.int64)
        self.injection_support = idx[self.injection_grid[idx] != 0.0]

    def injection_rate(self, z):
        """``norm * evolution(z) * injection_grid`` on the state grid."""
        return self.norm * self.evolution(z) * self.injection_grid

    @abstractmethod
    def injection_spectrum(self, pid, energy, params):
        """Spectrum of species ``pid`` on the per-nucleon energies ``energy``."""

    def evolution(self, z):
        """Relative source density at redshift ``z`` (scalar)."""
        if z < 0:
            raise Exception("Source evolution not defined for negative z = {:}".format(z))
        if self.z_max is not None and z > self.z_max:
            return 0.0
        m = self.source_evo_m
        if m == "flat":
            return 1.0
        if type(m) is float:
            return (1 + z) ** m * star_formation_rate(z)
        if type(m) is tuple:
            kwd, mval = m
            if kwd == "SFR":
                return (1 + z) ** mval * star_formation_rate(z)
            if kwd == "GRB":
                return (1 + z) ** mval * grb_rate_wp(z)
            if kwd == "AGN":
                return (1 + z) ** mval * agn_rate(z)
            if kwd == "TDE":
                return (1 + z) ** (mval - 3.0)
            if kwd == "simple":
                return (1 + z) ** mval
            if kwd == "simple_flat":
                return (1 + z) ** mval if z <= 1 else (1 + 1) ** mval
            if kwd == "simple_SFR":
                return (1 + z) ** mval if z <= 1 else (1 + 1) ** 3.6 * (1 + z) ** (mval - 3.6)
        raise Exception("Unknown source evo type: {:}".format(m))

    def evolution_array(self, z):
        """``evolution`` on an array of redshifts (vectorised for the common shapes)."""
        z = np.asarray(z, dtype=np.float64)
        m = self.source_evo_m
        if m == "flat":
            out = np.ones_like(z)
        elif type(m) is tuple and m[0] == "simple":
            out = (1 + z) ** m[1]
        elif type(m) is tuple and m[0] == "TDE":
            out = (1 + z) ** (m[1] - 3.0)
        else:
            out = np.array([self.evolution(float(zz)) for zz in z.ravel()]).reshape(z.shape)
            return out
        if np.any(z < 0):
            raise Exception("Source evolution not defined for negative z")
        if self.z_max is not None:
            out = np.where(z > self.z_max, 0.0, out)
        return out


class SimpleSource(CosmicRaySource):
    """``norm * E^-gamma * exp(-E / (Emax/A))``; params ``{pid: (gamma, Emax, norm)}``."""

    def injection_spectrum(self, pid, energy, params):
        gamma, emax, norm = params
        emax = emax / self.spec_man.pdgid2sref[pid].A
        return norm * energy ** (-gamma) * np.exp(-energy / emax)


class RigdityCutoffSource(CosmicRaySource):
    """``relnorm * A * (A E / 1 GeV)^-gamma * exp(1 - A E / (Z Rcut))``.

    params ``{pid: (gamma, Rcut, relnorm)}``.  Neutrons (Z = 0) get a zero
    spectrum through the exponential, as in ``cr_sources.py:182-198``.
    """

    def injection_spectrum(self, pid, energy, params):
        spectral_index, rcut, relnorm = params
        sref = self.spec_man.pdgid2sref[pid]
        A = float(sref.A)
        emax = rcut * sref.Z
        e_k = A * energy
        return relnorm * A * (e_k / 1e9) ** (-spectral_index) * np.exp(1 - e_k / emax)


class AugerFitSource(CosmicRaySource):
    """Power law below ``Z * Rcut``, times ``exp(1 - E/(Z Rcut))`` above it."""

    def injection_spectrum(self, pid, energy, params):
        spectral_index, rcut, relnorm = params
        sref = self.spec_man.pdgid2sref[pid]
        A = float(sref.A)
        emax = rcut * sref.Z
        e_k = A * energy
        return (relnorm * A * (e_k / 1e9) ** (-spectral_index)
                * np.where(e_k < emax, 1.0, np.exp(1 - e_k / emax)))


class SechCutoffSource(CosmicRaySource):
    """``relnorm * A * (E_k/1 GeV)^-gamma * sech((E_k / (Z Rcut))^2)``."""

    def injection_spectrum(self, pid, energy, params):
        spectral_index, rcut, relnorm = params
        sref = self.spec_man.pdgid2sref[pid]
        A = float(sref.A)
        emax = rcut * sref.Z
        e_k = A * energy
        ratio_sq = (e_k / emax) ** 2
        with np.errstate(over="ignore"):
            cutoff = 1.0 / np.cosh(ratio_sq)
        cutoff = np.where(np.isfinite(cutoff), cutoff, 0.0)
        return relnorm * A * (e_k / 1e9) ** (-spectral_index) * cutoff


class RigidityFlexSource(CosmicRaySource):
    """Like ``AugerFitSource`` with cutoff at ``Z^alpha * Rcut``; params (gamma, Rcut, alpha, norm)."""

    def injection_spectrum(self, pid, energy, params):
        spectral_index, rcut, alpha, relnorm = params
        sref = self.spec_man.pdgid2sref[pid]
        A = float(sref.A)
        emax = rcut * sref.Z ** alpha
        e_k = A * energy
        return (relnorm * A * (e_k / 1e9) ** (-spectral_index)
                * np.where(e_k < emax, 1.0, np.exp(1 - e_k / emax)))


class SpectrumSource(CosmicRaySource):
    """Tabulated spectrum ``{pid: (egrid, specgrid)}`` in total energy, interpolated."""

    def injection_spectrum(self, pid, energy, params):
        egrid, specgrid = params
        A = self.spec_man.pdgid2sref[pid].A
        return np.interp(energy, egrid / A, specgrid * A, left=0.0, right=0.0)
