"""Seeded synthetic photo-nuclear models and the benchmark workloads built on them.

No cross-section database is available offline, so the workloads use an
analytic model with realistic shapes and magnitudes:

* every nucleus has a giant-dipole resonance (Lorentzian, Berman-Fultz peak
  ``31.2 A^-1/3 + 20.6 A^-1/6`` MeV, strength from the TRK sum rule) plus a
  photo-pion bump at 0.34 GeV; free nucleons have the pion bump only;
* boost-conserving channels go to lighter residual nuclei and to the light
  fragments (2H, 3H, 3He, 4He) at equal Lorentz factor, with seeded
  branchings that differ between the resonance and the pion component;
* free nucleons (p, n) are redistributed in ``x = E_daughter/E_mother`` with
  a cumulative distribution ``H(x) = multiplicity * x^a``.

The fold kernel is assembled on the log grid of the rate integral: for a
rest-frame cross section ``sigma(eps)`` the response is
``g(y) = (1/2y^2) int_0^{2y} eps sigma(eps) deps`` with ``y = E eps / m_p``
and ``R(y) = int g dy``.  With both grids on the same log step the kernel
row of mother bin ``i`` at photon bin ``j`` is ``(m_p/E_i) dR[i+j]`` for a
boost-conserving channel, and
``(m_p/E_mo)(dE_mo/dE_da) dR[i_mo+j] dH[i_da-i_mo+d-1]`` for a redistributed
one (the kernel definition of ``src/prince_cr/interaction_rates.py:251-263``),
with the redistribution cuts of ``interaction_rates.py:579-593``.
"""

from __future__ import annotations

import numpy as np

from . import constants as C
from .data import get_AZN, make_nucleus_pdg

_MB = 1e-27  # cm^2


def nuclide_chart(max_mass, per_isobar=6):
    """Seeded-free list of nuclide PDG ids with ``2 <= A <= max_mass`` near stability.

    For each A, up to ``per_isobar`` charges closest to the stability line
    ``Z = A / (1.98 + 0.0155 A^(2/3))`` with ``1 <= Z`` and ``N >= 1``.
    """
    out = []
    for A in range(2, int(max_mass) + 1):
        zs = A / (1.98 + 0.0155 * A ** (2.0 / 3.0))
        cands = [Z for Z in range(1, A) if A - Z >= 1]
        cands.sort(key=lambda Z: (abs(Z - zs), Z))
        for Z in sorted(cands[:per_isobar]):
            out.append(make_nucleus_pdg(A, Z))
    return out


def _lorentz(eps, e0, width, peak, thr):
    s = peak * (eps * width) ** 2 / ((eps ** 2 - e0 ** 2) ** 2 + (eps * width) ** 2)
    return np.where(eps > thr, s, 0.0)


def _sigma_components(A, Z):
    """(sigma_gdr, sigma_pion) callables in cm^2 of the rest-frame photon energy (GeV)."""
    N = A - Z
    if A >= 2:
        e0 = (31.2 * A ** (-1.0 / 3.0) + 20.6 * A ** (-1.0 / 6.0)) * 1e-3
        width = 5e-3
        trk = 60.0 * N * Z / A * _MB * 1e-3  # mb MeV -> cm^2 GeV
        peak = 2.0 * trk / (np.pi * width)
        thr = 2e-3 if A > 4 else 2.2e-3
        gdr = lambda e: _lorentz(e, e0, width, peak, thr)
    else:
        gdr = lambda e: np.zeros_like(e)
    pion = lambda e: (_lorentz(e, 0.34, 0.12, 0.5 * A * _MB, 0.145)
                      + np.where(e > 0.5, 0.12 * A * _MB, 0.0))
    return gdr, pion


def _response_increments(sigma, y_edges):
    """``dR[k] = R(y_{k+1}) - R(y_k)`` on the log y edges, by fine quadrature."""
    lo = np.log10(y_edges[0]) - 1.0
    hi = np.log10(y_edges[-1]) + 0.5
    yf = np.logspace(lo, hi, 4000)
    ef = np.concatenate([[0.0], 2.0 * yf])
    integrand = ef * sigma(ef)
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (integrand[1:] + integrand[:-1]) * np.diff(ef))])
    g = cum[1:] / (2.0 * yf ** 2)
    R = np.concatenate([[0.0], np.cumsum(0.5 * (g[1:] + g[:-1]) * np.diff(yf))])
    Ry = np.interp(np.log(y_edges), np.log(yf), R)
    return np.maximum(np.diff(Ry), 0.0)


# (dA, dZ, emitted light fragment or None) of boost-conserving residual channels.
_RESIDUALS = (
    (1, 0, None), (1, 1, None), (2, 0, None), (2, 1, 1000010020), (2, 2, None),
    (3, 1, 1000010030), (3, 2, 1000020030), (4, 2, 1000020040), (5, 2, 1000020040),
    (6, 3, 1000020040), (8, 4, 1000020040), (10, 5, 1000020040), (12, 6, 1000020040),
)


class SyntheticPhotoNuclear:
    """Seeded synthetic photo-nuclear model (``known_species`` / ``build_kernel``).

    Args:
        species: PDG ids in the network (nuclei, p, n).
        seed: RNG seed for the channel branchings and x-shapes.
        x_cut, x_cut_proton: lower x cut for redistributed neutron / proton daughters.
        max_residuals: cap on boost-conserving residual channels per mother.
    """

    def __init__(self, species, seed=0, x_cut=C.x_cut, x_cut_proton=C.x_cut_proton,
                 max_residuals=len(_RESIDUALS)):
        self.known_species = sorted(set(int(s) for s in species))
        self.seed = int(seed)
        self.x_cut = float(x_cut)
        self.x_cut_proton = float(x_cut_proton)
        self.max_residuals = int(max_residuals)
        self.lifetimes = {}
        self._plan_channels()

    def _plan_channels(self):
        rng = np.random.default_rng(self.seed)
        present = set(self.known_species)
        self.bc = {}    # (mo, da) -> (w_gdr, w_pion)
        self.diff = {}  # (mo, da) -> (mult_gdr, mult_pion, shape exponent)
        for mo in self.known_species:
            A, Z, N = get_AZN(mo)
            if A == 0:
                continue
            if A == 1:
                for da in (2212, 2112):
                    if da in present:
                        same = da == mo
                        self.diff[(mo, da)] = (0.0, 0.7 if same else 0.3, rng.uniform(1.5, 3.0))
                continue
            chans = []
            for dA, dZ, frag in _RESIDUALS:
                Ad, Zd = A - dA, Z - dZ
                if Ad < 1 or Zd < 0 or Zd > Ad:
                    continue
                res = make_nucleus_pdg(Ad, Zd)
                if res not in present or res == mo:
                    continue
                chans.append((dA, dZ, frag, res))
                if len(chans) >= self.max_residuals:
                    break
            if not chans:
                continue
            k = np.arange(len(chans))
            wg = np.exp(-1.2 * k) * rng.uniform(0.5, 1.5, len(chans))
            wp = np.exp(-0.35 * k) * rng.uniform(0.5, 1.5, len(chans))
            wg /= wg.sum()
            wp /= wp.sum()
            mult = {}
            for (dA, dZ, frag, res), g, p in zip(chans, wg, wp):
                nA, nZ = dA, dZ
                if get_AZN(res)[0] == 1:
                    # A free-nucleon residual is redistributed, not boost-conserving.
                    nA, nZ = dA + 1, dZ + get_AZN(res)[1]
                else:
                    self.bc[(mo, res)] = (self.bc.get((mo, res), (0.0, 0.0))[0] + g,
                                          self.bc.get((mo, res), (0.0, 0.0))[1] + p)
                if frag is not None and frag in present and frag != res:
                    fg, fp = self.bc.get((mo, frag), (0.0, 0.0))
                    self.bc[(mo, frag)] = (fg + g, fp + p)
                    fA, fZ, _ = get_AZN(frag)
                    nA, nZ = dA - fA, dZ - fZ
                mg, mp_ = mult.get("p", (0.0, 0.0))
                mult["p"] = (mg + g * nZ, mp_ + p * nZ)
                mg, mp_ = mult.get("n", (0.0, 0.0))
                mult["n"] = (mg + g * (nA - nZ), mp_ + p * (nA - nZ))
            for key, da in (("p", 2212), ("n", 2112)):
                if da in present and key in mult and (mult[key][0] > 0 or mult[key][1] > 0):
                    self.diff[(mo, da)] = (mult[key][0], mult[key][1], rng.uniform(2.0, 4.0))

    def build_kernel_spec(self, cr_grid, ph_grid, spec_man):
        """The fold kernel as per-channel response samples (``prince_b200.kernel_build``).

        Per mother: the non-elastic increments ``dR_gdr + dR_pion``; per
        boost-conserving channel ``w_gdr dR_gdr + w_pion dR_pion``; per
        redistributed channel the outer product of ``m_gdr dR_gdr + m_pion dR_pion``
        (photon axis) and ``dH`` (x axis), with the x-cuts of the reference.
        """
        from .kernel_build import SpecBuilder, cut_pairs

        m_p = C.PRINCE_UNITS.m_proton
        ecr, bcr, bph = cr_grid.grid, cr_grid.bins, ph_grid.bins
        dcr, dph = cr_grid.d, ph_grid.d
        step = np.log10(ecr[1] / ecr[0])
        if not (np.isclose(step, np.log10(bcr[1] / bcr[0])) and np.isclose(step, np.log10(bph[1] / bph[0]))):
            raise RuntimeError("cosmic-ray and photon grids must share the log step")
        y_edges = ecr[0] * bph[0] / m_p * 10 ** (np.arange(dcr + dph) * step)
        x_edges = bcr[0] / ecr[0] * 10 ** ((np.arange(2 * dcr) - (dcr - 1)) * step)
        sb = SpecBuilder(dcr, dph, m_p / ecr, cr_grid.widths)
        resp = {}

        def dR(mo):
            if mo not in resp:
                A, Z, _ = get_AZN(mo)
                gdr, pion = _sigma_components(A, Z)
                resp[mo] = (_response_increments(gdr, y_edges), _response_increments(pion, y_edges))
            return resp[mo]

        sref = spec_man.pdgid2sref
        for mo in spec_man.known_species:
            A, _, _ = get_AZN(mo)
            if A == 0:
                continue
            rg, rp = dR(mo)
            nonel = sb.response(rg + rp, key=("nonel", mo))
            lo_mo = sref[mo].lidx()
            if (mo, mo) not in self.diff:
                sb.bc(-1, nonel, lo_mo, lo_mo)
            for (m2, da), (wg, wp) in self.bc.items():
                if m2 != mo or da not in sref:
                    continue
                sb.bc(sb.response(wg * rg + wp * rp), -1, sref[da].lidx(), lo_mo)
            for (m2, da), (mg, mp_, a) in self.diff.items():
                if m2 != mo or da not in sref:
                    continue
                dH = np.diff(np.minimum(x_edges, 1.0) ** a)
                cut = self.x_cut_proton if da == 2212 else self.x_cut
                ki, kd = cut_pairs(bcr, ecr, cut)
                sb.diff(ki, kd, sref[da].lidx(), lo_mo, nonel=nonel if da == mo else -1,
                        sep=(mg * rg + mp_ * rp, dH))
        return sb.spec()

    def build_kernel(self, cr_grid, ph_grid, spec_man):
        """Assemble ``(batch_matrix, rows, cols)`` on the host from ``build_kernel_spec``."""
        spec = self.build_kernel_spec(cr_grid, ph_grid, spec_man)
        return spec.materialize(), spec.rows, spec.cols


def light_network_species():
    """p, n, 2H, 3H, 3He, 4He -- the light-nuclei run."""
    return [2212, 2112, 1000010020, 1000010030, 1000020030, 1000020040]


def full_network_species(max_mass=56, n_species=350, per_isobar=7):
    """p, n and the ``n_species - 2`` nuclides with A <= max_mass closest to stability.

    At the defaults this is 350 species, i.e. 33,600 states on a 96-bin grid.
    """
    chart = nuclide_chart(max_mass, per_isobar)

    def dist(pdg):
        A, Z, _ = get_AZN(pdg)
        return abs(Z - A / (1.98 + 0.0155 * A ** (2.0 / 3.0))) / max(A, 1) ** 0.5

    keep = sorted(chart, key=lambda p: (dist(p), p))[: max(n_species - 2, 0)]
    return [2212, 2112] + sorted(keep)


def em_cascade_matrices(em_grid, cr_grid, z):
    """Seeded-free synthetic EM-cascade transfer ``(T_gamma, T_electron, R_BH)`` at redshift z.

    Stand-ins with the shapes and conservation laws of the kinetic cascade
    transfer and the Bethe-Heitler pair shape (whose construction from cross
    sections is outside the ETD2 path):

    * photons below the pair-production threshold ``E_abs = 1.1e6 GeV/(1+z)``
      pass through; above it their energy is re-emitted below ``E_abs`` with
      a universal cascade spectrum (``E^-1.5`` under ``E_X = 0.04 E_abs``,
      ``E^-2`` above), energy conserving;
    * electrons and positrons hand their energy to photons: above ``E_abs``
      through the same cascade, below it as inverse-Compton photons at
      ``E_ic = (4/3)(E/m_e)^2 2.7 E_CMB (1+z)`` (capped at E);
    * ``R_BH[:, j]`` is the per-sign e+- spectrum of a nucleon at ``E_j`` (per
      nucleon): log-normal around ``4 (m_e/m_p) E_j`` with one decade width,
      normalised so the pair carries ``E_j``: ``2 sum_i E_i R_ij dE_i = E_j``.

    The state is dN/dE per bin, so energy in bin i is ``E_i n_i dE_i``.
    """
    U = C.PRINCE_UNITS
    E = em_grid.grid
    dE = em_grid.widths
    n_em = E.size
    e_abs = 1.1e6 / (1.0 + z)
    e_x = 0.04 * e_abs
    shape = np.where(E < e_x, (E / e_x) ** -1.5, (E / e_x) ** -2.0) * (E < e_abs)
    norm = np.sum(E * shape * dE)
    Tg = np.zeros((n_em, n_em))
    Te = np.zeros((n_em, n_em))
    e_ic_all = (4.0 / 3.0) * (E / U.m_electron) ** 2 * 2.7 * C.E_CMB * (1.0 + z)
    for j in range(n_em):
        if E[j] < e_abs or norm <= 0:
            Tg[j, j] = 1.0
        else:
            Tg[:, j] = shape * (E[j] * dE[j]) / norm
        if E[j] >= e_abs and norm > 0:
            Te[:, j] = shape * (E[j] * dE[j]) / norm
        else:
            e_ic = min(e_ic_all[j], E[j])
            i = int(np.clip(np.searchsorted(em_grid.bins, e_ic) - 1, 0, n_em - 1))
            Te[i, j] = E[j] * dE[j] / (E[i] * dE[i])
    Ep = cr_grid.grid
    R = np.zeros((n_em, Ep.size))
    for j in range(Ep.size):
        e0 = 4.0 * (U.m_electron / U.m_proton) * Ep[j]
        g = np.exp(-0.5 * (np.log10(E / e0) / 0.5) ** 2)
        s = 2.0 * np.sum(E * g * dE)
        if s > 0:
            R[:, j] = g * Ep[j] / s
    return Tg, Te, R
