"""Propagation results: per-species spectra and group sums on a common grid.

``UHECRPropagationResult`` keeps the reference's result API
(``src/prince_cr/solvers/propagation.py:34-192``: ``state``, ``egrid``,
``spec_man``, ``get_solution``, ``get_solution_scale``,
``get_solution_group``, ``get_lnA``, ``get_energy_density``, ``+``, ``*``,
``to_dict`` / ``from_dict``) on its own implementation: every group
quantity goes through one batched projector, :class:`GroupProjector`, which
works on a ``(n, K)`` block of states at once and on torch tensors on the
GPU as well as on numpy arrays.

The projection is the reference's all-particle construction
(``propagation.py:103-167``): species ``s`` with mass number ``A`` has total
energies ``A E_i`` and spectrum ``(A E_i)^epow n_i / A``; its positive bins
are interpolated linearly in (ln E, ln spectrum) onto a common total-energy
grid, points outside the span of the positive bins contribute zero, and the
species are summed.  The default common grid spans the cosmic-ray grid's
edges shifted by ``log10 A_max`` at four times its bins per decade
(``propagation.py:107-111``).
"""

from __future__ import annotations

import numpy as np

from .data import EnergyGrid, is_nucleus

_NEUTRINOS = (12, -12, 14, -14, 16, -16)
_TINY = np.finfo(np.float64).tiny


def grid_triple(grid):
    """``(log10 lower edge, log10 upper edge, bins per decade)`` of a cosmic-ray grid.

    ``grid`` is an :class:`EnergyGrid` (its own triple), another grid object
    with bin centres in ``grid.grid`` (the reference's), or an array of bin
    centres; the triple of a log-spaced grid is recovered from its centres.
    """
    if isinstance(grid, EnergyGrid):
        return grid.lower, grid.upper, grid.bins_dec
    c = np.asarray(getattr(grid, "grid", grid), dtype=np.float64)
    r = c[1] / c[0]
    lo = 2.0 * c[0] / (1.0 + r)
    hi = lo * r ** c.size
    return (float(np.round(np.log10(lo), 9)), float(np.round(np.log10(hi), 9)),
            float(np.round(1.0 / np.log10(r), 9)))


def common_energy_grid(grid, max_mass):
    """Total-energy grid shared by all species of a group (``propagation.py:107-111``)."""
    lo, hi, bpd = grid_triple(grid)
    return EnergyGrid(lo, hi + np.log10(max_mass), 4 * bpd).grid


def select_species(spec_man, which):
    """PDG ids of a group: a list, ``"CR"`` (nuclei), ``"nu"`` (neutrinos),
    ``"all"``, or ``(key, lo, hi)`` selecting ``lo <= key(pdg) <= hi``
    (``propagation.py:114-129``)."""
    known = list(spec_man.known_species)
    if isinstance(which, list):
        return which
    if isinstance(which, tuple):
        key, lo, hi = which
        return [p for p in known if lo <= key(p) <= hi]
    if which == "CR":
        return [p for p in known if is_nucleus(p)]
    if which == "nu":
        return [p for p in known if p in _NEUTRINOS]
    if which == "all":
        return known
    raise ValueError(f"unknown species group {which!r}")


class GroupProjector:
    """Batched log-log projection of species spectra onto one common grid.

    Built once per (species list, energy grid, common grid); ``__call__``
    maps a state block ``(n, K)`` (or ``(n,)``) to per-species spectra on the
    common grid ``(n_species, G, K)``.  Interpolation runs between the
    nearest positive bins on either side of each common-grid point, found
    for all columns at once by forward and backward fills of the indices of
    positive bins; it is differentiable in torch through the two bins it
    reads.
    """

    def __init__(self, spec_man, egrid, species, com_egrid):
        self.refs = [spec_man.pdgid2sref[p] for p in species]
        self.egrid = np.asarray(egrid, dtype=np.float64)
        self.com = np.asarray(com_egrid, dtype=np.float64)
        d = self.egrid.size
        self.d = d
        lx = np.log(self.com)
        self.A = np.array([float(s.A) for s in self.refs])
        # per species: total energies, their logs, and the bracket of each
        # common-grid point among them (j with le[j] <= x < le[j+1], -1 below)
        self.etot = self.A[:, None] * self.egrid[None, :]
        self.le = np.log(self.etot)
        self.lx = lx
        self.j = np.stack([np.searchsorted(le, lx, side="right") - 1 for le in self.le])
        self.at_node = np.take_along_axis(self.le, np.clip(self.j, 0, d - 1), axis=1) == lx[None, :]
        self.rows = np.stack([np.arange(s.lidx(), s.uidx()) for s in self.refs]) if self.refs else \
            np.zeros((0, d), dtype=np.int64)

    def spectra(self, X, epow):
        """Per-species ``(A E)^epow n / A`` on the species' own total-energy grid:
        ``(n_species, d, K)``."""
        import torch

        X, back = _as_torch(X)
        X2 = X[:, None] if X.dim() == 1 else X
        rows = torch.as_tensor(self.rows, device=X2.device)
        Y = X2[rows]                                            # (S, d, K)
        scale = torch.as_tensor(self.etot ** epow, dtype=X2.dtype, device=X2.device)
        A = torch.as_tensor(self.A, dtype=X2.dtype, device=X2.device)
        return scale[:, :, None] * Y / A[:, None, None], back, X.dim() == 1

    def __call__(self, X, epow=0):
        """Per-species spectra on the common grid, ``(n_species, G, K)`` (K dropped for 1-D input)."""
        import torch

        spec, back, flat = self.spectra(X, epow)
        S, d, K = spec.shape
        dev, dt = spec.device, spec.dtype
        if S == 0:
            out = torch.zeros((0, self.lx.size, K), dtype=dt, device=dev)
            return back(out[..., 0] if flat else out)
        pos = spec > 0
        idx = torch.arange(d, device=dev)[None, :, None].expand(S, d, K)
        # nearest positive bin at or below / at or above every bin
        below = torch.where(pos, idx, torch.full_like(idx, -1)).cummax(dim=1).values
        above = torch.where(pos, idx, torch.full_like(idx, d)).flip(1).cummin(dim=1).values.flip(1)
        # log of the positive bins; subnormal values enter at the smallest normal
        # double, so that the derivative 1/spec stays finite
        ls = torch.log(torch.where(pos, spec.clamp(min=_TINY), torch.ones_like(spec)))
        le = torch.as_tensor(self.le, dtype=dt, device=dev)
        lx = torch.as_tensor(self.lx, dtype=dt, device=dev)
        j = torch.as_tensor(self.j, device=dev)                                  # (S, G)
        jl = j.clamp(0, d - 1)[:, :, None].expand(S, j.shape[1], K)
        jr = (j + 1).clamp(0, d - 1)[:, :, None].expand(S, j.shape[1], K)
        L = torch.gather(below, 1, jl)
        L = torch.where((j >= 0)[:, :, None], L, torch.full_like(L, -1))
        R = torch.gather(above, 1, jr)
        R = torch.where((j + 1 <= d - 1)[:, :, None], R, torch.full_like(R, d))
        # a point that falls on a positive bin takes that bin's value
        on = torch.as_tensor(self.at_node, device=dev)[:, :, None] & (L == jl)
        inside = (L >= 0) & ((R < d) | on)
        Lc, Rc = L.clamp(0, d - 1), R.clamp(0, d - 1)
        lsL, lsR = torch.gather(ls, 1, Lc), torch.gather(ls, 1, Rc)
        leS = le[:, :, None].expand(S, d, K)
        leL, leR = torch.gather(leS, 1, Lc), torch.gather(leS, 1, Rc)
        span = torch.where(Rc > Lc, leR - leL, torch.ones_like(leL))
        slope = (lsR - lsL) / span
        val = slope * (lx[None, :, None] - leL) + lsL
        val = torch.where(on, lsL, val)
        # points outside the span are zero; their log value is masked before
        # exp so that no overflow there reaches the derivative
        val = torch.where(inside, val, torch.zeros_like(val))
        out = torch.where(inside, torch.exp(val), torch.zeros_like(val))
        return back(out[..., 0] if flat else out)


def _as_torch(X):
    """``(tensor, convert back)``: numpy arrays go through CPU tensors and come back as numpy."""
    import torch

    if isinstance(X, torch.Tensor):
        return X, lambda t: t
    t = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64))
    return t, lambda r: r.detach().cpu().numpy()


class UHECRPropagationResult:
    """Final state of a propagation (``(n,)`` or ``(n, K)``) with its grid and species."""

    def __init__(self, state, egrid, spec_man, grid=None, grids=None):
        self.spec_man = spec_man
        self.egrid = egrid
        self.state = state
        # the grid's (lower, upper, bins/decade); recovered from the centres when not given
        self._grid = grid if grid is not None else egrid
        # energies of the other home grids by tag (gamma and e+- on a decoupled EM grid)
        self._grids = dict(grids or {})
        self._projectors = {}

    def _energies(self, s):
        """Energies of species ``s``: its home grid's (the shared grid's by default)."""
        if s.grid_tag == "default":
            return self.egrid
        return self._grids[s.grid_tag]

    # -- container protocol ------------------------------------------------
    def to_dict(self):
        return {"egrid": self.egrid, "state": self.state, "known_spec": self.known_species}

    @classmethod
    def from_dict(cls, dic):
        from .data import SpeciesManager

        egrid = dic["egrid"]
        return cls(dic["state"], egrid, SpeciesManager(dic["known_spec"], np.size(egrid)))

    @property
    def known_species(self):
        return self.spec_man.known_species

    def _compatible(self, other):
        if not np.array_equal(self.egrid, other.egrid):
            raise ValueError("results live on different energy grids and cannot be added")
        if not np.array_equal(self.known_species, other.known_species):
            raise ValueError("results carry different species tables and cannot be added")

    def __add__(self, other):
        self._compatible(other)
        return UHECRPropagationResult(self.state + other.state, self.egrid, self.spec_man, self._grid, self._grids)

    def __mul__(self, number):
        if not np.isscalar(number):
            raise TypeError(f"a result scales by a scalar only, not by {type(number).__name__}")
        return UHECRPropagationResult(self.state * number, self.egrid, self.spec_man, self._grid, self._grids)

    # -- single species ------------------------------------------------------
    def get_solution(self, pdg_id):
        """``(egrid, n)``: the species' spectrum per energy per nucleon."""
        s = self.spec_man.pdgid2sref[pdg_id]
        return self._energies(s), self.state[s.sl]

    def get_solution_scale(self, pdg_id, epow=0):
        """``(A E, (A E)^epow n / A)``: the spectrum in total energy."""
        s = self.spec_man.pdgid2sref[pdg_id]
        etot = s.A * np.asarray(self._energies(s))
        y = self.state[s.sl]
        scale = etot ** epow
        return etot, (scale[:, None] if np.ndim(y) == 2 else scale) * y / s.A

    # -- groups ----------------------------------------------------------------
    def _projector(self, pdg_ids, egrid):
        species = select_species(self.spec_man, pdg_ids)
        off = [p for p in species if self.spec_man.pdgid2sref[p].grid_tag != "default"]
        if off:
            raise ValueError(f"species {off} live on another grid; group projections take the shared grid's species")
        if egrid is None:
            amax = max(s.A for s in self.spec_man.species_refs)
            com = common_energy_grid(self._grid, amax)
        else:
            com = np.asarray(egrid, dtype=np.float64)
        key = (tuple(species), com.size, float(com[0]), float(com[-1]))
        if key not in self._projectors:
            self._projectors[key] = GroupProjector(self.spec_man, self.egrid, species, com)
        return self._projectors[key]

    def get_solution_group(self, pdg_ids, epow=3, egrid=None):
        """``(common grid, summed spectrum)`` of a group of species in total energy."""
        pr = self._projector(pdg_ids, egrid)
        return pr.com, pr(self.state, epow).sum(axis=0)

    def get_lnA(self, pdg_ids, egrid=None):
        """``(common grid, <ln A>, Var ln A)`` weighted by the group's spectra."""
        pr = self._projector(pdg_ids, egrid)
        spec = pr(self.state, 0)
        lnA = np.log(pr.A).reshape((-1,) + (1,) * (spec.ndim - 1))
        total = spec.sum(axis=0)
        with np.errstate(invalid="ignore", divide="ignore"):
            mean = (lnA * spec).sum(axis=0) / total
            var = (lnA ** 2 * spec).sum(axis=0) / total - mean ** 2
        return pr.com, mean, var

    def get_energy_density(self, pdg_id):
        """``int A E n dE`` of one species (trapezoidal rule on the bin centres)."""
        from scipy.integrate import trapezoid

        s = self.spec_man.pdgid2sref[pdg_id]
        E = np.asarray(self.egrid)
        y = self.state[s.sl]
        w = s.A * E
        return trapezoid((w[:, None] if np.ndim(y) == 2 else w) * y, E, axis=0)
