"""Energy grids, PDG helpers and the species layout of the state vector.

The state vector is species-major: species are ordered by PDG id and each
species owns one contiguous block of energy bins on its home grid (``d`` bins
of the cosmic-ray grid, or of a separate EM grid for gamma and e+- when the
EM sector is decoupled).  This is the layout contract of the reference
(``src/prince_cr/data.py:1385-1446`` for the ordering, ``data.py:1256-1310``
for the per-species slices, ``data.py:1664-1711`` for the home grids and the
transport offsets); the CSR structure and every per-state vector in this
package index into it.
"""

from __future__ import annotations

import numpy as np

_PDG_PROTON = 2212
_PDG_NEUTRON = 2112
_NUCLEUS_PREFIX = 1_000_000_000

#: Charges of the non-nuclear species the ETD2 path may carry.
_LIGHT_CHARGE = {22: 0, 11: -1, -11: 1, 12: 0, -12: 0, 14: 0, -14: 0, 16: 0, -16: 0}


def make_nucleus_pdg(A: int, Z: int) -> int:
    """PDG id of a ground-state nucleus (``1000000000 + Z*10000 + A*10``).

    Free nucleons keep their hadron codes (2212, 2112), as in
    ``src/prince_cr/util.py:282-295``.
    """
    if A == 1 and Z == 1:
        return _PDG_PROTON
    if A == 1 and Z == 0:
        return _PDG_NEUTRON
    return _NUCLEUS_PREFIX + Z * 10000 + A * 10


def is_nucleus(pdg_id: int) -> bool:
    """True for free p/n and for ``10LZZZAAAI`` nuclei (``util.py:264-279``)."""
    pdg_id = int(pdg_id)
    if pdg_id in (_PDG_PROTON, _PDG_NEUTRON):
        return True
    if pdg_id // _NUCLEUS_PREFIX != 1:
        return False
    rest = pdg_id - _NUCLEUS_PREFIX
    Z = (rest // 10000) % 1000
    A = (rest // 10) % 1000
    return Z <= A and A >= 1


def get_AZN(pdg_id: int):
    """``(A, Z, N)`` of a nucleus, ``(0, 0, 0)`` otherwise (``util.py:297-316``)."""
    pdg_id = int(pdg_id)
    if pdg_id == _PDG_PROTON:
        return 1, 1, 0
    if pdg_id == _PDG_NEUTRON:
        return 1, 0, 1
    if pdg_id // _NUCLEUS_PREFIX != 1:
        return 0, 0, 0
    rest = pdg_id - _NUCLEUS_PREFIX
    Z = (rest // 10000) % 1000
    A = (rest // 10) % 1000
    return A, Z, A - Z


def is_decoupled(spec_man):
    """True when some species of a species manager (this package's or the
    reference's) live on a home grid other than the default one."""
    return any(getattr(s, "grid_tag", "default") != "default" for s in spec_man.species_refs)


class EnergyGrid:
    """Log-spaced bins: ``bins`` (edges), ``grid`` (centres), ``widths``, ``d``.

    ``lower``/``upper`` are log10 of the outer edges and ``bins_dec`` the bins
    per decade.  The edge count is ``int((upper - lower) * bins_dec + 1)``,
    exactly as ``src/prince_cr/data.py:1080-1083``, so grids built from the
    same triple are bit-identical to the reference's.
    """

    def __init__(self, lower, upper, bins_dec):
        self.lower, self.upper, self.bins_dec = lower, upper, bins_dec
        self.bins = np.logspace(lower, upper, int((upper - lower) * bins_dec + 1))
        self.grid = 0.5 * (self.bins[1:] + self.bins[:-1])
        self.widths = self.bins[1:] - self.bins[:-1]
        self.d = self.grid.size


class PrinceSpecies:
    """One species block of the state vector.

    Carries the attributes the ETD2 path reads from the reference's
    ``PrinceSpecies`` (``data.py:1130-1330``): ``pdgid``, ``princeidx``,
    ``A``/``Z``/``N``, ``charge``, ``is_nucleus``, ``lifetime`` and the
    slice helpers ``sl``/``lidx``/``uidx``/``lbin``/``ubin``.
    """

    def __init__(self, pdgid, princeidx, d, lifetime=np.inf):
        self.pdgid = int(pdgid)
        self.princeidx = int(princeidx)
        self.grid_tag = "default"
        self._d = int(d)
        # transport block: offset and size in the state vector, offset in the bin-edge vector
        self._tr_lidx = self.princeidx * self._d
        self._tr_dim = self._d
        self._tr_lbin = self.princeidx * (self._d + 1)
        self.is_nucleus = is_nucleus(self.pdgid)
        if self.is_nucleus:
            self.A, self.Z, self.N = get_AZN(self.pdgid)
            self.charge = self.Z
        else:
            self.A, self.Z, self.N = 1, None, None
            self.charge = _LIGHT_CHARGE.get(self.pdgid, 0)
        self.is_charged = self.charge != 0
        self.lifetime = float(lifetime)
        self.is_stable = not np.isfinite(self.lifetime)
        self.sname = f"nucleus_{self.pdgid}" if self.is_nucleus else f"pdg_{self.pdgid}"

    @property
    def sl(self):
        return slice(self.lidx(), self.uidx())

    def lidx(self):
        return self._tr_lidx

    def uidx(self):
        return self._tr_lidx + self._tr_dim

    def lbin(self):
        return self._tr_lbin

    def ubin(self):
        return self._tr_lbin + self._tr_dim + 1

    def __repr__(self):
        return f"PrinceSpecies({self.pdgid}, idx={self.princeidx})"


class SpeciesManager:
    """Species table: PDG ids sorted ascending define ``princeidx``.

    ``lifetimes`` optionally maps PDG id to a rest-frame lifetime in seconds
    (used by the explicit-decay operator).
    """

    def __init__(self, pdgid_list, ed, lifetimes=None):
        lifetimes = lifetimes or {}
        self.grid_dims = {"default": int(ed)}
        ids = sorted(set(int(p) for p in pdgid_list))
        self.species_refs = [
            PrinceSpecies(p, i, ed, lifetimes.get(p, np.inf)) for i, p in enumerate(ids)
        ]
        self.known_species = [s.pdgid for s in self.species_refs]
        self.nspec = len(self.species_refs)
        self.pdgid2sref = {s.pdgid: s for s in self.species_refs}
        self.pdgid2princeidx = {s.pdgid: s.princeidx for s in self.species_refs}
        self.princeidx2sref = {s.princeidx: s for s in self.species_refs}
        self.princeidx2pdgid = {s.princeidx: s.pdgid for s in self.species_refs}
        self.dim_states = self.nspec * int(ed)
        self.dim_bins = self.nspec * (int(ed) + 1)

    def add_grid(self, tag, d):
        """Register a home grid of ``d`` bins (moves no species onto it)."""
        self.grid_dims[tag] = int(d)

    def set_grid_tag(self, pdgid, tag):
        """Home species ``pdgid`` on the registered grid ``tag`` and recompute the offsets."""
        if tag not in self.grid_dims:
            raise KeyError(f"grid {tag!r} is not registered; call add_grid first")
        self.pdgid2sref[int(pdgid)].grid_tag = tag
        self.compute_transport_offsets()

    def compute_transport_offsets(self):
        """Blocks of ``grid_dims[s.grid_tag]`` states in ``princeidx`` order
        (``data.py:1677-1700``); sets ``dim_states`` and ``dim_bins``."""
        off = offb = 0
        for s in sorted(self.species_refs, key=lambda x: x.princeidx):
            d = self.grid_dims[s.grid_tag]
            s._tr_lidx, s._tr_dim, s._tr_lbin = off, d, offb
            off += d
            offb += d + 1
        self.dim_states = off
        self.dim_bins = offb

    @property
    def decoupled(self):
        """True when some species live on a grid other than the default one."""
        return is_decoupled(self)
