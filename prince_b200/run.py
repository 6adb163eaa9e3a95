"""``PriNCeRun``: the run object the propagation solvers consume.

It holds the grids, the species table, the photon field, the continuous
loss-rate objects and the photo-nuclear rate kernel -- the inputs the
reference's ETD2 path reads from its own ``PriNCeRun``
(``src/prince_cr/core.py:12-264``).  Attribute names follow the reference
(``cr_grid``, ``ph_grid``, ``spec_man``, ``dim_states``, ``int_rates``,
``adia_loss_rates_grid``, ``pair_loss_rates_grid``, ``backend``), so the
solvers also accept a reference run object that was built with FP64 kernel
settings.

The rate kernel comes from a *cross-section model* object with
``known_species`` and either ``build_kernel_spec(cr_grid, ph_grid, spec_man)``
returning a ``prince_b200.kernel_build.KernelSpec`` (per-channel response
samples; the GPU expands it, the host only when the oracle asks) or
``build_kernel(...)`` returning ``(batch_matrix, rows, cols)``: one kernel row
per coupling-matrix entry (daughter state ``rows[i]``, mother state
``cols[i]``), ``dph`` photon-bin columns.  Sampling response functions from
tabulated cross sections is outside the ETD2 path; ``prince_b200.synth``
provides seeded synthetic models and ``FixedKernelModel`` wraps a precomputed
kernel.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import constants as C
from .data import EnergyGrid, SpeciesManager, get_AZN, is_nucleus
from .operators import coupling_structure


class FixedKernelModel:
    """A precomputed fold kernel: ``batch_matrix`` (R x dph) with its coupling pairs."""

    def __init__(self, known_species, batch_matrix, rows, cols, lifetimes=None):
        self.known_species = [int(s) for s in known_species]
        self.batch_matrix = np.ascontiguousarray(batch_matrix, dtype=np.float64)
        self.rows = np.asarray(rows, dtype=np.int64)
        self.cols = np.asarray(cols, dtype=np.int64)
        self.lifetimes = dict(lifetimes or {})

    def build_kernel(self, cr_grid, ph_grid, spec_man):
        if self.batch_matrix.shape[1] != ph_grid.d:
            raise ValueError("kernel photon axis does not match the photon grid")
        return self.batch_matrix, self.rows, self.cols


class PhotoNuclearInteractionRate:
    """Fold kernel in CSR order plus the fixed coupling pattern.

    ``_batch_matrix[i]`` is the kernel row of coupling entry ``i`` in CSR
    order, so ``_batch_matrix @ photon_vector(z)`` is the coupling matrix's
    ``data`` at redshift ``z`` (``interaction_rates.py:966-1067``).

    Built from a kernel (``batch_matrix``) or from a ``kernel_spec``
    (``prince_b200.kernel_build.KernelSpec``).  With a spec the host kernel is
    expanded only when ``_batch_matrix`` is first read (the CPU oracle); the
    device builds its own copy from the spec.
    """

    def __init__(self, prince_run, batch_matrix, rows, cols, kernel_spec=None):
        self.prince_run = prince_run
        self.spec_man = prince_run.spec_man
        self.e_photon = prince_run.ph_grid
        self.e_cosmicray = prince_run.cr_grid
        n = prince_run.dim_states
        indptr, indices, order = coupling_structure(rows, cols, n)
        self._batch_rows = np.asarray(rows, dtype=np.int64)[order]
        self._batch_cols = np.asarray(cols, dtype=np.int64)[order]
        self.kernel_spec = kernel_spec
        self._bm = None if batch_matrix is None else np.ascontiguousarray(batch_matrix[order], dtype=np.float64)
        self.sortidx = order
        self.coupling_mat = sp.csr_matrix(
            (np.zeros(indices.size), indices, indptr), shape=(n, n)
        )

    @property
    def _batch_matrix(self):
        if self._bm is None:
            self._bm = np.ascontiguousarray(self.kernel_spec.materialize()[self.sortidx])
        return self._bm

    @property
    def photon_field(self):
        return self.prince_run.photon_field

    def photon_vector(self, z, pfield=None):
        pf = pfield if pfield is not None else self.photon_field
        return pf.get_photon_density(self.e_photon.grid, z)

    def get_hadr_jacobian(self, z, scale_fac=1.0, force_update=False, pfield=None):
        """The coupling matrix at redshift z on the host: its values are the fold
        ``_batch_matrix @ photon_vector(z)`` (times ``scale_fac``), the contract of
        ``interaction_rates.py:966-1120``.  The B200 solvers never call it; it lets
        the reference's own CPU solver run on this run object."""
        vec = np.dot(self._batch_matrix, self.photon_vector(z, pfield=pfield))
        if scale_fac != 1.0:
            vec = scale_fac * vec
        self.coupling_mat.data[:] = vec
        return self.coupling_mat

    def build_split_fold(self, off_to_M, diag_to_M):
        """Row-subset kernels of the off-diagonal values and the diagonal
        (the contract of ``interaction_rates.py:780-822``), rebuilt whenever the
        maps change (the reference keeps the first solve's, which a later solve
        from another first window would misread)."""
        key = (np.asarray(off_to_M).tobytes(), np.asarray(diag_to_M).tobytes())
        if getattr(self, "_sf_key", None) != key:
            bm = self._batch_matrix
            present = np.asarray(diag_to_M) >= 0
            self._sf_off_kernel = bm[np.asarray(off_to_M, dtype=np.int64)]
            self._sf_diag_present = present
            self._sf_diag_kernel = bm[np.asarray(diag_to_M, dtype=np.int64)[present]]
            self._sf_key = key
        self._split_fold_ready = True

    def fold_split(self, z, moff_data_out, dmg_out):
        """Fold straight into ``M_off.data`` and the diagonal (``interaction_rates.py:824-847``)."""
        ph = np.asarray(self.photon_vector(z), dtype=np.float64)
        if moff_data_out.size:
            np.copyto(moff_data_out, self._sf_off_kernel.dot(ph))
        dmg_out.fill(0.0)
        if self._sf_diag_kernel.shape[0]:
            dmg_out[self._sf_diag_present] = self._sf_diag_kernel.dot(ph)


class _ContinuousLossBase:
    def __init__(self, prince_run, energy="grid"):
        if energy not in ("grid", "bins"):
            raise ValueError(
                "Unexpected energy keyword ({}), use either 'grid' or 'bins'".format(energy)
            )
        self.spec_man = prince_run.spec_man
        self.e_cosmicray = prince_run.cr_grid
        self.energy = energy
        self._grids = getattr(prince_run, "grids", {"default": prince_run.cr_grid})
        if energy == "grid":
            self._dim = prince_run.dim_states
            self._earr = prince_run.cr_grid.grid
            self._lo = lambda s: s.lidx()
            self._hi = lambda s: s.uidx()
        else:
            self._dim = prince_run.dim_bins
            self._earr = prince_run.cr_grid.bins
            self._lo = lambda s: s.lbin()
            self._hi = lambda s: s.ubin()

    def _species_earr(self, s):
        """Energies of species ``s`` on its home grid (``interaction_rates.py:1159-1165``)."""
        g = self._grids.get(s.grid_tag, self.e_cosmicray)
        return g.grid if self.energy == "grid" else g.bins


class ContinuousAdiabaticLossRate(_ContinuousLossBase):
    """Adiabatic (redshift) loss ``kappa_adia(z) = H(z) cm2sec E`` per state.

    Same definition as ``interaction_rates.py:1194-1224``.
    """

    def __init__(self, prince_run, energy="grid"):
        super().__init__(prince_run, energy)
        self.energy_vector = np.zeros(self._dim)
        for s in self.spec_man.species_refs:
            self.energy_vector[self._lo(s):self._hi(s)] = self._species_earr(s)

    def loss_vector(self, z, energy=None):
        from .cosmology import H

        e = self.energy_vector if energy is None else energy
        return H(z) * C.PRINCE_UNITS.cm2sec * e


def bethe_heitler_phi(xi):
    """Blumenthal (1970) pair-production function phi(xi) with the Chodorowski fit.

    Low branch (xi < 25): ``pi/12 (xi-2)^4 / sum_k c_k (xi-2)^k``; high
    branch: ``xi P(ln xi) / (1 - f1/xi - f2/xi^2 - f3/xi^3)`` with the cubic
    ``P`` in Horner form.  The fit constants are those of
    ``interaction_rates.py:1346-1386``.
    """
    xi = np.asarray(xi, dtype=np.float64)
    c1, c2, c3, c4 = 0.8048, 0.1459, 1.137e-3, -3.879e-6
    f1, f2, f3 = 2.91, 78.35, 1837
    res = np.zeros(xi.shape)
    lo = xi < 25.0
    hi = ~lo
    u = xi[lo] - 2
    res[lo] = np.pi / 12.0 * u ** 4 / (c1 * u ** 1 + c2 * u ** 2 + c3 * u ** 3 + c4 * u ** 4)
    x = xi[hi]
    L = np.log(x)
    poly = np.zeros_like(L)
    for coef in (2.667, -14.45, 50.95, -86.07):
        poly = poly * L + coef
    res[hi] = x * poly / (1 - f1 * x ** -1 - f2 * x ** -2 - f3 * x ** -3)
    return res


class ContinuousPairProductionLossRate(_ContinuousLossBase):
    """Bethe-Heitler pair-production loss ``kappa_pair(z)`` per state.

    ``kappa_pair = scale_vec * rate(z)`` on nucleus blocks, with
    ``rate_i = trapz_xi( n_gamma(m_e xi / (2 gamma_i), z) phi(xi)/xi^2 )``,
    ``gamma_i = E_i/m_p``, 400 log-spaced xi from 2+1e-8 to 1e16 and
    ``scale_vec = alpha r_e^2 m_e^2 Z^2 / A`` (``interaction_rates.py:1238-1332``).
    """

    def __init__(self, prince_run, energy="grid", xi_steps=400):
        super().__init__(prince_run, energy)
        self.prince_run = prince_run
        self.xi = np.logspace(np.log10(2 + 1e-8), 16.0, xi_steps)
        self.phi_xi2 = bethe_heitler_phi(self.xi) / (self.xi ** 2)
        U = C.PRINCE_UNITS
        units = U.fine_structure * U.r_electron ** 2 * U.m_electron ** 2
        self.scale_vec = np.zeros(self._dim)
        for s in self.spec_man.species_refs:
            if not s.is_nucleus:
                continue
            self.scale_vec[self._lo(s):self._hi(s)] = (
                units * abs(s.charge) ** 2 / float(s.A) * np.ones_like(self._earr, dtype="double")
            )
        gamma = self._earr / U.m_proton
        self.photon_grid = np.outer(1 / gamma, self.xi) * U.m_electron / 2.0

    @property
    def photon_field(self):
        return self.prince_run.photon_field

    def loss_vector(self, z, pfield=None):
        from scipy.integrate import trapezoid

        pf = pfield if pfield is not None else self.photon_field
        dens = pf.get_photon_density(self.photon_grid.reshape(-1), z).reshape(self.photon_grid.shape)
        rate_single = trapezoid(dens * self.phi_xi2, self.xi, axis=1)
        rate_full = np.zeros(self._dim)
        for s in self.spec_man.species_refs:
            if s.is_nucleus:
                rate_full[self._lo(s):self._hi(s)] = rate_single
        return self.scale_vec * rate_full


def default_em_grid(cosmic_ray_grid, bins_dec=16):
    """The reference's decoupled EM grid (``core.py:105-129``): log10 m_e snapped
    up to the step 1/bins_dec below the cosmic-ray grid's top."""
    import math

    top = float(cosmic_ray_grid[1])
    m_e_log10 = float(np.log10(C.PRINCE_UNITS.m_electron))
    steps = math.floor((top - m_e_log10) * bins_dec)
    return (top - steps / bins_dec, top, bins_dec)


class PriNCeRun:
    """Grids, species, photon field, loss rates and the fold kernel of one run.

    Args:
        cross_sections: a model with ``known_species`` and ``build_kernel``.
        photon_field: a ``prince_b200.photonfields`` field.
        cosmic_ray_grid / photon_grid: ``(log10 lo, log10 hi, bins per decade)``;
            both grids must share the log step (the kernel construction contract).
        max_mass: keep species with ``A <= max_mass``.
        backend: a ``constants.BackendConfig`` (default backend ``"b200"``).
        enable_em_cascade: co-evolve gamma and e+- with the nuclei (the
            reference run's flag of the same name; gamma, e- and e+ join the
            species).  The EM species share the cosmic-ray grid unless
            ``enable_em_decoupled_grid``.
        enable_em_decoupled_grid: home gamma and e+- on their own EM grid
            (``core.py:44-56, 105-137, 206-214``): blocks of ``em_grid.d``
            states while the nuclei keep the cosmic-ray grid.
        em_grid: ``(log10 lo, log10 hi, bins per decade)`` of that grid; by
            default the reference's: from the electron mass (snapped to the
            step, rounded up) to the top of the cosmic-ray grid at 16 bins per
            decade.
        em_cascade_model: ``callable(z) -> (T_gamma, T_electron, R_BH)``, the
            per-redshift cascade transfer (on the EM species' grid) and the
            Bethe-Heitler pair shape (EM grid x cosmic-ray grid), read by the
            solvers' ``_em_transfer_at`` / ``_em_bh_at``.
    """

    def __init__(self, cross_sections, photon_field, cosmic_ray_grid=(3, 14, 8),
                 photon_grid=(-15, -6, 8), max_mass=np.inf, backend=None, species_list=None,
                 enable_em_cascade=False, em_cascade_model=None, enable_em_decoupled_grid=False,
                 em_grid=None):
        self.backend = backend if backend is not None else C.BackendConfig()
        self.cross_sections = cross_sections
        self.photon_field = photon_field
        self.cr_grid = EnergyGrid(*cosmic_ray_grid)
        self.ph_grid = EnergyGrid(*photon_grid)
        self.grids = {"default": self.cr_grid}
        if species_list is not None:
            species = sorted(set(species_list) & set(cross_sections.known_species))
        else:
            species = [s for s in cross_sections.known_species
                       if not is_nucleus(s) or get_AZN(s)[0] <= max_mass]
        self.enable_em_cascade = bool(enable_em_cascade)
        self.enable_em_decoupled_grid = bool(enable_em_decoupled_grid) and self.enable_em_cascade
        self.em_grid = None
        if self.enable_em_cascade:
            species = list(species) + [p for p in (22, 11, -11) if p not in species]
        lifetimes = getattr(cross_sections, "lifetimes", None)
        self.spec_man = SpeciesManager(species, self.cr_grid.d, lifetimes=lifetimes)
        if self.enable_em_decoupled_grid:
            self.em_grid = EnergyGrid(*(em_grid if em_grid is not None else default_em_grid(cosmic_ray_grid)))
            self.grids["em"] = self.em_grid
            self.spec_man.add_grid("em", self.em_grid.d)
            for p in (22, 11, -11):
                self.spec_man.set_grid_tag(p, "em")
        self.dim_states = self.spec_man.dim_states
        self.dim_bins = self.spec_man.dim_bins
        self.adia_loss_rates_grid = ContinuousAdiabaticLossRate(self, "grid")
        self.pair_loss_rates_grid = ContinuousPairProductionLossRate(self, "grid")
        self.adia_loss_rates_bins = ContinuousAdiabaticLossRate(self, "bins")
        self.pair_loss_rates_bins = ContinuousPairProductionLossRate(self, "bins")
        if hasattr(cross_sections, "build_kernel_spec"):
            spec = cross_sections.build_kernel_spec(self.cr_grid, self.ph_grid, self.spec_man)
            self.int_rates = PhotoNuclearInteractionRate(self, None, spec.rows, spec.cols, kernel_spec=spec)
        else:
            bm, rows, cols = cross_sections.build_kernel(self.cr_grid, self.ph_grid, self.spec_man)
            self.int_rates = PhotoNuclearInteractionRate(self, bm, rows, cols)
        self.em_int_rates = None
        self.em_cascade_model = em_cascade_model
        self.spec_man.add_grid("ph", self.ph_grid.d)

    def set_photon_field(self, pfield):
        self.photon_field = pfield
