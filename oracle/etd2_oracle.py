"""CPU oracle of the ETD2 propagation path -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy/scipy, the reference CPU backend of the ETD2
solver (``ETD2SolverCPU`` and ``_MultiRHSETD2SolverCPU`` of PriNCe).  It is
the checker for the CUDA path: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / reference arm of ``bench.py`` may import it.  The
product path (``prince_b200``) never calls it.

Parity of this restatement is pinned against golden vectors produced by the
reference itself (``tests/golden/make_golden.py`` runs PriNCe's own
``ETD2SolverCPU`` / ``MultiRHSPropagationSolverETD2`` on synthetic
cross sections and stores inputs and outputs under ``tests/golden/``).

Reference files restated here (paths inside the PriNCe project):

* ``src/prince_cr/solvers/propagation.py:813-832`` -- z grid of ``solve``;
* ``propagation.py:1017-1120`` -- per-window refresh (fold, diag/off split,
  in-place value refresh, pair-loss cache);
* ``propagation.py:1360-1429`` -- per-step operator (dl/dz, kappa, b, d);
* ``propagation.py:1473-1486`` / ``2605-2616`` -- ``apply_F`` (SpMV / SpMM);
* ``propagation.py:2476-2488`` -- multi-RHS injection columns;
* ``src/prince_cr/solvers/etd2.py:329-439`` -- phi functions and the step;
* ``src/prince_cr/solvers/partial_diff.py:48-110`` -- FD loss operator;
* ``src/prince_cr/interaction_rates.py:966-1067`` -- rate fold;
* ``interaction_rates.py:1202-1210, 1277-1294`` -- loss vectors;
* ``propagation.py:555-665`` -- EM-cascade step hooks (Bethe-Heitler pair
  injection, then the cascade transfer of gamma and e+-).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
from scipy.integrate import trapezoid

# Physical constants used by the restatement (same expressions as the reference
# unit table, src/prince_cr/data.py:722-740, and config.py:128-135).
import scipy.constants as _spc

CM2SEC = 1e-2 / _spc.c
H_0S = 2.28475e-18
OMEGA_M = 0.27
OMEGA_L = 0.73

PHI1_SMALL = 1e-6   # etd2.py:43
PHI2_SMALL = 1e-3   # etd2.py:44


def hubble(z):
    """cosmology.py:10-21."""
    return H_0S * np.sqrt(OMEGA_M * (1 + z) ** 3 + OMEGA_L)


def dldz(z):
    """propagation.py:360-361."""
    return -1.0 / ((1.0 + z) * hubble(z) * CM2SEC)


def z_grid(initial_z, final_z, dz):
    """Uniform descending grid with a truncated last step (propagation.py:828-832)."""
    dz_step = -float(abs(dz))
    n_full = int(np.floor((final_z - initial_z) / dz_step))
    zg = initial_z + np.arange(n_full + 1) * dz_step
    if abs(zg[-1] - final_z) > 1e-12:
        zg = np.concatenate([zg, [final_z]])
    return zg


def window_starts(zg, thr):
    """Redshifts at which the rate cache is refreshed (propagation.py:1383-1387)."""
    cur = None
    out = []
    for k in range(len(zg) - 1):
        z = zg[k]
        if cur is None or abs(z - cur) > thr:
            cur = z
            out.append(z)
    return out


def phi_factors(h, d, exp=np.exp):
    """eD, phi1, phi2 with the Taylor patches of etd2.py:329-390.

    ``exp`` is the exponential: numpy's (as the reference) or the correctly
    rounded one of ``oracle.crexp`` (as the CUDA path).
    """
    hD = d * h
    eD = exp(hD)
    a = np.abs(hD)
    m1 = a > PHI1_SMALL
    m2 = a > PHI2_SMALL
    den1 = np.where(m1, hD, 1.0)
    phi1 = (eD - 1.0) / den1
    t1 = hD * (1.0 / 6.0)
    t1 = (t1 + 0.5) * hD + 1.0
    phi1 = np.where(m1, phi1, t1)
    den2 = np.where(m2, hD * hD, 1.0)
    phi2 = ((eD - 1.0) - hD) / den2
    t2 = hD * (1.0 / 24.0)
    t2 = (t2 + 1.0 / 6.0) * hD + 0.5
    phi2 = np.where(m2, phi2, t2)
    return eD, phi1, phi2


def fd_operator_run(run):
    """The run's FD loss operator, one block per species on its home grid in
    princeidx order (partial_diff.py:28-46, heterogeneous path)."""
    sm = run.spec_man
    grids = getattr(run, "grids", {"default": run.cr_grid})
    refs = sorted(sm.species_refs, key=lambda s: s.princeidx)
    if all(s.grid_tag == "default" for s in refs):
        return fd_operator(run.cr_grid, sm.nspec)
    blocks = {}
    for s in refs:
        if s.grid_tag not in blocks:
            blocks[s.grid_tag] = fd_operator(grids[s.grid_tag], 1)
    return sp.block_diag([blocks[s.grid_tag] for s in refs]).tocsr()


def fd_operator(cr_grid, nspec):
    """Block-diagonal FD loss operator (partial_diff.py:28-110)."""
    h = np.log(cr_grid.bins[1] / cr_grid.bins[0])
    d = cr_grid.d
    last = d - 1
    op = np.zeros((d, d))
    op[0, [1, 2, 3]] = np.asarray([-3, 4, -1]) / (2.0 * h)
    for r in (1, 2):
        op[r, r + np.asarray([-1, 0, 1, 2])] = np.asarray([-2, -3, 6, -1]) / (6.0 * h)
    op[last, last + np.asarray([-3, -2, -1])] = np.asarray([1, -4, 3]) / (2.0 * h)
    for r in (last - 1, last - 2):
        op[r, r + np.asarray([-2, -1, 0, 1])] = np.asarray([1, -6, 3, 2]) / (6.0 * h)
    for r in range(3, d - 3):
        op[r, r + np.asarray([-1, 0, 1, 2, 3])] = np.asarray([-3, -10, 18, -6, 1]) / (12.0 * h)
    blk = sp.coo_matrix(op * (1.0 / cr_grid.grid)[:, None])
    return sp.block_diag(nspec * [blk]).tocsr()


def split(L):
    """etd2.py:246-252 (host branch)."""
    d = np.asarray(L.diagonal(), dtype=np.float64)
    off = L - sp.diags(d, format=L.format)
    off = off.tocsr()
    off.eliminate_zeros()
    off.sort_indices()
    return d, off


def index_maps(M, M_off):
    """off_to_M / diag_to_M of propagation.py:721-807 (sorted CSR inputs)."""
    n = M.shape[0]
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(M.indptr))
    keys = rows * n + M.indices.astype(np.int64)
    dmask = M.indices == rows
    diag_to_M = np.full(n, -1, dtype=np.int64)
    diag_to_M[rows[dmask]] = np.flatnonzero(dmask)
    orow = np.repeat(np.arange(n, dtype=np.int64), np.diff(M_off.indptr))
    okeys = orow * n + M_off.indices.astype(np.int64)
    off_to_M = np.searchsorted(keys, okeys).astype(np.int64)
    if not np.array_equal(keys[off_to_M], okeys):
        raise RuntimeError("M_off has columns with no source in M")
    return off_to_M, diag_to_M


@dataclass
class Flags:
    """Solver enable flags (propagation.py:196-209)."""

    adiabatic: bool = True
    pairprod: bool = True
    photohad: bool = True
    injection: bool = True
    partial_diff: bool = True


@dataclass
class Trace:
    """Intermediate quantities recorded for tests."""

    windows: list = field(default_factory=list)
    M_off_first: object = None
    d_M_first: object = None
    kappa_pair_first: object = None


def _pair_loss(run, z):
    """interaction_rates.py:1277-1294 on the run's precomputed arrays."""
    pl = run.pair_loss_rates_grid
    pg = pl.photon_grid
    dens = run.photon_field.get_photon_density(pg.reshape(-1), z).reshape(pg.shape)
    rate_single = trapezoid(dens * pl.phi_xi2, pl.xi, axis=1)
    rate_full = np.zeros(run.dim_states)
    for s in run.spec_man.species_refs:
        if s.is_nucleus:
            rate_full[s.lidx():s.uidx()] = rate_single
    return pl.scale_vec * rate_full


class OracleSolver:
    """CPU ETD2 solve of one run; ``K=None`` for the single-RHS path.

    ``sources`` is a list of source objects (single RHS) or a list of K
    lists (one per column).  Sources expose ``injection_rate(z)``.
    """

    def __init__(self, run, initial_z, final_z, flags=None, thr=None, K=None, decay=None, exp="numpy",
                 em=None, perturb=None):
        self.run = run
        self.initial_z = float(initial_z)
        self.final_z = float(final_z)
        self.flags = flags or Flags()
        self.thr = run.backend.update_rates_z_threshold if thr is None else float(thr)
        self.K = K
        self.n = run.dim_states
        ir = run.int_rates
        self.bm = np.ascontiguousarray(ir._batch_matrix, dtype=np.float64)
        self.cpl_indptr = np.asarray(ir.coupling_mat.indptr)
        self.cpl_indices = np.asarray(ir.coupling_mat.indices)
        self.D = fd_operator_run(run)
        self.D_diag, self.D_off = split(self.D)
        self.E = np.asarray(run.adia_loss_rates_grid.energy_vector, dtype=np.float64)
        # Explicit decay (propagation.py:1148-1358, 1418-1422, 1479-1482):
        # ``decay = (Lambda_diag, Lambda_off CSR)``, constant over the solve.
        self.L_diag, self.L_off = (None, None) if decay is None else decay
        # ``exp="cr"`` evaluates the phi functions with the correctly rounded
        # exp (the CUDA path's); ``"numpy"`` with the host numpy exp (the
        # reference's, whose rounding depends on the CPU's SIMD level).
        if exp == "cr":
            from oracle import crexp
            self._exp = crexp.exp
        else:
            self._exp = np.exp
        # Co-evolved EM cascade (propagation.py:555-665): ``em(z)`` returns the
        # window's (T_gamma, T_electron, R_BH); applied after every step.
        self.em = em
        if em is not None:
            sm = run.spec_man
            self._em_gamma_sl = sm.pdgid2sref[22].sl
            self._em_lep_sl = [sm.pdgid2sref[p].sl for p in (11, -11) if p in sm.pdgid2sref]
            self._em_bh_species = [(sp.sl, float(sp.A)) for sp in sm.species_refs
                                   if sp.is_nucleus and abs(sp.charge) >= 1]
        # ``perturb=(delta, seed)`` multiplies every window's operator values
        # (M_off, its diagonal, kappa_pair) by 1 + delta N(0, 1): a probe of how
        # far each output bin moves under operator differences of the size
        # that different math libraries and summation orders produce.
        self._perturb = None
        if perturb is not None:
            self._perturb = (float(perturb[0]), np.random.default_rng(int(perturb[1])))
        self.trace = Trace()

    # -- per window --------------------------------------------------------
    def _refresh(self, z, first):
        photon = self.run.int_rates.photon_vector(z)
        vec = np.dot(self.bm, photon)
        if not self.flags.photohad:
            vec = np.zeros_like(vec)
        if first:
            M = sp.csr_matrix((vec, self.cpl_indices, self.cpl_indptr), shape=(self.n, self.n))
            M.sort_indices()
            self.d_M, self.M_off = split(M)
            self.off_to_M, self.diag_to_M = index_maps(M, self.M_off)
            self.trace.M_off_first = self.M_off.copy()
            self.trace.d_M_first = self.d_M.copy()
        else:
            if self.M_off.data.size:
                self.M_off.data[:] = vec[self.off_to_M]
            d_M = np.zeros(self.n)
            present = self.diag_to_M >= 0
            d_M[present] = vec[self.diag_to_M[present]]
            self.d_M = d_M
        self.kappa_pair = _pair_loss(self.run, z) if self.flags.pairprod else None
        if self._perturb is not None:
            delta, rng = self._perturb
            self.M_off.data *= 1.0 + delta * rng.standard_normal(self.M_off.data.size)
            self.d_M = self.d_M * (1.0 + delta * rng.standard_normal(self.d_M.size))
            if self.kappa_pair is not None:
                self.kappa_pair = self.kappa_pair * (1.0 + delta * rng.standard_normal(self.kappa_pair.size))
        if self.em is not None:
            self._em_T = self.em(z)
            self._em_z = float(z)
        if first:
            self.trace.kappa_pair_first = None if self.kappa_pair is None else self.kappa_pair.copy()
        self.trace.windows.append(z)

    # -- injection ---------------------------------------------------------
    def _injection(self, z, sources):
        f = dldz(z) * 1.0 * CM2SEC
        if self.K is None:
            if len(sources) > 1:
                return f * np.sum([s.injection_rate(z) for s in sources], axis=0)
            return f * sources[0].injection_rate(z)
        out = np.zeros((self.n, self.K))
        for k, srcs in enumerate(sources):
            if not srcs:
                continue
            if len(srcs) > 1:
                col = np.sum([s.injection_rate(z) for s in srcs], axis=0)
            else:
                col = srcs[0].injection_rate(z)
            out[:, k] = f * col
        return out

    def solve(self, sources, dz=1e-3, state=None):
        zg = z_grid(self.initial_z, self.final_z, dz)
        shape = (self.n,) if self.K is None else (self.n, self.K)
        x = np.zeros(shape) if state is None else np.array(state, dtype=np.float64)
        have_src = any(sources) if self.K is not None else bool(sources)
        cur = None
        for k in range(len(zg) - 1):
            z0 = zg[k]
            h = zg[k + 1] - z0
            if cur is None or abs(z0 - cur) > self.thr:
                self._refresh(z0, first=cur is None)
                cur = z0
            dl = dldz(z0)
            if self.flags.partial_diff:
                kappa = np.zeros(self.n)
                if self.flags.adiabatic:
                    kappa += hubble(z0) * CM2SEC * self.E
                if self.kappa_pair is not None:
                    kappa += self.kappa_pair
            else:
                kappa = None
            b = self._injection(z0, sources) if (self.flags.injection and have_src) else None
            d = self.d_M * dl
            if kappa is not None:
                kx = kappa * self.D_diag
                kx = kx * dl
                d = d + kx
            if self.L_diag is not None:
                d = d + self.L_diag * dl
            x = self._step(x, h, d, dl, kappa, b)
            if self.em is not None:
                self._inject_bh_pairs(x, dz)
                self._apply_em_cascade(x)
        return x

    def _inject_bh_pairs(self, x, dz):
        """propagation.py:620-665."""
        Tg, Te, R = self._em_T
        z = self._em_z
        E_p = self.run.cr_grid.grid
        dE = np.gradient(E_p)
        loss_full = _pair_loss(self.run, z)
        dl_step = 1e2 * _spc.c * abs(dz) / ((1.0 + z) * hubble(z))
        w = None
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_E = np.where(E_p > 0, 1.0 / E_p, 0.0)
            for sl, A in self._em_bh_species:
                n_s = x[sl]
                cw = A * loss_full[sl] * dl_step * inv_E * dE
                if n_s.ndim == 2:
                    cw = cw[:, None]
                term = cw * n_s
                w = term if w is None else w + term
        e_src = R @ w
        for sl in self._em_lep_sl:
            x[sl] = x[sl] + e_src

    def _apply_em_cascade(self, x):
        """propagation.py:555-571."""
        Tg, Te, R = self._em_T
        ph = np.array(x[self._em_gamma_sl])
        lep = np.zeros_like(ph)
        for sl in self._em_lep_sl:
            lep = lep + x[sl]
            x[sl] = 0.0
        x[self._em_gamma_sl] = Tg @ ph + Te @ lep

    def _apply_F(self, x, dl, kappa, b):
        out = np.asarray(self.M_off.dot(x))
        if kappa is not None:
            kx = (kappa[:, None] * x) if x.ndim == 2 else kappa * x
            out = out + self.D_off.dot(kx)
        if self.L_off is not None:
            out = out + self.L_off.dot(x)
        out = out * dl
        if b is not None:
            out = out + b
        return out

    def _step(self, x, h, d, dl, kappa, b):
        eD, phi1, phi2 = phi_factors(h, d, self._exp)
        if x.ndim == 2:
            eD, phi1, phi2 = eD[:, None], phi1[:, None], phi2[:, None]
        F_phi = self._apply_F(x, dl, kappa, b)
        a = eD * x
        s = phi1 * F_phi
        s = s * h
        a = a + s
        F_a = self._apply_F(a, dl, kappa, b)
        s = F_a - F_phi
        s = s * h
        s = (phi2 * s) if x.ndim == 2 else (s * phi2)
        return a + s


def integrate_const(state, zg, d, L_off=None, exp=np.exp):
    """ETD2 with a z-independent operator (etd2.py:478-517 with a constant closure)."""
    x = np.array(state, dtype=np.float64)
    for k in range(len(zg) - 1):
        h = zg[k + 1] - zg[k]
        eD, phi1, phi2 = phi_factors(h, np.asarray(d, dtype=np.float64), exp)

        def F(v):
            return np.zeros_like(v) if L_off is None else np.asarray(L_off @ v)

        F_phi = F(x)
        a = eD * x + (phi1 * F_phi) * h
        F_a = F(a)
        x = a + ((F_a - F_phi) * h) * phi2
    return x
