#!/usr/bin/env python
"""Generate the golden vectors of the ETD2 path by running the PriNCe reference.

Run it with ``PRINCE_REFERENCE`` set to a checkout of the PriNCe reference
source tree (the directory that holds ``src/prince_cr``)::

    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py        # light network
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --em   # light network + EM cascade
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --em-decoupled  # ... on a decoupled EM grid
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --groups  # result post-processing
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --ebl     # tabulated EBL (Gilmore 2012)
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --kernel  # fold-kernel construction inputs
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --cascade # kinetic EM-cascade transfer
    PRINCE_REFERENCE=<path> python tests/golden/make_golden.py --cascade-128  # ... on the 128-bin EM grid

The reference package is copied to a scratch directory (it tries to
download its HDF5 database at import unless a file is present, and it
imports ``h5py``, which this environment lacks), so the script

* places an empty ``prince_db_05.h5`` next to the copied package,
* puts a minimal ``h5py`` stand-in first on ``sys.path``,
* selects the FP64 settings (dense fold kernel, float64 cross-section
  dtype, scipy backend, ``tau_dec_threshold = 0``),
* defines a small synthetic cross-section model (Lorentzian resonances plus
  a photo-pion bump) because the FLUKA
  database is not available offline.

It then builds the light-nuclei run (p, n, 2H, 3H, 3He, 4He; 64 bins over
1e6-1e14 GeV at 8 bins/decade; CMB; z = 1 -> 0, dz = 1e-3) and records the
inputs the ETD2 path consumes together with the reference's own outputs
(final states of single- and multi-RHS solves, per-window intermediates).
The result is ``tests/golden/light_network.npz`` (and, with ``--em``,
``tests/golden/light_network_em.npz``).

``--groups`` feeds states of ``light_network.npz`` (and variants with
non-positive bins inside and at the ends of the spectra) to the reference's
own ``UHECRPropagationResult`` and records ``get_solution_group``,
``get_lnA`` and ``get_solution_scale`` in ``tests/golden/result_groups.npz``.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PRINCE_REFERENCE")


def _prepare_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "src", "prince_cr")):
        raise SystemExit("set PRINCE_REFERENCE to the PriNCe source tree (the directory holding src/prince_cr)")
    tmp = tempfile.mkdtemp(prefix="prince_golden_")
    shutil.copytree(os.path.join(REF, "src", "prince_cr"), os.path.join(tmp, "prince_cr"))
    os.chmod(os.path.join(tmp, "prince_cr", "data"), 0o755)
    open(os.path.join(tmp, "prince_cr", "data", "prince_db_05.h5"), "wb").close()

    h5 = types.ModuleType("h5py")

    class _File:
        def __init__(self, *a, **k):
            self.attrs = {"version": "stub"}

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def __contains__(self, k):
            return False

    h5.File = _File
    sys.modules["h5py"] = h5
    sys.path.insert(0, tmp)
    return tmp


def _lorentz(eg, e0, w, peak, thr):
    return peak * (eg * w) ** 2 / ((eg ** 2 - e0 ** 2) ** 2 + (eg * w) ** 2) * (eg > thr)


def build(config, base, photon_field=None):
    """Return the reference's light-nuclei run (CMB unless ``photon_field`` is given)."""
    from prince_cr import core, photonfields

    class SynthXS(base):
        def __init__(self):
            self.supports_redistributions = True
            base.__init__(self)
            # The table reaches y = E eps / m_p beyond the largest value the grids
            # probe (1e14 GeV x 1e-6 GeV / m_p), so no kernel row crosses the end of
            # the tabulated response.
            eg = np.logspace(-3, 9, 481)
            self._egrid_tab = eg
            self.xbins = np.logspace(-5, 0, 101)
            mb = 1e-27
            pion = lambda A: (_lorentz(eg, 0.34, 0.12, 0.5 * A * mb, 0.145)
                              + 0.12 * A * mb * (eg > 0.5))
            gdr = {1000010020: (0.0042, 0.004, 2.4), 1000010030: (0.012, 0.006, 1.3),
                   1000020030: (0.012, 0.006, 1.4), 1000020040: (0.026, 0.008, 2.2)}
            A_of = {2212: 1, 2112: 1, 1000010020: 2, 1000010030: 3, 1000020030: 3,
                    1000020040: 4}
            for mo, A in A_of.items():
                tab = pion(A)
                if mo in gdr:
                    e0, w, s = gdr[mo]
                    tab = tab + _lorentz(eg, e0, w, s * mb, 0.0022)
                self._nonel_tab[mo] = tab
            # Channel yields conserve the nucleon number: 4He -> 3He+n | 3H+p | d+d,
            # 3He -> d+p | p+p+n, 3H -> d+n | p+n+n, d -> p+n.
            bc = {1000020040: [(1000020030, 0.45), (1000010030, 0.45), (1000010020, 0.2)],
                  1000020030: [(1000010020, 0.9)], 1000010030: [(1000010020, 0.9)]}
            nuc = {1000020040: (0.45, 0.45), 1000020030: (1.1, 0.1), 1000010030: (0.1, 1.1),
                   1000010020: (1.0, 1.0)}
            for mo, das in bc.items():
                for da, w in das:
                    self._incl_tab[(mo, da)] = w * self._nonel_tab[mo]
            for mo, (mp, mn) in nuc.items():
                self._incl_tab[(mo, 2212)] = mp * self._nonel_tab[mo]
                self._incl_tab[(mo, 2112)] = mn * self._nonel_tab[mo]
            # Nucleon yields are given as total cross sections; the reference
            # places them in the x = 1 bin of its redistribution grid.
            for mo in (2212, 2112):
                self._incl_tab[(mo, mo)] = 0.7 * self._nonel_tab[mo]
                self._incl_tab[(mo, 4324 - mo)] = 0.3 * self._nonel_tab[mo]
            self.set_range()
            self._optimize_and_generate_index()

    run = core.PriNCeRun(max_mass=4, photon_field=photon_field or photonfields.CMBPhotonSpectrum(),
                         cross_sections=SynthXS())
    return run


def main():
    _prepare_reference()
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (6, 14, 8)
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"

    from prince_cr import cr_sources
    from prince_cr.cross_sections.base import CrossSectionBase
    from prince_cr.solvers import MultiRHSPropagationSolverETD2, UHECRPropagationSolverETD2
    from prince_cr.solvers import etd2 as ref_etd2

    run = build(config, CrossSectionBase)
    run.backend.xs_dtype = "float64"
    ir = run.int_rates
    sm = run.spec_man
    species = np.array(sm.known_species, dtype=np.int64)

    class ZmaxRigidity(cr_sources.RigdityCutoffSource):
        def __init__(self, *a, z_max=np.inf, **k):
            self.z_max = z_max
            super().__init__(*a, **k)

        def evolution(self, z):
            if z > self.z_max:
                return 0.0
            return super().evolution(z)

    # Source set: (kind, params, norm, m, z_max).  Columns of the multi-RHS run
    # are lists of these.
    eq = {int(p): (2.0, 1e10, 1.0) for p in species}
    SRC = {
        "eq": ("RigdityCutoffSource", eq, 1.0, "flat", np.inf),
        "auger": ("AugerFitSource", {2212: (1.0, 10 ** 9.5, 2.0), 1000020040: (1.0, 10 ** 9.5, 1.0)},
                  3.0, ("simple", 3.0), np.inf),
        "soft": ("SimpleSource", {2212: (2.6, 1e11, 1.0), 1000010020: (2.2, 1e11, 0.5)},
                 0.5, ("simple", -1.0), np.inf),
        "late": ("RigdityCutoffSource", {1000020040: (-0.5, 10 ** 9.2, 1.0), 2212: (1.5, 10 ** 10.5, 0.3)},
                 2.0, ("simple", 1.5), 0.55),
    }

    def make(key):
        kind, params, norm, m, zmax = SRC[key]
        if kind == "RigdityCutoffSource" and np.isfinite(zmax):
            return ZmaxRigidity(run, norm=norm, params=params, m=m, z_max=zmax)
        return getattr(cr_sources, kind)(run, norm=norm, params=params, m=m)

    out = {}
    out["species"] = species
    out["cr_grid"] = np.array(config.cosmic_ray_grid, dtype=np.float64)
    out["ph_grid"] = np.array(config.photon_grid, dtype=np.float64)
    out["batch_matrix"] = np.asarray(ir._batch_matrix, dtype=np.float64)
    out["batch_rows"] = np.asarray(ir._batch_rows, dtype=np.int64)
    out["batch_cols"] = np.asarray(ir._batch_cols, dtype=np.int64)
    out["cpl_indptr"] = np.asarray(ir.coupling_mat.indptr, dtype=np.int64)
    out["cpl_indices"] = np.asarray(ir.coupling_mat.indices, dtype=np.int64)
    out["photon_vector_z1"] = ir.photon_vector(1.0)
    out["xi"] = run.pair_loss_rates_grid.xi
    out["phi_xi2"] = run.pair_loss_rates_grid.phi_xi2
    out["pair_scale_vec"] = run.pair_loss_rates_grid.scale_vec
    out["adia_energy"] = run.adia_loss_rates_grid.energy_vector
    out["kappa_pair_z1"] = run.pair_loss_rates_grid.loss_vector(1.0)
    out["kappa_pair_z05"] = run.pair_loss_rates_grid.loss_vector(0.5)
    for key in SRC:
        kind, params, norm, m, zmax = SRC[key]
        out[f"src_{key}_grid"] = make(key).injection_grid

    def fresh_fold_cache():
        # The reference caches its row-subset fold kernels on the run after the
        # first solve and reuses them in later solves, although the M_off
        # pattern depends on the first window's photon field: a later solve
        # from another initial z would read a stale cache.  Dropping the cache
        # before each solve keeps every solve on its own first-window pattern.
        ir._sf_off_kernel = None

    def single(keys, zi=1.0, zf=0.0, dz=1e-3, thr=None, **flags):
        fresh_fold_cache()
        s = UHECRPropagationSolverETD2(initial_z=zi, final_z=zf, prince_run=run, **flags)
        if thr is not None:
            s.recomp_z_threshold = thr
        windows = []
        orig = s._refresh_z_caches

        def rec(z):
            windows.append(z)
            return orig(z)

        s._refresh_z_caches = rec
        for k in keys:
            s.add_source_class(make(k))
        s.solve(dz=dz)
        return s, np.asarray(s.state), np.asarray(windows)

    s, st, win = single(["eq"])
    out["state_plain"] = st
    out["windows_plain"] = win
    # Intermediates from a fresh solver stopped after its first window.
    fresh_fold_cache()
    probe = UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
    probe._reset_for_solve()
    probe._ensure_D_split()
    probe._refresh_z_caches(1.0)
    out["M_off_indptr"] = np.asarray(probe._etd2_M_raw_off.indptr, dtype=np.int64)
    out["M_off_indices"] = np.asarray(probe._etd2_M_raw_off.indices, dtype=np.int64)
    out["M_off_data_z1"] = np.asarray(probe._etd2_M_raw_off.data)
    out["M_diag_z1"] = np.asarray(probe._etd2_M_raw_diag)
    out["D_diag"] = np.asarray(probe._etd2_D_diag)
    out["D_off_indptr"] = np.asarray(probe._etd2_D_off.indptr, dtype=np.int64)
    out["D_off_indices"] = np.asarray(probe._etd2_D_off.indices, dtype=np.int64)
    out["D_off_data"] = np.asarray(probe._etd2_D_off.data)

    out["state_no_pair"] = single(["eq"], enable_pairprod_losses=False)[1]
    out["state_no_adia"] = single(["eq"], enable_adiabatic_losses=False)[1]
    out["state_no_pdiff"] = single(["eq"], enable_partial_diff_jacobian=False)[1]
    out["state_no_photohad"] = single(["eq"], enable_photohad_losses=False)[1]
    out["state_two_src"] = single(["auger", "soft"])[1]
    s_thr, st_thr, win_thr = single(["eq"], zi=0.5, zf=0.0, dz=2e-3, thr=1e-3)
    out["state_thr"] = st_thr
    out["windows_thr"] = win_thr
    s_dec, st_dec, _ = single(["eq"], enable_decay=True)
    out["state_decay"] = st_dec
    lam_d = s_dec._etd2_Lambda_diag
    lam_o = s_dec._etd2_Lambda_off
    out["lambda_diag"] = np.zeros(run.dim_states) if lam_d is None else np.asarray(lam_d)
    if lam_o is not None:
        lam_o = lam_o.tocsr()
        lam_o.sort_indices()
        out["lambda_indptr"] = np.asarray(lam_o.indptr, dtype=np.int64)
        out["lambda_indices"] = np.asarray(lam_o.indices, dtype=np.int64)
        out["lambda_data"] = np.asarray(lam_o.data)

    cols = [["eq"], ["auger"], ["soft", "auger"], ["late"]]
    fresh_fold_cache()
    m = MultiRHSPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run, K=len(cols))
    for k, keys in enumerate(cols):
        for key in keys:
            m[k].add_source_class(make(key))
    m.solve(dz=1e-3)
    out["state_multi"] = np.asarray(m.state)
    out["multi_columns"] = np.array([",".join(c) for c in cols])

    # Kernel-level known answers of the integrator with a constant operator.
    zg = np.linspace(0.0, 6.0, 2001)
    x = np.array([1.0, 0.0, 0.0])
    dconst = np.array([-1.0, -0.4, 0.0])
    import scipy.sparse as sps

    L = sps.csr_matrix(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.4, 0.0]]))

    def op(z):
        def apply_F(v, o):
            np.copyto(o, L @ v)
        return dconst, apply_F

    ref_etd2.integrate(x, zg, op)
    out["chain3_state"] = x

    for key, (kind, params, norm, mm, zmax) in SRC.items():
        out[f"src_{key}_kind"] = np.array(kind)
        out[f"src_{key}_norm"] = np.array(norm)
        out[f"src_{key}_zmax"] = np.array(zmax)
        out[f"src_{key}_m"] = np.array(repr(mm))
        out[f"src_{key}_params"] = np.array(repr(params))

    path = os.path.join(HERE, "light_network.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_em():
    """Light network with the co-evolved EM cascade (gamma, e+-) on the shared grid.

    The per-window cascade transfer and Bethe-Heitler pair shape are supplied by
    the synthetic stand-ins ``prince_b200.synth.em_cascade_matrices`` (patched
    into the reference solver's ``_em_transfer_at`` / ``_em_bh_at``); the
    reference then runs its own step hooks ``_inject_bh_pairs`` and
    ``_apply_em_cascade`` after every ETD2 step.
    """
    _prepare_reference()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from prince_b200 import synth
    from prince_b200.data import EnergyGrid
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (8, 12, 8)
    config.em_cascade_grid_lo = 7.0
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"

    from prince_cr import core, cr_sources
    from prince_cr.cross_sections.base import CrossSectionBase
    from prince_cr.solvers import MultiRHSPropagationSolverETD2, UHECRPropagationSolverETD2

    orig = core.PriNCeRun

    def em_run(*a, **k):
        k.update(enable_em_cascade=True, enable_em_decoupled_grid=False)
        return orig(*a, **k)

    core.PriNCeRun = em_run
    run = build(config, CrossSectionBase)
    core.PriNCeRun = orig
    ir = run.int_rates
    grid = run.cr_grid
    lo, hi = np.log10(grid.bins[0]), np.log10(grid.bins[-1])
    mine = EnergyGrid(lo, hi, 8)
    assert np.allclose(mine.grid, grid.grid, rtol=1e-14)

    def patch(s):
        s._em_transfer_at = lambda z: synth.em_cascade_matrices(mine, mine, float(z))[:2]
        s._em_bh_at = lambda z: synth.em_cascade_matrices(mine, mine, float(z))[2]
        return s

    eq = {2212: (2.0, 1e10, 1.0), 1000020040: (2.0, 1e10, 1.0)}
    soft = {2212: (2.5, 3e10, 1.0)}
    out = {}
    out["species"] = np.array(run.spec_man.known_species, dtype=np.int64)
    out["cr_grid"] = np.array([lo, hi, 8.0])
    out["ph_grid"] = np.array(config.photon_grid, dtype=np.float64)
    out["batch_matrix"] = np.asarray(ir._batch_matrix, dtype=np.float64)
    out["batch_rows"] = np.asarray(ir._batch_rows, dtype=np.int64)
    out["batch_cols"] = np.asarray(ir._batch_cols, dtype=np.int64)
    out["cpl_indptr"] = np.asarray(ir.coupling_mat.indptr, dtype=np.int64)
    out["cpl_indices"] = np.asarray(ir.coupling_mat.indices, dtype=np.int64)
    s = patch(UHECRPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run))
    s.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=eq))
    s.solve(dz=1e-3)
    out["state_em"] = np.asarray(s.state)
    m = patch(MultiRHSPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run, K=2))
    m[0].add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=eq))
    m[1].add_source_class(cr_sources.SimpleSource(run, norm=1.0, params=soft, m=("simple", 2.0)))
    m.solve(dz=1e-3)
    out["state_em_multi"] = np.asarray(m.state)
    out["src_eq"] = np.array(repr(eq))
    out["src_soft"] = np.array(repr(soft))
    path = os.path.join(HERE, "light_network_em.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_em_decoupled():
    """Light network with the co-evolved EM cascade on a decoupled EM grid.

    gamma and e+- live on the reference's own EM grid (from the electron mass
    to the top of the nuclear grid, 8 bins per decade) while the nuclei keep
    the 8-12 nuclear grid; the per-window transfer (EM grid) and the
    Bethe-Heitler pair shape (EM grid x nuclear grid) are the synthetic
    stand-ins of ``prince_b200.synth.em_cascade_matrices``, patched into the
    reference solver as in ``main_em``.
    """
    _prepare_reference()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from prince_b200 import synth
    from prince_b200.data import EnergyGrid
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (8, 12, 8)
    config.em_grid_bins_dec = 8
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"

    from prince_cr import core, cr_sources
    from prince_cr.cross_sections.base import CrossSectionBase
    from prince_cr.solvers import MultiRHSPropagationSolverETD2, UHECRPropagationSolverETD2

    orig = core.PriNCeRun

    def em_run(*a, **k):
        k.update(enable_em_cascade=True, enable_em_decoupled_grid=True)
        return orig(*a, **k)

    core.PriNCeRun = em_run
    run = build(config, CrossSectionBase)
    core.PriNCeRun = orig
    assert run.em_grid is not None
    ir = run.int_rates
    grid, egrid = run.cr_grid, run.em_grid
    lo, hi = np.log10(grid.bins[0]), np.log10(grid.bins[-1])
    elo, ehi = np.log10(egrid.bins[0]), np.log10(egrid.bins[-1])
    mine = EnergyGrid(lo, hi, 8)
    mine_em = EnergyGrid(elo, ehi, 8)
    assert np.allclose(mine.grid, grid.grid, rtol=1e-14)
    assert np.allclose(mine_em.grid, egrid.grid, rtol=1e-14)

    def patch(s):
        s._em_transfer_at = lambda z: synth.em_cascade_matrices(mine_em, mine, float(z))[:2]
        s._em_bh_at = lambda z: synth.em_cascade_matrices(mine_em, mine, float(z))[2]
        return s

    eq = {2212: (2.0, 1e10, 1.0), 1000020040: (2.0, 1e10, 1.0)}
    soft = {2212: (2.5, 3e10, 1.0)}
    out = {}
    out["species"] = np.array(run.spec_man.known_species, dtype=np.int64)
    out["cr_grid"] = np.array([lo, hi, 8.0])
    out["em_grid"] = np.array([elo, ehi, 8.0])
    out["ph_grid"] = np.array(config.photon_grid, dtype=np.float64)
    out["dim_states"] = np.array(run.dim_states)
    out["lidx"] = np.array([s.lidx() for s in sorted(run.spec_man.species_refs, key=lambda s: s.princeidx)])
    out["adia_energy"] = np.asarray(run.adia_loss_rates_grid.energy_vector)
    out["batch_matrix"] = np.asarray(ir._batch_matrix, dtype=np.float64)
    out["batch_rows"] = np.asarray(ir._batch_rows, dtype=np.int64)
    out["batch_cols"] = np.asarray(ir._batch_cols, dtype=np.int64)
    out["cpl_indptr"] = np.asarray(ir.coupling_mat.indptr, dtype=np.int64)
    out["cpl_indices"] = np.asarray(ir.coupling_mat.indices, dtype=np.int64)
    s = patch(UHECRPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run))
    s._ensure_D_split()
    out["D_diag"] = np.asarray(s._etd2_D_diag)
    out["D_off_indptr"] = np.asarray(s._etd2_D_off.indptr, dtype=np.int64)
    out["D_off_indices"] = np.asarray(s._etd2_D_off.indices, dtype=np.int64)
    out["D_off_data"] = np.asarray(s._etd2_D_off.data)
    s.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=eq))
    s.solve(dz=1e-3)
    out["state_em"] = np.asarray(s.state)
    m = patch(MultiRHSPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run, K=2))
    m[0].add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=eq))
    m[1].add_source_class(cr_sources.SimpleSource(run, norm=1.0, params=soft, m=("simple", 2.0)))
    m.solve(dz=1e-3)
    out["state_em_multi"] = np.asarray(m.state)
    out["src_eq"] = np.array(repr(eq))
    out["src_soft"] = np.array(repr(soft))
    path = os.path.join(HERE, "light_network_em_decoupled.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_groups():
    """The reference's result post-processing on recorded states."""
    _prepare_reference()
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (6, 14, 8)
    from prince_cr.data import EnergyGrid as RefGrid
    from prince_cr.data import SpeciesManager as RefSpeciesManager
    from prince_cr.solvers import UHECRPropagationResult as RefResult

    z = dict(np.load(os.path.join(HERE, "light_network.npz")))
    egrid = RefGrid(*config.cosmic_ray_grid).grid
    species = [int(p) for p in z["species"]]
    sm = RefSpeciesManager(species, egrid.size)
    rng = np.random.default_rng(17)
    mixed = np.array(z["state_two_src"])
    d = egrid.size
    for i in range(len(species)):
        blk = mixed[i * d:(i + 1) * d]
        interior = rng.choice(np.arange(3, d - 3), 6, replace=False)
        blk[interior[:3]] *= -1.0
        blk[interior[3:]] = 0.0
        blk[:2] = -abs(blk[:2])
        blk[-1] = 0.0
    states = {"plain": z["state_plain"], "two_src": z["state_two_src"], "mixed": mixed}
    for k in range(z["state_multi"].shape[1]):
        states[f"multi{k}"] = z["state_multi"][:, k]
    out = {"species": np.array(species, dtype=np.int64), "cr_grid": np.array(config.cosmic_ray_grid)}
    custom = np.logspace(6.2, 14.4, 57)
    out["custom_grid"] = custom
    for name, st in states.items():
        res = RefResult(np.array(st), egrid, sm)
        out[f"{name}_state"] = np.array(st)
        g, f = res.get_solution_group("CR", epow=3)
        out["common_grid"] = g
        out[f"{name}_CR_e3"] = f
        out[f"{name}_CR_e0"] = res.get_solution_group("CR", epow=0)[1]
        out[f"{name}_heavy_e2"] = res.get_solution_group([1000020030, 1000020040, 1000010030], epow=2)[1]
        out[f"{name}_custom_e3"] = res.get_solution_group("all", epow=3, egrid=custom)[1]
        _, mean, var = res.get_lnA("CR")
        out[f"{name}_lnA_mean"] = mean
        out[f"{name}_lnA_var"] = var
        out[f"{name}_He4_scale_e1"] = res.get_solution_scale(1000020040, epow=1)[1]
    path = os.path.join(HERE, "result_groups.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_ebl():
    """The light network in CMB + the tabulated Gilmore (2012) EBL.

    Records the two tabulated EBL models' tables (the inputs), the reference's
    densities at sample points, its photon vector and Bethe-Heitler loss vector
    at three redshifts, and a plain z = 1 -> 0 solve.
    """
    _prepare_reference()
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (6, 14, 8)
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"
    from prince_cr import cr_sources, photonfields
    from prince_cr.cross_sections.base import CrossSectionBase
    from prince_cr.solvers import UHECRPropagationSolverETD2

    out = {}
    gil = photonfields.CIBGilmore2012()
    fra = photonfields.CIBFranceschini2008()
    for key, f in (("gilmore", gil), ("franceschini", fra)):
        out[f"{key}_z"] = np.asarray(f._z)
        out[f"{key}_log10_e"] = np.asarray(f._leps_GeV)
        out[f"{key}_log10_dnde"] = np.asarray(f._log_dnde)
        rng = np.random.default_rng(5)
        E = 10 ** rng.uniform(f._leps_GeV[0] - 0.3, f._leps_GeV[-1] + 0.3, 400)
        E[:3] = 10 ** np.asarray(f._leps_GeV[[0, 7, -1]])   # table nodes and the ends
        zs = np.concatenate([rng.uniform(0.0, f._z[-1] + 0.5, 8), [0.0, f._z[3], f._z[-1]]])
        out[f"{key}_E"] = E
        out[f"{key}_zs"] = zs
        out[f"{key}_density"] = np.stack([f.get_photon_density(E, zz) for zz in zs])
    field = photonfields.CombinedPhotonField([photonfields.CMBPhotonSpectrum, photonfields.CIBGilmore2012])
    run = build(config, CrossSectionBase, photon_field=field)
    run.backend.xs_dtype = "float64"
    ir = run.int_rates
    out["species"] = np.array(run.spec_man.known_species, dtype=np.int64)
    out["cr_grid"] = np.array(config.cosmic_ray_grid, dtype=np.float64)
    out["ph_grid"] = np.array(config.photon_grid, dtype=np.float64)
    out["batch_matrix"] = np.asarray(ir._batch_matrix, dtype=np.float64)
    out["batch_rows"] = np.asarray(ir._batch_rows, dtype=np.int64)
    out["batch_cols"] = np.asarray(ir._batch_cols, dtype=np.int64)
    for zz in (0.0, 0.5, 1.0):
        tag = str(zz).replace(".", "p")
        out[f"photon_vector_z{tag}"] = ir.photon_vector(zz)
        out[f"kappa_pair_z{tag}"] = run.pair_loss_rates_grid.loss_vector(zz)
    eq = {int(p): (2.0, 1e10, 1.0) for p in run.spec_man.known_species}
    ir._sf_off_kernel = None
    s = UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
    s.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=eq))
    s.solve(dz=1e-3)
    out["state_ebl"] = np.asarray(s.state)
    path = os.path.join(HERE, "light_network_ebl.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_kernel():
    """The reference's fold-kernel construction inputs, as a channel spec.

    Samples the light network's response increments exactly as
    ``PhotoNuclearInteractionRate._init_matrices`` does (its fast path: the
    response-integral operator for the 1-D increments, the stacked bilinear
    antiderivative for the 2-D ones), walks its channel loop with the same
    branch conditions, and records the result as a
    ``prince_b200.kernel_build.KernelSpec``.  The spec, expanded, must equal the
    reference's own ``_batch_matrix`` bit for bit (checked here).
    """
    _prepare_reference()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (6, 14, 8)
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"
    import itertools

    import prince_cr.interaction_rates as IR
    from prince_cr.cross_sections.base import CrossSectionBase
    from prince_cr.data import PRINCE_UNITS
    from prince_cr.util import is_nucleus
    from prince_b200.kernel_build import SpecBuilder, cut_pairs

    run = build(config, CrossSectionBase)
    ir = run.int_rates
    resp = ir.cross_sections.resp
    m_pr = PRINCE_UNITS.m_proton
    ecr, bcr, bph = ir.e_cosmicray.grid, ir.e_cosmicray.bins, ir.e_photon.bins
    dcr, dph = ir.e_cosmicray.d, ir.e_photon.d
    log_step = np.log10(ecr[1] / ecr[0])
    y_grid = ecr[0] * bph[0] / m_pr * 10 ** (np.arange(dcr + dph) * log_step)
    x_grid = bcr[0] / ecr[0] * 10 ** ((np.arange(2 * dcr) - (dcr - 1)) * log_step)
    M = IR._response_integral_operator(resp.response_ygrid, y_grid)
    dRn = np.diff(resp.nonel_f_stack @ M.T, axis=1)
    nonel_dR = {mo: dRn[i] for i, mo in enumerate(resp.nonel_keys)}
    dRi = np.diff(resp.incl_f_stack @ M.T, axis=1)
    incl_dR = {key: dRi[i] for i, key in enumerate(resp.incl_keys)}
    Y2d, X2d = np.meshgrid(y_grid, x_grid, indexing="ij")
    keys = resp.incl_diff_integral_keys
    R_stack = resp.incl_diff_integral_stack_intp.ev(X2d.ravel(), Y2d.ravel()).reshape(*Y2d.shape, len(keys))
    ddR_stack = R_stack[1:, 1:, :] - R_stack[1:, :-1, :] - R_stack[:-1, 1:, :] + R_stack[:-1, :-1, :]
    diff_ddR = {key: ddR_stack[..., i] for i, key in enumerate(keys)}
    assert len(keys) == len(resp.incl_diff_intp_integral)

    sm = run.spec_man
    sref = sm.pdgid2sref
    sb = SpecBuilder(dcr, dph, m_pr / ecr, ir.e_cosmicray.widths)
    bc_set = ir.cross_sections.known_bc_channels_set
    diff_set = ir.cross_sections.known_diff_channels_set
    rev = sm.known_species[::-1]
    for moid, daid in itertools.product(rev, rev):
        if not is_nucleus(moid):
            continue
        has_nonel = (moid == daid) and (moid in nonel_dR)
        in_bc, in_diff = (moid, daid) in bc_set, (moid, daid) in diff_set
        nonel = sb.response(nonel_dR[moid], key=("nonel", moid)) if has_nonel else -1
        if in_bc or (has_nonel and not in_diff):
            incl = sb.response(incl_dR[(moid, daid)]) if (moid, daid) in incl_dR else -1
            sb.bc(incl, nonel, sref[daid].lidx(), sref[moid].lidx())
        elif in_diff:
            cut = config.x_cut_proton if daid == 2212 else config.x_cut
            ki, kd = cut_pairs(bcr, ecr, cut)
            if ki.size:
                sb.diff(ki, kd, sref[daid].lidx(), sref[moid].lidx(), nonel=nonel, table=diff_ddR[(moid, daid)])
    spec = sb.spec()
    bm = spec.materialize()
    order = np.lexsort((spec.cols, spec.rows))
    assert np.array_equal(spec.rows[order], ir._batch_rows) and np.array_equal(spec.cols[order], ir._batch_cols)
    assert np.array_equal(bm[order], ir._batch_matrix), "the spec does not reproduce the reference kernel"
    out = dict(d=spec.d, dph=spec.dph, f_mo=spec.f_mo, dE=spec.dE, resp=spec.resp, ddr=spec.ddr,
               sep_a=spec.sep_a, sep_b=spec.sep_b, channels=spec.channels, rows=spec.rows, cols=spec.cols,
               chan=spec.chan)
    path = os.path.join(HERE, "kernel_spec_light.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes;", spec.channels.shape[0], "channels,", spec.n_rows, "rows")


def main_cascade():
    """The reference's kinetic EM-cascade transfer on a small EM grid.

    ``kinetic_cascade_transfer_batched`` (its FP64 iteration) for CMB + the
    synthetic 40 K grey-body CIB of ``prince_b200.photonfields``, a 40-bin
    grid from 1e-3 to 1e14 GeV and three redshifts, per-step escape for
    dz = 1e-3.  Records the inputs and ``(T_gamma, T_electron)`` per z.
    """
    _prepare_reference()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import prince_cr.config as config

    config.debug_level = 0
    config.linear_algebra_backend = "scipy"
    from prince_cr.cascade.cascade import kinetic_cascade_transfer_batched
    from prince_b200 import photonfields as pf
    from prince_b200.data import EnergyGrid

    grid = EnergyGrid(-3, 14, 40 / 17)
    E = grid.grid
    zs = [0.0, 0.37, 1.0]
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])
    out = {"E": E, "grid": np.array([-3.0, 14.0, 40 / 17]), "zs": np.array(zs), "dz": np.array(1e-3)}
    Ts = kinetic_cascade_transfer_batched(E, zs, field, dz=1e-3, iter_dtype="float64")
    out["T_gamma"] = np.stack([t[0] for t in Ts])
    out["T_electron"] = np.stack([t[1] for t in Ts])
    # the Bethe-Heitler e+- pair shape as the solver builds it (propagation.py:573-618):
    # e+- on this EM grid from nucleons on a 24-bin nucleon grid, 40 target energies
    from prince_cr.cascade.bethe_heitler import bh_pair_shape_matrix
    Ep = EnergyGrid(8, 12, 6).grid
    eps = np.logspace(-12.5, -7.0, 40)
    out["bh_E_p"] = Ep
    out["bh_eps"] = eps
    Rs = []
    for zz in zs:
        n_eps = np.asarray(field.get_photon_density(eps, zz), dtype="double")
        n_eps = np.where(np.isfinite(n_eps) & (n_eps > 0), n_eps, 0.0)
        Rs.append(bh_pair_shape_matrix(E, Ep, eps, n_eps))
    out["R_BH"] = np.stack(Rs)
    path = os.path.join(HERE, "em_cascade_transfer.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main_cascade_128():
    """The reference's kinetic transfer on the 128-bin EM grid of the coupled-EM
    workload (1e-3 to 1e14 GeV), CMB + the synthetic grey-body CIB, five
    redshifts up to z = 4, per-step escape at dz = 1e-3, FP64 iteration; and its
    Bethe-Heitler shape on that grid against the 96-bin nuclear grid."""
    _prepare_reference()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import prince_cr.config as config

    config.debug_level = 0
    config.linear_algebra_backend = "scipy"
    from prince_cr.cascade.cascade import kinetic_cascade_transfer_batched
    from prince_cr.cascade.bethe_heitler import bh_pair_shape_matrix
    from prince_b200 import photonfields as pf
    from prince_b200.data import EnergyGrid

    E = EnergyGrid(-3, 14, 128 / 17).grid
    Ep = EnergyGrid(5, 14, 96 / 9).grid
    zs = [0.0, 0.5, 1.0, 2.0, 4.0]
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])
    Ts = kinetic_cascade_transfer_batched(E, zs, field, dz=1e-3, iter_dtype="float64")
    eps = np.logspace(-12.5, -7.0, 40)
    Rs = []
    for zz in zs:
        n_eps = np.asarray(field.get_photon_density(eps, zz), dtype="double")
        n_eps = np.where(np.isfinite(n_eps) & (n_eps > 0), n_eps, 0.0)
        Rs.append(bh_pair_shape_matrix(E, Ep, eps, n_eps))
    out = {"E": E, "E_p": Ep, "zs": np.array(zs), "dz": np.array(1e-3), "bh_eps": eps,
           "T_gamma": np.stack([t[0] for t in Ts]), "T_electron": np.stack([t[1] for t in Ts]),
           "R_BH": np.stack(Rs)}
    path = os.path.join(HERE, "em_cascade_transfer_128.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if "--em-decoupled" in sys.argv:
        main_em_decoupled()
    elif "--em" in sys.argv:
        main_em()
    elif "--groups" in sys.argv:
        main_groups()
    elif "--ebl" in sys.argv:
        main_ebl()
    elif "--kernel" in sys.argv:
        main_kernel()
    elif "--cascade-128" in sys.argv:
        main_cascade_128()
    elif "--cascade" in sys.argv:
        main_cascade()
    else:
        main()
