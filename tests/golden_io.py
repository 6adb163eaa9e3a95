"""Load the golden fixtures produced by ``tests/golden/make_golden.py``.

``light_network()`` returns the fixture arrays and a ``prince_b200`` run
built from the fixture's own fold kernel, grids and species, plus a source
factory that rebuilds each recorded source with ``prince_b200.cr_sources``.
"""

from __future__ import annotations

import ast
import os

import numpy as np

from prince_b200 import cr_sources, photonfields
from prince_b200.run import FixedKernelModel, PriNCeRun

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def light_network():
    z = dict(np.load(os.path.join(GOLDEN, "light_network.npz")))
    model = FixedKernelModel(z["species"], z["batch_matrix"], z["batch_rows"], z["batch_cols"])
    run = PriNCeRun(model, photonfields.CMBPhotonSpectrum(),
                    cosmic_ray_grid=tuple(z["cr_grid"]), photon_grid=tuple(z["ph_grid"]),
                    max_mass=4)

    def source(key):
        kind = str(z[f"src_{key}_kind"])
        params = ast.literal_eval(str(z[f"src_{key}_params"]))
        m = ast.literal_eval(str(z[f"src_{key}_m"]))
        zmax = float(z[f"src_{key}_zmax"])
        cls = getattr(cr_sources, kind)
        return cls(run, norm=float(z[f"src_{key}_norm"]), params=params, m=m,
                   z_max=None if not np.isfinite(zmax) else zmax)

    return z, run, source


def rel_err_on_support(x, ref, species_blocks, floor=1e-20):
    """Max relative error over bins whose |ref| exceeds ``floor`` x the species max
    (infinite when either side holds a non-finite value)."""
    if not (np.isfinite(np.asarray(x)).all() and np.isfinite(np.asarray(ref)).all()):
        return np.inf
    worst = 0.0
    for sl in species_blocks:
        r = ref[sl]
        if r.ndim == 1:
            r = r[:, None]
            v = x[sl][:, None]
        else:
            v = x[sl]
        for k in range(r.shape[1]):
            rk = r[:, k]
            m = np.abs(rk).max()
            if m == 0:
                if np.abs(v[:, k]).max() != 0:
                    return np.inf
                continue
            mask = np.abs(rk) > floor * m
            e = np.abs(v[mask, k] - rk[mask]) / np.abs(rk[mask])
            if e.size:
                worst = max(worst, float(e.max()))
    return worst


def local_scale_check(x, ref, species_blocks, tol=1e-10, floor=1e-20):
    """Per-bin parity that tolerates zero crossings of oscillating spectra.

    On the support (``ref > floor`` x the species maximum) every bin is
    measured twice: strictly, ``|x - ref| / |ref|``, and against its local
    magnitude, ``|x - ref| / max(|ref|)`` over the bin and its two neighbours.
    Returns ``(worst local error, bins whose strict error exceeds tol, bins on
    the support)``.
    """
    if not (np.isfinite(np.asarray(x)).all() and np.isfinite(np.asarray(ref)).all()):
        return np.inf, -1, 0
    worst, above, total = 0.0, 0, 0
    for sl in species_blocks:
        r, v = ref[sl], x[sl]
        if r.ndim == 1:
            r, v = r[:, None], v[:, None]
        a = np.abs(r)
        local = a.copy()
        local[1:] = np.maximum(local[1:], a[:-1])
        local[:-1] = np.maximum(local[:-1], a[1:])
        for k in range(r.shape[1]):
            m = a[:, k].max()
            if m == 0:
                continue
            sel = r[:, k] > floor * m
            err = np.abs(v[sel, k] - r[sel, k])
            total += int(sel.sum())
            above += int(np.count_nonzero(err > tol * a[sel, k]))
            if err.size:
                worst = max(worst, float(np.max(err / local[sel, k])))
    return worst, above, total


def light_network_em():
    """The EM-cascade fixture: run (gamma, e+- on the shared grid) and the
    synthetic per-window transfer used by the reference run."""
    from prince_b200 import synth
    from prince_b200.data import EnergyGrid

    z = dict(np.load(os.path.join(GOLDEN, "light_network_em.npz")))
    model = FixedKernelModel(z["species"], z["batch_matrix"], z["batch_rows"], z["batch_cols"])
    grid = EnergyGrid(*tuple(z["cr_grid"]))

    def em(zz):
        return synth.em_cascade_matrices(grid, grid, float(zz))

    run = PriNCeRun(model, photonfields.CMBPhotonSpectrum(), cosmic_ray_grid=tuple(z["cr_grid"]),
                    photon_grid=tuple(z["ph_grid"]), enable_em_cascade=True, em_cascade_model=em)

    def source(key, m="flat"):
        params = ast.literal_eval(str(z[f"src_{key}"]))
        if key == "soft":
            return cr_sources.SimpleSource(run, norm=1.0, params=params, m=("simple", 2.0))
        return cr_sources.RigdityCutoffSource(run, norm=1.0, params=params)

    return z, run, em, source


def light_network_em_decoupled():
    """The decoupled-grid EM fixture: gamma and e+- on the reference's EM grid,
    the nuclei on the nuclear grid, and the synthetic per-window transfer."""
    from prince_b200 import synth
    from prince_b200.data import EnergyGrid

    z = dict(np.load(os.path.join(GOLDEN, "light_network_em_decoupled.npz")))
    model = FixedKernelModel(z["species"], z["batch_matrix"], z["batch_rows"], z["batch_cols"])
    grid = EnergyGrid(*tuple(z["cr_grid"]))
    egrid = EnergyGrid(*tuple(z["em_grid"]))

    def em(zz):
        return synth.em_cascade_matrices(egrid, grid, float(zz))

    run = PriNCeRun(model, photonfields.CMBPhotonSpectrum(), cosmic_ray_grid=tuple(z["cr_grid"]),
                    photon_grid=tuple(z["ph_grid"]), enable_em_cascade=True, em_cascade_model=em,
                    enable_em_decoupled_grid=True, em_grid=tuple(z["em_grid"]))

    def source(key):
        params = ast.literal_eval(str(z[f"src_{key}"]))
        if key == "soft":
            return cr_sources.SimpleSource(run, norm=1.0, params=params, m=("simple", 2.0))
        return cr_sources.RigdityCutoffSource(run, norm=1.0, params=params)

    return z, run, em, source


def light_network_ebl():
    """The light network in CMB + the tabulated Gilmore (2012) EBL: fixture arrays,
    the run (this package's classes on the fixture's kernel and EBL table) and
    the EBL field alone."""
    z = dict(np.load(os.path.join(GOLDEN, "light_network_ebl.npz")))
    model = FixedKernelModel(z["species"], z["batch_matrix"], z["batch_rows"], z["batch_cols"])
    ebl = photonfields.TabulatedPhotonField(z["gilmore_z"], z["gilmore_log10_e"], z["gilmore_log10_dnde"])
    field = photonfields.CombinedPhotonField([photonfields.CMBPhotonSpectrum(), ebl])
    run = PriNCeRun(model, field, cosmic_ray_grid=tuple(z["cr_grid"]), photon_grid=tuple(z["ph_grid"]),
                    max_mass=4)
    return z, run, ebl
