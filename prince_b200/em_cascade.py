"""The kinetic EM-cascade transfer, built on the device.

``kinetic_transfer(ctx, field, E, zs, dz)`` returns the per-redshift photon
and electron transfer ``(T_gamma, T_electron)`` of an EM grid ``E`` on a
photon field (set on the device context ``ctx``), for per-step escape at the
step ``dz``: PriNCe's
``kinetic_cascade_transfer_batched`` (``src/prince_cr/cascade/cascade.py:444-589``)
with an FP64 iteration, computed by ``pb_em_transfer`` -- field-free
inverse-Compton, pair and gamma-gamma opacity kernels, their contractions with
the photon densities as FP64 tensor-core GEMMs, the per-redshift matrices and
the scattering iteration, all on the GPU.

``KineticCascadeModel(run, dz)`` is a run's ``em_cascade_model`` built on it:
``model(z) -> (T_gamma, T_electron, R_BH)`` with the transfer from the device
(cached per redshift; ``prefetch(zs)`` builds all windows of a solve in one
device call) and the Bethe-Heitler pair shape ``R_BH`` from ``pb_bh_shape``
(the reference solver's ``_em_bh_at``, ``src/prince_cr/solvers/propagation.py:573-618``:
40 target energies from 10^-12.5 to 10^-7 GeV, e+- on the EM species' grid --
the run's decoupled EM grid or the shared one -- and nucleons on the
cosmic-ray grid), or from a caller-supplied function.  It refuses a
transfer that is not finite (the reference's pair normalisation overflows on
EM grids whose top stops near the pair threshold).
"""

from __future__ import annotations

import numpy as np

from . import constants as C
from .cosmology import H
from .photonfields import device_components, device_table


def default_grids():
    """Target, opacity and angle grids of the reference (``cascade.py:466-468``)."""
    return np.logspace(-15, -9, 400), np.logspace(-12, -7, 256), np.linspace(-1.0, 1.0, 128)


def dl_step(zs, dz):
    """c |dz| / ((1+z) H(z)) [cm] per redshift (``cascade.py:505``)."""
    return np.array([C.PRINCE_UNITS.c * abs(dz) / ((1.0 + z) * H(z)) for z in zs])


def kinetic_transfer(ctx, field, E, zs, dz, photon_scale=1.0, **kw):
    """``(T_gamma, T_electron, passes)``: ``(n_z, n, n)`` arrays from the device."""
    eps, eps_o, mu = default_grids()
    ctx.set_photon_field(device_components(field), table=device_table(field))
    zs = np.atleast_1d(np.asarray(zs, dtype=np.float64))
    return ctx.em_transfer(np.asarray(E, dtype=np.float64), zs, dl_step(zs, dz), eps, eps_o, mu,
                           photon_scale=photon_scale, **kw)


def bh_target_grid():
    """Target photon energies of the BH pair shape (``propagation.py:592``)."""
    return np.logspace(-12.5, -7.0, 40)


def bh_shape(ctx, field, E_e, E_p, zs, e_p_min=1e5, photon_scale=1.0):
    """Device Bethe-Heitler pair shapes ``(n_z, n_e, n_p)`` on ``field``."""
    ctx.set_photon_field(device_components(field), table=device_table(field))
    return ctx.bh_shape(E_e, E_p, bh_target_grid(), zs, e_p_min=e_p_min, photon_scale=photon_scale)


class KineticCascadeModel:
    """``em_cascade_model`` of a run: the device kinetic transfer plus the BH pair shape.

    ``bh_shape(z) -> R_BH`` (n_em x n_cr), when given, replaces the device BH shape.
    """

    def __init__(self, run, dz, bh_shape=None, device=0):
        self.run = run
        self.dz = float(dz)
        self.bh_shape = bh_shape
        self.device = device
        self._cache = {}

    def prefetch(self, zs):
        from .solvers import DeviceRun

        todo = sorted({float(z) for z in zs} - set(self._cache))
        if not todo:
            return
        ctx = DeviceRun.of(self.run, self.device).ctx
        em_grid = getattr(self.run, "em_grid", None)
        E = (em_grid if em_grid is not None else self.run.cr_grid).grid
        Tg, Te, _ = kinetic_transfer(ctx, self.run.photon_field, E, todo, self.dz)
        R = (bh_shape(ctx, self.run.photon_field, E, self.run.cr_grid.grid, todo) if self.bh_shape is None
             else [self.bh_shape(z) for z in todo])
        for i, z in enumerate(todo):
            if not (np.isfinite(Tg[i]).all() and np.isfinite(Te[i]).all() and np.isfinite(R[i]).all()):
                raise FloatingPointError(
                    f"the cascade transfer at z = {z} is not finite on this EM grid (the pair-production "
                    "normalisation divides by the energy a near-threshold column carries, as the reference's "
                    "cascade.py:513-515 does, and overflows); choose a grid whose top bins lie above the pair "
                    "threshold, e.g. up to 1e14 GeV")
            self._cache[z] = (Tg[i], Te[i], R[i])

    def __call__(self, z):
        self.prefetch([z])
        return self._cache[float(z)]
