"""Host-side redshift schedule of one solve.

Everything here is scalar bookkeeping evaluated in float64 with the same
expressions as the reference solver, so the device sees the identical step
sizes, window boundaries and per-step scalars:

* the z grid of ``solve`` (``src/prince_cr/solvers/propagation.py:828-832``);
* the rate-cache windows: a refresh at ``z_k`` whenever
  ``|z_k - z_current| > threshold`` (``propagation.py:1383-1387``);
* per step ``h = z[k+1] - z[k]`` (``etd2.py:509-511``), ``dl/dz(z_k)``
  (``propagation.py:360-361``), ``H(z_k) cm2sec`` (the adiabatic loss scale,
  ``interaction_rates.py:1208``) and the injection prefactor
  ``dl/dz(z_k) * 1.0 * cm2sec`` (``propagation.py:366``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import constants as C
from .cosmology import H, dldz


def z_grid(initial_z, final_z, dz):
    dz_step = -float(abs(dz))
    n_full = int(np.floor((final_z - initial_z) / dz_step))
    zg = initial_z + np.arange(n_full + 1) * dz_step
    if abs(zg[-1] - final_z) > 1e-12:
        zg = np.concatenate([zg, [final_z]])
    return zg


@dataclass
class Schedule:
    z: np.ndarray          # z grid (n_steps + 1)
    window: np.ndarray     # int32 window index of each step
    z_window: np.ndarray   # redshift of each window refresh
    h: np.ndarray
    dldz: np.ndarray
    hc: np.ndarray
    finj: np.ndarray

    @property
    def n_steps(self):
        return int(self.h.size)


def make_schedule(zg, threshold):
    zg = np.asarray(zg, dtype=np.float64)
    n_steps = zg.size - 1
    zs = zg[:-1]
    win = np.zeros(max(n_steps, 0), dtype=np.int32)
    starts = []
    cur = None
    for k in range(n_steps):
        z = zs[k]
        if cur is None or abs(z - cur) > threshold:
            cur = z
            starts.append(z)
        win[k] = len(starts) - 1
    if not starts:
        starts = [zg[0]]
    # Scalar evaluation per step: numpy's vectorised pow/sqrt paths can differ
    # from the scalar ones by an ulp, and the reference evaluates scalars.
    cm2sec = C.PRINCE_UNITS.cm2sec
    dl = np.array([dldz(z) for z in zs], dtype=np.float64)
    hc = np.array([H(z) * cm2sec for z in zs], dtype=np.float64)
    return Schedule(
        z=zg,
        window=win,
        z_window=np.asarray(starts, dtype=np.float64),
        h=zg[1:] - zg[:-1],
        dldz=dl,
        hc=hc,
        finj=np.array([d * 1.0 * cm2sec for d in dl], dtype=np.float64),
    )
