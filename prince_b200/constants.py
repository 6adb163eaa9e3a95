"""Physical units and the physics/numerics settings the ETD2 path reads.

PriNCe works in cm, s and GeV.  The unit table below is built from
``scipy.constants`` with the same expressions as the reference unit table
(``src/prince_cr/data.py:722-740``), so every derived constant (``cm2sec``,
``m_proton``, ...) is bit-identical to the reference's value.

The cosmology and grid settings mirror ``src/prince_cr/config.py:125-138``
(Hubble rate, Omega_m, Omega_Lambda, E_CMB) and ``config.py:254-257``
(redistribution cuts).  ``BackendConfig`` mirrors the per-run dispatch
handle ``config.BackendConfig`` (``config.py:370-407``); the backend name
this package registers is ``"b200"``.
"""

from __future__ import annotations

from dataclasses import dataclass
from types import SimpleNamespace
from typing import Optional

import scipy.constants as _spc

PRINCE_UNITS = SimpleNamespace(
    c=1e2 * _spc.c,
    cm2Mpc=1.0 / (_spc.parsec * _spc.mega * 1e2),
    Mpc2cm=_spc.mega * _spc.parsec * 1e2,
    m_proton=_spc.physical_constants["proton mass energy equivalent in MeV"][0] * 1e-3,
    m_electron=_spc.physical_constants["electron mass energy equivalent in MeV"][0] * 1e-3,
    r_electron=_spc.physical_constants["classical electron radius"][0] * 1e2,
    fine_structure=_spc.fine_structure,
    GeV2erg=1.0 / 624.15,
    erg2GeV=624.15,
    km2cm=1e5,
    yr2sec=_spc.year,
    Gyr2sec=_spc.giga * _spc.year,
    cm2sec=1e-2 / _spc.c,
    sec2cm=_spc.c * 1e2,
)

#: Hubble rate today in 1/s, matter and vacuum density parameters.
H_0s = 2.28475e-18
Omega_m = 0.27
Omega_Lambda = 0.73

#: CMB energy k_B * T0 in GeV (T0 = 2.725 K).
E_CMB = 2.34823e-13

#: Lower cut on x = E_daughter / E_mother for redistributed daughters, and the
#: separate cut used for proton daughters.
x_cut = 1e-4
x_cut_proton = 1e-1

#: Default redshift resolution of the rate cache (operator refresh windows).
update_rates_z_threshold = 0.01


@dataclass
class BackendConfig:
    """Per-run backend handle read by the solvers.

    ``linear_algebra_backend`` selects the implementation; this package only
    implements ``"b200"`` (hand-written sm_100a kernels).  The remaining
    knobs keep the reference's names so code written against the reference
    run object reads the same fields.
    """

    linear_algebra_backend: str = "b200"
    update_rates_z_threshold: float = update_rates_z_threshold
    cupy_dtype: str = "float64"
    xs_dtype: Optional[str] = "float64"
    use_cuda_graphs: bool = True
