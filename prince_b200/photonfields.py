"""Target photon fields ``n(E, z)`` in 1/(GeV cm^3).

The classes keep the reference's names and ``get_photon_density(E, z)``
interface (``src/prince_cr/photonfields.py:16-127``).  Every analytic field
here also describes itself to the device through ``device_components()``:
a list of ``(kind, p0, p1, p2)`` tuples that the CUDA photon-density
evaluator sums.  The device evaluates the same expression in the same
order, so the per-window photon vectors and the Bethe-Heitler loss
integrand agree with the host formula to the last bits of ``exp``.

Tabulated fields (``TabulatedPhotonField``: the corrected EBL tables of
Gilmore 2012 and Franceschini 2008) are evaluated on the device from their
table; a field the device cannot describe (the legacy spline EBLs) raises
``NotImplementedError`` rather than evaluating it on the host.

Kinds (mirrored in ``prince_b200/csrc/prince_b200.cu``):

* ``PF_CMB`` (0): ``((p0 (1+z)^2) Ered^2) / (exp(Ered/p1) - 1)`` with
  ``Ered = E/(1+z)``, zero where ``Ered/p1 >= 709``.
* ``PF_FLAT`` (1): ``(1+z)^2 * p0``.
* ``PF_MBB`` (2): ``((p0 (1+z)^2) Ered^p2) / (exp(Ered/p1) - 1)``, zero
  where ``Ered/p1 >= 709`` -- a modified black body (grey body).
* ``PF_TABLE`` (3): a tabulated field, ``10^v`` with ``v`` the bilinear
  interpolation in ``(z, log10 E)`` of a table of ``log10 dn/de``, zero
  outside the table (the corrected tabulated EBL models of the reference,
  ``photonfields.py:227-345``).  At most one table per field.
"""

from __future__ import annotations

from abc import abstractmethod

import numpy as np

from . import constants as C

PF_CMB = 0
PF_FLAT = 1
PF_MBB = 2
PF_TABLE = 3


class PhotonField:
    """Base class: ``get_photon_density(E, z)`` and ``device_components()``."""

    @abstractmethod
    def get_photon_density(self, E, z):
        raise Exception("Base class method called accidentally.")

    def device_components(self):
        raise NotImplementedError(
            f"{type(self).__name__} has no device description; the b200 backend "
            "evaluates photon fields on the GPU and supports the analytic fields "
            "(CMBPhotonSpectrum, FlatPhotonSpectrum, ModifiedBlackBodyCIB and "
            "their CombinedPhotonField / ScaledPhotonField wrappers)."
        )


class CombinedPhotonField(PhotonField):
    """Sum of several fields; entries are classes or ``(class, *args)`` tuples."""

    def __init__(self, list_of_classes_and_args):
        self.model_list = []
        for arg in list_of_classes_and_args:
            if isinstance(arg, PhotonField):
                self.model_list.append(arg)
            elif type(arg) in (tuple, list):
                self.model_list.append(arg[0](*arg[1:]))
            else:
                self.model_list.append(arg())

    def add_model(self, model_class, model_args=()):
        self.model_list.append(model_class(*model_args))

    def get_photon_density(self, E, z):
        E = np.atleast_1d(E)
        return np.sum([m.get_photon_density(E, z) for m in self.model_list], axis=0)

    def device_components(self):
        out = []
        for m in self.model_list:
            out.extend(m.device_components())
        return out


class FlatPhotonSpectrum(PhotonField):
    """Constant density ``1e12 (1+z)^2`` (a test field)."""

    def get_photon_density(self, E, z):
        nlocal = np.ones_like(E, dtype="double") * 1e12
        return (1.0 + z) ** 2 * nlocal

    def device_components(self):
        return [(PF_FLAT, 1e12, 0.0, 0.0)]


def _grey_body(E, z, pref, kT, power):
    Ered = E / (1.0 + z)
    eratio = Ered / kT
    exp_range = eratio < 709.0
    nlocal = np.zeros_like(Ered)
    pz = pref * (1.0 + z) ** 2
    if power == 2.0:
        num = pz * Ered[exp_range] ** 2
    else:
        num = pz * Ered[exp_range] ** power
    nlocal[exp_range] = num / (np.exp(eratio[exp_range]) - 1.0)
    return nlocal


class CMBPhotonSpectrum(PhotonField):
    """Black-body CMB with T = 2.725 (1+z) K, ``n(E,z) = (1+z)^2 n0(E/(1+z))``."""

    pref = 1.31868e40  # 1/pi^2/(hbar c)^3 in GeV^-3 cm^-3

    def get_photon_density(self, E, z):
        return _grey_body(np.asarray(E, dtype=np.float64), z, self.pref, C.E_CMB, 2.0)

    def device_components(self):
        return [(PF_CMB, self.pref, C.E_CMB, 2.0)]


class ModifiedBlackBodyCIB(PhotonField):
    """Synthetic cosmic infrared background: a grey body ``E^(2+beta)/(e^(E/kT)-1)``.

    Defaults: T = 40 K, emissivity index beta = 1.5, normalised so that its
    photon number density at z = 0 is ``number_fraction`` (1e-3) of the
    CMB's.  Redshift scaling follows the CMB convention.
    """

    def __init__(self, T_K=40.0, beta=1.5, number_fraction=1e-3):
        from scipy.special import gamma as _gamma, zeta as _zeta

        self.kT = C.E_CMB * (T_K / 2.725)
        self.power = 2.0 + beta
        n_cmb = CMBPhotonSpectrum.pref * C.E_CMB ** 3 * 2.0 * _zeta(3.0)
        shape_int = self.kT ** (self.power + 1.0) * _gamma(self.power + 1.0) * _zeta(self.power + 1.0)
        self.pref = number_fraction * n_cmb / shape_int

    def get_photon_density(self, E, z):
        return _grey_body(np.asarray(E, dtype=np.float64), z, self.pref, self.kT, self.power)

    def device_components(self):
        return [(PF_MBB, self.pref, self.kT, self.power)]


class ScaledPhotonField(PhotonField):
    """``scale * field`` -- the shared photon-density scale of the gradient workload."""

    def __init__(self, field, scale=1.0):
        self.field = field
        self.scale = float(scale)

    def get_photon_density(self, E, z):
        return self.scale * self.field.get_photon_density(E, z)

    def device_components(self):
        return self.field.device_components()


class TabulatedPhotonField(PhotonField):
    """``n(E, z) = 10^v`` with ``v`` linear in ``(z, log10 E)`` between the
    table's nodes and the field zero outside the table: the log-log
    interpolation of the reference's corrected EBL classes
    (``photonfields.py:227-345``, a ``RegularGridInterpolator`` with
    ``method="linear"`` and ``fill_value=-inf``).

    ``z`` (nz, increasing), ``log10_e`` (ne, log10 E/GeV, increasing) and
    ``log10_dnde`` (nz x ne, log10 of dn/de in GeV^-1 cm^-3).
    """

    def __init__(self, z, log10_e, log10_dnde):
        from scipy.interpolate import RegularGridInterpolator

        self.table_z = np.ascontiguousarray(z, dtype=np.float64)
        self.table_log10_e = np.ascontiguousarray(log10_e, dtype=np.float64)
        self.table_log10_dnde = np.ascontiguousarray(log10_dnde, dtype=np.float64)
        if self.table_log10_dnde.shape != (self.table_z.size, self.table_log10_e.size):
            raise ValueError("log10_dnde must be (len(z), len(log10_e))")
        self._rgi = RegularGridInterpolator((self.table_z, self.table_log10_e), self.table_log10_dnde,
                                            method="linear", bounds_error=False, fill_value=-np.inf)

    def get_photon_density(self, E, z):
        E = np.atleast_1d(np.asarray(E, dtype=np.float64))
        pts = np.column_stack([np.full(E.size, float(z)), np.log10(E.reshape(-1))])
        return (10.0 ** self._rgi(pts)).reshape(E.shape)

    def device_components(self):
        return [(PF_TABLE, 0.0, 0.0, 0.0)]

    def device_table(self):
        return self.table_z, self.table_log10_e, self.table_log10_dnde


def _ebl_table_file(table_file, name):
    import os

    if table_file is None:
        base = os.environ.get("PRINCE_DATA_DIR")
        if base is None:
            raise FileNotFoundError(
                f"{name}: pass table_file=<path to {name}> (the reference ships it in its data "
                "directory) or set PRINCE_DATA_DIR")
        table_file = os.path.join(base, name)
    return table_file


class CIBGilmore2012(TabulatedPhotonField):
    """Gilmore et al. (2012) EBL from the published flux tables, log-log
    interpolated (the reference's ``CIBGilmore2012``, ``photonfields.py:227-298``).

    ``table_file`` is the reference's ``gilmore2012_ebl_tables.npz`` (keys
    ``z``, ``log10_eps_eV``, ``log10_eps_dndeps_cm3_<model>``); ``model`` is
    ``"fiducial"`` or ``"fixed"``.
    """

    def __init__(self, model="fiducial", simple_scaling=False, table_file=None):
        if model not in ("fixed", "fiducial"):
            raise ValueError(f"model must be 'fiducial' or 'fixed', got {model!r}")
        f = np.load(_ebl_table_file(table_file, "gilmore2012_ebl_tables.npz"))
        le = f["log10_eps_eV"] - 9.0
        super().__init__(f["z"], le, f["log10_eps_dndeps_cm3_" + model] - le[None, :])


class CIBFranceschini2008(TabulatedPhotonField):
    """Franceschini et al. (2008) EBL from the paper's tables, log-log
    interpolated (the reference's ``CIBFranceschini2008``, ``photonfields.py:301-345``).

    ``table_file`` is the reference's ``franceschini2008_ebl_tables.npz``.
    """

    def __init__(self, simple_scaling=False, table_file=None):
        f = np.load(_ebl_table_file(table_file, "franceschini2008_ebl_tables.npz"))
        le = f["log10_eps_eV"] - 9.0
        super().__init__(f["z"], le, f["log10_eps_dndeps_cm3"] - le[None, :])


def _reference_table(field):
    """The table of the reference's own corrected EBL objects (same attributes as
    ``photonfields.py:273-283`` / ``324-334``), or ``None``."""
    if type(field).__name__ in ("CIBGilmore2012", "CIBFranceschini2008") and not hasattr(field, "device_table") \
            and getattr(field, "_fallback", None) is None and hasattr(field, "_log_dnde"):
        return (np.asarray(field._z, dtype=np.float64), np.asarray(field._leps_GeV, dtype=np.float64),
                np.asarray(field._log_dnde, dtype=np.float64))
    return None


def device_table(field):
    """The one tabulated component of ``field`` as ``(z, log10 E, log10 dn/de)``, or ``None``."""
    tables = []

    def walk(f):
        if hasattr(f, "device_table"):
            tables.append(f.device_table())
        for sub in getattr(f, "model_list", []):
            walk(sub)
        if hasattr(f, "field"):
            walk(f.field)

    walk(field)
    if _reference_table(field) is not None:
        tables.append(_reference_table(field))
    for sub in getattr(field, "model_list", []):
        if _reference_table(sub) is not None:
            tables.append(_reference_table(sub))
    if len(tables) > 1:
        raise NotImplementedError("the device evaluates at most one tabulated photon field")
    return tables[0] if tables else None


def device_components(field):
    """Device description of ``field`` (this package's classes, or the reference's
    analytic ``CMBPhotonSpectrum`` / ``FlatPhotonSpectrum`` / ``CombinedPhotonField``
    matched by class name).  Raises ``NotImplementedError`` for anything else.
    """
    if hasattr(field, "device_components"):
        return field.device_components()
    name = type(field).__name__
    if _reference_table(field) is not None:
        return [(PF_TABLE, 0.0, 0.0, 0.0)]
    if name == "CMBPhotonSpectrum":
        return [(PF_CMB, CMBPhotonSpectrum.pref, C.E_CMB, 2.0)]
    if name == "FlatPhotonSpectrum":
        return [(PF_FLAT, 1e12, 0.0, 0.0)]
    if name == "CombinedPhotonField":
        out = []
        for m in field.model_list:
            out.extend(device_components(m))
        return out
    return PhotonField.device_components(field)
