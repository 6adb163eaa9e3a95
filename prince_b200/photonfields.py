"""Target photon fields ``n(E, z)`` in 1/(GeV cm^3).

The classes keep the reference's names and ``get_photon_density(E, z)``
interface (``src/prince_cr/photonfields.py:16-127``).  Every analytic field
here also describes itself to the device through ``device_components()``:
a list of ``(kind, p0, p1, p2)`` tuples that the CUDA photon-density
evaluator sums.  The device evaluates the same expression in the same
order, so the per-window photon vectors and the Bethe-Heitler loss
integrand agree with the host formula to the last bits of ``exp``.

Tabulated EBL models are not describable on the device yet; passing one to
the GPU solver raises ``NotImplementedError`` rather than evaluating the
field on the host.

Kinds (mirrored in ``prince_b200/csrc/prince_b200.cu``):

* ``PF_CMB`` (0): ``((p0 (1+z)^2) Ered^2) / (exp(Ered/p1) - 1)`` with
  ``Ered = E/(1+z)``, zero where ``Ered/p1 >= 709``.
* ``PF_FLAT`` (1): ``(1+z)^2 * p0``.
* ``PF_MBB`` (2): ``((p0 (1+z)^2) Ered^p2) / (exp(Ered/p1) - 1)``, zero
  where ``Ered/p1 >= 709`` -- a modified black body (grey body).
"""

from __future__ import annotations

from abc import abstractmethod

import numpy as np

from . import constants as C

PF_CMB = 0
PF_FLAT = 1
PF_MBB = 2


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


def device_components(field):
    """Device description of ``field`` (this package's classes, or the reference's
    analytic ``CMBPhotonSpectrum`` / ``FlatPhotonSpectrum`` / ``CombinedPhotonField``
    matched by class name).  Raises ``NotImplementedError`` for anything else.
    """
    if hasattr(field, "device_components"):
        return field.device_components()
    name = type(field).__name__
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
