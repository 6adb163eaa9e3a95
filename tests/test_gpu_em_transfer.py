"""The kinetic EM-cascade transfer and the Bethe-Heitler pair shape built on the device (needs a B200).

``pb_em_transfer`` against PriNCe's own ``kinetic_cascade_transfer_batched``
(FP64 iteration; ``tests/golden/em_cascade_transfer.npz``) and against the CPU
restatement on a 128-bin EM grid (1e-3 to 1e14 GeV) at five redshifts up to
z = 4, CMB + the synthetic grey-body CIB; ``pb_bh_shape`` against PriNCe's own
``bh_pair_shape_matrix`` (the same fixture) and the restatement.
"""

import os

import numpy as np
import pytest

from golden_io import GOLDEN
from oracle import em_cascade as EC

pytestmark = pytest.mark.gpu


def _field():
    from prince_b200 import photonfields as pf
    return pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])


def _close(dev, ref):
    assert np.isfinite(dev).all() and np.isfinite(ref).all()
    scale = np.abs(ref).max()
    assert np.array_equal(np.abs(dev) > 1e-12 * scale, np.abs(ref) > 1e-12 * scale)
    np.testing.assert_allclose(dev, ref, rtol=1e-9, atol=1e-12 * scale)


def test_device_transfer_matches_the_reference():
    from prince_b200 import _lib
    from prince_b200.em_cascade import kinetic_transfer
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer.npz"))
    ctx = _lib.Context(0)
    Tg, Te, passes = kinetic_transfer(ctx, _field(), z["E"], z["zs"], float(z["dz"]))
    assert 0 < passes < 4000
    for i in range(len(z["zs"])):
        _close(Tg[i], z["T_gamma"][i])
        _close(Te[i], z["T_electron"][i])


def test_device_transfer_on_the_128_bin_grid_matches_the_restatement():
    from prince_b200 import _lib
    from prince_b200.data import EnergyGrid
    from prince_b200.em_cascade import kinetic_transfer
    E = EnergyGrid(-3, 14, 128 / 17).grid
    assert E.size == 128
    zs = [0.0, 0.5, 1.0, 2.0, 4.0]
    ctx = _lib.Context(0)
    Tg, Te, passes = kinetic_transfer(ctx, _field(), E, zs, 1e-3)
    ref = EC.transfer(E, zs, _field(), 1e-3)
    for i, (tg, te) in enumerate(ref):
        _close(Tg[i], tg)
        _close(Te[i], te)
    # energy conservation of the photon transfer (to the convergence tolerance)
    dE = np.gradient(E)
    for i in range(len(zs)):
        ratio = ((E * dE) @ Tg[i]) / (E * dE)
        assert np.all(np.abs(ratio - 1.0) < 2e-3)


def test_device_bh_shape_matches_the_reference():
    from prince_b200 import _lib
    from prince_b200.em_cascade import bh_shape, bh_target_grid
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer.npz"))
    assert np.array_equal(bh_target_grid(), z["bh_eps"])
    ctx = _lib.Context(0)
    R = bh_shape(ctx, _field(), z["E"], z["bh_E_p"], z["zs"])
    assert R.shape == z["R_BH"].shape
    for i in range(len(z["zs"])):
        _close(R[i], z["R_BH"][i])
        # the pair carries the nucleon energy
        carried = 2.0 * np.trapezoid(z["E"][:, None] * R[i], z["E"], axis=0)
        good = carried > 0
        np.testing.assert_allclose(carried[good], z["bh_E_p"][good], rtol=1e-12)


def test_device_bh_shape_on_a_square_grid_matches_the_restatement():
    from prince_b200 import _lib
    from prince_b200.data import EnergyGrid
    from prince_b200.em_cascade import bh_shape, bh_target_grid
    E = EnergyGrid(3, 14, 8).grid
    zs = [0.0, 1.5, 4.0]
    ctx = _lib.Context(0)
    R = bh_shape(ctx, _field(), E, E, zs)
    eps = bh_target_grid()
    for i, zz in enumerate(zs):
        n = np.asarray(_field().get_photon_density(eps, zz))
        n = np.where(np.isfinite(n) & (n > 0), n, 0.0)
        _close(R[i], EC.bh_shape(E, E, eps, n))


def test_device_transfer_and_bh_shape_match_the_reference_on_the_128_bin_grid():
    """The coupled-EM workload's 128-bin EM grid, five redshifts up to z = 4,
    against the reference's own transfer and Bethe-Heitler shape
    (``em_cascade_transfer_128.npz``; e+- on the EM grid, nucleons on the
    96-bin nuclear grid)."""
    from prince_b200 import _lib
    from prince_b200.em_cascade import bh_shape, kinetic_transfer
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer_128.npz"))
    ctx = _lib.Context(0)
    Tg, Te, passes = kinetic_transfer(ctx, _field(), z["E"], z["zs"], float(z["dz"]))
    for i in range(len(z["zs"])):
        _close(Tg[i], z["T_gamma"][i])
        _close(Te[i], z["T_electron"][i])
    R = bh_shape(ctx, _field(), z["E"], z["E_p"], z["zs"])
    for i in range(len(z["zs"])):
        _close(R[i], z["R_BH"][i])


def test_device_transfer_on_a_tabulated_ebl_matches_the_restatement():
    """The cascade transfer and the Bethe-Heitler shape on CMB + the Gilmore (2012)
    EBL table (the device's log-log table evaluation) against the restatement,
    which evaluates the same table on the host."""
    from golden_io import light_network_ebl
    from prince_b200 import _lib
    from prince_b200 import photonfields as pf
    from prince_b200.data import EnergyGrid
    from prince_b200.em_cascade import bh_shape, bh_target_grid, kinetic_transfer
    _, _, ebl = light_network_ebl()
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), ebl])
    E = EnergyGrid(-3, 14, 40 / 17).grid
    zs = [0.1, 1.5]
    ctx = _lib.Context(0)
    Tg, Te, _ = kinetic_transfer(ctx, field, E, zs, 1e-3)
    ref = EC.transfer(E, zs, field, 1e-3)
    for i, (tg, te) in enumerate(ref):
        _close(Tg[i], tg)
        _close(Te[i], te)
    Ep = EnergyGrid(8, 12, 6).grid
    R = bh_shape(ctx, field, E, Ep, zs)
    eps = bh_target_grid()
    for i, zz in enumerate(zs):
        n = np.asarray(field.get_photon_density(eps, zz))
        n = np.where(np.isfinite(n) & (n > 0), n, 0.0)
        _close(R[i], EC.bh_shape(E, Ep, eps, n))
