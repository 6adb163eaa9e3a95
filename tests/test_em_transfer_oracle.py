"""The CPU restatement of the kinetic EM-cascade transfer against the reference.

``tests/golden/em_cascade_transfer.npz`` holds PriNCe's own
``kinetic_cascade_transfer_batched`` output (FP64 iteration; CMB + the
synthetic grey-body CIB, a 40-bin grid from 1e-3 to 1e14 GeV, three
redshifts, per-step escape at dz = 1e-3).
"""

import os

import numpy as np

from golden_io import GOLDEN
from oracle import em_cascade as EC


def test_restated_transfer_matches_the_reference():
    from prince_b200 import photonfields as pf
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer.npz"))
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])
    Ts = EC.transfer(z["E"], list(z["zs"]), field, float(z["dz"]))
    for i, (tg, te) in enumerate(Ts):
        for mine, ref in ((tg, z["T_gamma"][i]), (te, z["T_electron"][i])):
            assert np.array_equal(mine != 0, ref != 0)
            np.testing.assert_allclose(mine, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_restated_bh_shape_matches_the_reference():
    from prince_b200 import photonfields as pf
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer.npz"))
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])
    for i, zz in enumerate(z["zs"]):
        n = np.asarray(field.get_photon_density(z["bh_eps"], zz))
        n = np.where(np.isfinite(n) & (n > 0), n, 0.0)
        R = EC.bh_shape(z["E"], z["bh_E_p"], z["bh_eps"], n)
        ref = z["R_BH"][i]
        assert np.array_equal(R != 0, ref != 0)
        np.testing.assert_allclose(R, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_restated_transfer_on_the_128_bin_grid():
    """The transfer on the coupled-EM workload's 128-bin EM grid (1e-3 to 1e14
    GeV), five redshifts up to z = 4, against ``em_cascade_transfer_128.npz``
    (its Bethe-Heitler shapes are checked against the device)."""
    from prince_b200 import photonfields as pf
    z = np.load(os.path.join(GOLDEN, "em_cascade_transfer_128.npz"))
    field = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])
    Ts = EC.transfer(z["E"], list(z["zs"]), field, float(z["dz"]))
    for i, (tg, te) in enumerate(Ts):
        for mine, ref in ((tg, z["T_gamma"][i]), (te, z["T_electron"][i])):
            assert np.isfinite(mine).all()
            assert np.array_equal(mine != 0, ref != 0)
            np.testing.assert_allclose(mine, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
