"""Tabulated photon fields against the reference's corrected EBL models.

``tests/golden/light_network_ebl.npz`` (``make_golden.py --ebl``) holds the
tables of the reference's ``CIBGilmore2012`` and ``CIBFranceschini2008``,
their densities at sample points (inside, at the nodes and beyond the
table), and the photon vector, Bethe-Heitler loss vector and a plain
z = 1 -> 0 solve of the light network in CMB + Gilmore (2012).
"""

import numpy as np
import pytest

from golden_io import light_network_ebl, rel_err_on_support
from oracle import etd2_oracle as O
from prince_b200 import photonfields as pf


@pytest.fixture(scope="module")
def golden():
    return light_network_ebl()


@pytest.mark.parametrize("key", ["gilmore", "franceschini"])
def test_table_densities_match_reference(golden, key):
    z = golden[0]
    f = pf.TabulatedPhotonField(z[f"{key}_z"], z[f"{key}_log10_e"], z[f"{key}_log10_dnde"])
    got = np.stack([f.get_photon_density(z[f"{key}_E"], zz) for zz in z[f"{key}_zs"]])
    ref = z[f"{key}_density"]
    assert np.array_equal(got == 0, ref == 0)
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=0)
    assert (ref == 0).any() and (ref > 0).any()   # the samples reach beyond the table


def test_named_classes_read_the_reference_table_files(tmp_path, golden):
    z = golden[0]
    le_ev = z["gilmore_log10_e"] + 9.0
    np.savez(tmp_path / "gilmore2012_ebl_tables.npz", z=z["gilmore_z"], log10_eps_eV=le_ev,
             log10_eps_dndeps_cm3_fiducial=z["gilmore_log10_dnde"] + z["gilmore_log10_e"][None, :],
             log10_eps_dndeps_cm3_fixed=z["gilmore_log10_dnde"])
    g = pf.CIBGilmore2012(table_file=str(tmp_path / "gilmore2012_ebl_tables.npz"))
    np.testing.assert_allclose(g.table_log10_dnde, z["gilmore_log10_dnde"], rtol=1e-15, atol=1e-13)
    with pytest.raises(ValueError):
        pf.CIBGilmore2012(model="upper", table_file=str(tmp_path / "gilmore2012_ebl_tables.npz"))
    assert pf.device_components(g) == [(pf.PF_TABLE, 0.0, 0.0, 0.0)]
    comb = pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), g])
    assert [c[0] for c in pf.device_components(comb)] == [pf.PF_CMB, pf.PF_TABLE]
    assert pf.device_table(comb)[0] is g.table_z
    with pytest.raises(NotImplementedError):
        pf.device_table(pf.CombinedPhotonField([g, g]))


def test_run_photon_and_pair_vectors_match_reference(golden):
    z, run, _ = golden
    for zz in (0.0, 0.5, 1.0):
        tag = str(zz).replace(".", "p")
        np.testing.assert_allclose(run.int_rates.photon_vector(zz), z[f"photon_vector_z{tag}"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(run.pair_loss_rates_grid.loss_vector(zz), z[f"kappa_pair_z{tag}"],
                                   rtol=1e-13, atol=0)


def test_oracle_solve_in_cmb_plus_gilmore_matches_reference(golden):
    z, run, _ = golden
    from prince_b200 import cr_sources
    params = {p: (2.0, 1e10, 1.0) for p in run.spec_man.known_species}
    src = cr_sources.RigdityCutoffSource(run, norm=1.0, params=params)
    x = O.OracleSolver(run, 1.0, 0.0).solve([src], dz=1e-3)
    assert rel_err_on_support(x, z["state_ebl"], [s.sl for s in run.spec_man.species_refs]) < 1e-10
