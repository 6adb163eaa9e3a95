"""The CPU oracle and the host data model against the reference's golden vectors.

The fixture ``tests/golden/light_network.npz`` was produced by PriNCe's own
``ETD2SolverCPU`` / ``MultiRHSPropagationSolverETD2`` (see
``tests/golden/make_golden.py``).  These tests pin

* the host-side inputs this package builds (coupling pattern, loss vectors,
  FD operator, injection grids) bit-for-bit or to 1e-14;
* the oracle's final states to 1e-10 relative per bin above 1e-20 of the
  species maximum (observed agreement is ~1e-15).
"""

import numpy as np
import pytest
import scipy.sparse as sp

from golden_io import light_network, rel_err_on_support
from oracle import etd2_oracle as O
from prince_b200 import operators

TOL = 1e-10


@pytest.fixture(scope="module")
def golden():
    return light_network()


def _blocks(run):
    return [s.sl for s in run.spec_man.species_refs]


def test_coupling_pattern_bit_exact(golden):
    z, run, _ = golden
    cm = run.int_rates.coupling_mat
    assert np.array_equal(cm.indptr, z["cpl_indptr"])
    assert np.array_equal(cm.indices, z["cpl_indices"])
    assert np.array_equal(run.int_rates._batch_rows, z["batch_rows"])
    assert np.array_equal(run.int_rates._batch_cols, z["batch_cols"])
    assert np.array_equal(run.int_rates._batch_matrix, z["batch_matrix"])


def test_species_order(golden):
    z, run, _ = golden
    assert run.spec_man.known_species == [int(s) for s in z["species"]]


def test_loss_inputs(golden):
    z, run, _ = golden
    pl = run.pair_loss_rates_grid
    assert np.array_equal(pl.xi, z["xi"])
    assert np.array_equal(pl.phi_xi2, z["phi_xi2"])
    assert np.array_equal(pl.scale_vec, z["pair_scale_vec"])
    assert np.array_equal(run.adia_loss_rates_grid.energy_vector, z["adia_energy"])
    np.testing.assert_allclose(pl.loss_vector(1.0), z["kappa_pair_z1"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(pl.loss_vector(0.5), z["kappa_pair_z05"], rtol=1e-14, atol=0)


def test_photon_vector(golden):
    z, run, _ = golden
    np.testing.assert_allclose(run.int_rates.photon_vector(1.0), z["photon_vector_z1"],
                               rtol=1e-15, atol=0)


@pytest.mark.parametrize("builder", ["package", "oracle"])
def test_fd_operator(golden, builder):
    z, run, _ = golden
    if builder == "package":
        D = operators.fd_loss_operator(run.cr_grid, run.spec_man.nspec)
        d, off = operators.split_diagonal(D)
    else:
        d, off = O.split(O.fd_operator(run.cr_grid, run.spec_man.nspec))
    assert np.array_equal(d, z["D_diag"])
    assert np.array_equal(off.indptr, z["D_off_indptr"])
    assert np.array_equal(off.indices, z["D_off_indices"])
    assert np.array_equal(off.data, z["D_off_data"])


@pytest.mark.parametrize("key", ["eq", "auger", "soft", "late"])
def test_injection_grids(golden, key):
    z, run, source = golden
    np.testing.assert_allclose(source(key).injection_grid, z[f"src_{key}_grid"], rtol=1e-15, atol=0)


def test_first_window_split(golden):
    z, run, source = golden
    o = O.OracleSolver(run, 1.0, 0.0)
    o.solve([source("eq")], dz=0.5)
    assert np.array_equal(o.trace.M_off_first.indptr, z["M_off_indptr"])
    assert np.array_equal(o.trace.M_off_first.indices, z["M_off_indices"])
    np.testing.assert_allclose(o.trace.M_off_first.data, z["M_off_data_z1"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(o.trace.d_M_first, z["M_diag_z1"], rtol=1e-13, atol=0)


CASES = {
    "plain": (dict(), ["eq"], 1.0, 1e-3, None),
    "no_pair": (dict(pairprod=False), ["eq"], 1.0, 1e-3, None),
    "no_adia": (dict(adiabatic=False), ["eq"], 1.0, 1e-3, None),
    "no_pdiff": (dict(partial_diff=False), ["eq"], 1.0, 1e-3, None),
    "no_photohad": (dict(photohad=False), ["eq"], 1.0, 1e-3, None),
    "two_src": (dict(), ["auger", "soft"], 1.0, 1e-3, None),
    "thr": (dict(), ["eq"], 0.5, 2e-3, 1e-3),
}


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_single_rhs(golden, case):
    z, run, source = golden
    flags, keys, zi, dz, thr = CASES[case]
    o = O.OracleSolver(run, zi, 0.0, flags=O.Flags(**flags), thr=thr)
    x = o.solve([source(k) for k in keys], dz=dz)
    err = rel_err_on_support(x, z[f"state_{case}"], _blocks(run))
    assert err < TOL, err
    if f"windows_{case}" in z:
        assert np.array_equal(np.asarray(o.trace.windows), z[f"windows_{case}"])


def test_oracle_decay(golden):
    z, run, source = golden
    n = run.dim_states
    Loff = sp.csr_matrix((z["lambda_data"], z["lambda_indices"], z["lambda_indptr"]), shape=(n, n))
    o = O.OracleSolver(run, 1.0, 0.0, decay=(z["lambda_diag"], Loff))
    x = o.solve([source("eq")])
    assert rel_err_on_support(x, z["state_decay"], _blocks(run)) < TOL


def test_oracle_multi_rhs(golden):
    z, run, source = golden
    cols = [str(c).split(",") for c in z["multi_columns"]]
    o = O.OracleSolver(run, 1.0, 0.0, K=len(cols))
    X = o.solve([[source(k) for k in c] for c in cols])
    assert rel_err_on_support(X, z["state_multi"], _blocks(run)) < TOL


def test_multi_column_equals_single(golden):
    z, run, source = golden
    ref = z["state_multi"]
    assert rel_err_on_support(ref[:, 0], z["state_plain"], _blocks(run)) < TOL


def test_constant_operator_chain(golden):
    """a -> b -> c with rates 1, 0.4 (c stable): reference integrator and closed form."""
    z, _, _ = golden
    zg = np.linspace(0.0, 6.0, 2001)
    L = sp.csr_matrix(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.4, 0.0]]))
    x = O.integrate_const([1.0, 0.0, 0.0], zg, [-1.0, -0.4, 0.0], L)
    np.testing.assert_allclose(x, z["chain3_state"], rtol=1e-13)
    t, la, lb = 6.0, 1.0, 0.4
    na = np.exp(-la * t)
    nb = la / (lb - la) * (np.exp(-la * t) - np.exp(-lb * t))
    np.testing.assert_allclose(x[:2], [na, nb], rtol=1e-6)
    np.testing.assert_allclose(x.sum(), 1.0, rtol=1e-5)  # second-order in the step


def test_single_exponential_known_answer():
    zg = np.linspace(0.0, 5.0, 1001)
    x = O.integrate_const([1.0], zg, [-1.0 / 0.7])
    np.testing.assert_allclose(x[0], np.exp(-5.0 / 0.7), rtol=1e-10)


def test_oracle_em_cascade_single_and_multi():
    """EM step hooks (BH pair injection + cascade transfer) against the reference."""
    from golden_io import light_network_em

    z, run, em, source = light_network_em()
    blocks = [s.sl for s in run.spec_man.species_refs]
    x = O.OracleSolver(run, 0.2, 0.0, em=em).solve([source("eq")], dz=1e-3)
    assert rel_err_on_support(x, z["state_em"], blocks) < TOL
    X = O.OracleSolver(run, 0.2, 0.0, K=2, em=em).solve([[source("eq")], [source("soft")]], dz=1e-3)
    assert rel_err_on_support(X, z["state_em_multi"], blocks) < TOL


def test_decoupled_em_grid_layout_matches_the_reference():
    """gamma and e+- on their own EM grid: offsets, sizes and the per-grid loss energies."""
    from golden_io import light_network_em_decoupled

    z, run, em, source = light_network_em_decoupled()
    refs = sorted(run.spec_man.species_refs, key=lambda s: s.princeidx)
    assert run.dim_states == int(z["dim_states"])
    assert [s.lidx() for s in refs] == list(z["lidx"])
    assert np.array_equal(run.adia_loss_rates_grid.energy_vector, z["adia_energy"])
    D = operators.run_fd_loss_operator(run)
    d, off = operators.split_diagonal(D)
    assert np.array_equal(d, z["D_diag"])
    assert np.array_equal(off.indptr, z["D_off_indptr"]) and np.array_equal(off.indices, z["D_off_indices"])
    assert np.array_equal(off.data, z["D_off_data"])


def test_oracle_em_cascade_on_a_decoupled_grid():
    """The EM hooks with gamma/e+- on the EM grid and R_BH (EM x nuclear) against the reference."""
    from golden_io import light_network_em_decoupled

    z, run, em, source = light_network_em_decoupled()
    blocks = [s.sl for s in run.spec_man.species_refs]
    x = O.OracleSolver(run, 0.2, 0.0, em=em).solve([source("eq")], dz=1e-3)
    assert rel_err_on_support(x, z["state_em"], blocks) < TOL
    X = O.OracleSolver(run, 0.2, 0.0, K=2, em=em).solve([[source("eq")], [source("soft")]], dz=1e-3)
    assert rel_err_on_support(X, z["state_em_multi"], blocks) < TOL
