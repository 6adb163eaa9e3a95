"""Tabulated photon field on the device against the reference (needs a B200).

The light network in CMB + the Gilmore (2012) EBL table: the device's window
operator (photon vector folded into M, and the Bethe-Heitler loss vector from
the table) and the z = 1 -> 0 state against the reference's own recorded
values (``tests/golden/light_network_ebl.npz``), and a batched solve against
the oracle.
"""

import numpy as np
import pytest

from golden_io import light_network_ebl, rel_err_on_support
from oracle import etd2_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def golden():
    return light_network_ebl()


def _eq(run):
    from prince_b200 import cr_sources
    return cr_sources.RigdityCutoffSource(run, norm=1.0, params={p: (2.0, 1e10, 1.0)
                                                                 for p in run.spec_man.known_species})


def test_device_pair_loss_and_state_with_gilmore_table(golden):
    from prince_b200.solvers import UHECRPropagationSolverETD2
    z, run, _ = golden
    s = UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
    s.add_source_class(_eq(run))
    s.solve(dz=1e-3)
    off, diag, kp = s.window_values(0)
    np.testing.assert_allclose(kp, z["kappa_pair_z1p0"], rtol=1e-13, atol=0)
    o = O.OracleSolver(run, 1.0, 0.0, exp="cr")
    o._refresh(1.0, first=True)
    nz = o.M_off.data != 0
    np.testing.assert_allclose(off[nz], o.M_off.data[nz], rtol=1e-13, atol=0)
    assert rel_err_on_support(s.state, z["state_ebl"], [sp.sl for sp in run.spec_man.species_refs]) < TOL


def test_batched_solve_with_gilmore_table_vs_oracle(golden):
    from prince_b200 import cr_sources
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, _ = golden
    K = 5
    rng = np.random.default_rng(4)
    srcs = []
    for k in range(K):
        params = {p: (rng.uniform(1.0, 2.5), 10 ** rng.uniform(9.5, 11), rng.uniform(0.2, 1.0))
                  for p in (2212, 1000020040)}
        srcs.append(cr_sources.RigdityCutoffSource(run, norm=1.0, params=params, m=("simple", rng.uniform(-1, 3)),
                                                   z_max=rng.uniform(0.3, 0.6)))
    m = MultiRHSPropagationSolverETD2(initial_z=0.6, final_z=0.0, prince_run=run, K=K)
    for k, src in enumerate(srcs):
        m[k].add_source_class(src)
    m.solve(dz=1e-3)
    ref = O.OracleSolver(run, 0.6, 0.0, K=K, exp="cr").solve([[x] for x in srcs], dz=1e-3)
    assert rel_err_on_support(m.state, ref, [sp.sl for sp in run.spec_man.species_refs]) < TOL
