"""The reference's own CPU solver on this package's run objects (CPU).

The run object provides the reference's run contract (``get_hadr_jacobian``,
``build_split_fold`` / ``fold_split``, the loss objects, the species and
grids), so PriNCe's ``ETD2SolverCPU`` and ``_MultiRHSETD2SolverCPU`` -- taken
from the installed reference in ``baseline/_ref`` -- run on the synthetic
workloads unchanged.  That is how the bench's reference arm times the
reference itself.  Its states must equal the oracle's.
"""

import numpy as np
import pytest

import reference_env
from golden_io import rel_err_on_support
from oracle import etd2_oracle as O

pytestmark = pytest.mark.skipif(not reference_env.available(), reason="reference not installed in baseline/_ref")


@pytest.fixture(scope="module")
def ref_solvers():
    config = reference_env.load_package()
    config.linear_algebra_backend = "scipy"
    from prince_cr.solvers import MultiRHSPropagationSolverETD2, UHECRPropagationSolverETD2
    return UHECRPropagationSolverETD2, MultiRHSPropagationSolverETD2


def test_reference_single_solver_on_this_run(ref_solvers):
    from prince_b200 import cr_sources
    from workloads import light_run
    single, _ = ref_solvers
    run = light_run()
    run.backend.linear_algebra_backend = "scipy"
    src = cr_sources.RigdityCutoffSource(run, norm=1.0, params={p: (2.0, 1e10, 1.0)
                                                                 for p in run.spec_man.known_species})
    s = single(initial_z=0.3, final_z=0.0, prince_run=run)
    assert type(s).__name__ == "ETD2SolverCPU"
    s.add_source_class(src)
    s.solve(dz=1e-3)
    ref = O.OracleSolver(run, 0.3, 0.0).solve([src], dz=1e-3)
    assert rel_err_on_support(np.asarray(s.state), ref, [b.sl for b in run.spec_man.species_refs]) < 1e-13


def test_reference_multi_solver_on_this_run(ref_solvers):
    from workloads import draw_points, network_run, point_source
    _, multi = ref_solvers
    run = network_run(max_mass=16, n_species=60, seed=5)
    run.backend.linear_algebra_backend = "scipy"
    pts = draw_points(run, 5, seed=3, z_range=(0.05, 0.1))
    srcs = [point_source(run, p) for p in pts]
    m = multi(initial_z=0.1, final_z=0.0, prince_run=run, K=5)
    assert type(m).__name__ == "_MultiRHSETD2SolverCPU"
    for k, s in enumerate(srcs):
        m[k].add_source_class(s)
    m.solve(dz=1e-3)
    ref = O.OracleSolver(run, 0.1, 0.0, K=5).solve([[s] for s in srcs], dz=1e-3)
    assert rel_err_on_support(np.asarray(m.state), ref, [b.sl for b in run.spec_man.species_refs]) < 1e-13
