"""The B200 solvers plugged into PriNCe itself (needs a B200 and the installed reference).

The reference is imported from its installed copy (``baseline/_ref``); its own
``PriNCeRun`` of the light network (synthetic cross sections, FP64 settings)
and its own source classes drive the solve.  ``prince_b200.plugin.register``
adds the ``"b200"`` backend to the reference's solver factories, so the
reference's ``UHECRPropagationSolverETD2(...)`` / ``MultiRHSPropagationSolverETD2(...)``
construct this package's solvers.  The states must match the reference's own
CPU solver on the same run, and the golden states recorded from the
reference, to 1e-10 per bin above 1e-20 of each species' maximum.
"""

import numpy as np
import pytest

import reference_env
from golden_io import light_network, rel_err_on_support

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_env.available(), reason="reference not installed in baseline/_ref")]
TOL = 1e-10


@pytest.fixture(scope="module")
def ref():
    prince_cr, run = reference_env.load_light_run()
    import prince_cr.solvers.propagation as P
    from prince_b200 import plugin

    plugin.register(P)
    return prince_cr, P, run


def _blocks(run):
    return [s.sl for s in run.spec_man.species_refs]


def _eq(run):
    from prince_cr import cr_sources
    return cr_sources.RigdityCutoffSource(run, norm=1.0, params={int(p): (2.0, 1e10, 1.0)
                                                                   for p in run.spec_man.known_species})


def test_reference_factory_builds_the_b200_solver_and_matches(ref):
    prince_cr, P, run = ref
    from prince_b200 import solvers as B

    run.backend.linear_algebra_backend = "scipy"
    cpu = P.UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
    assert type(cpu).__name__ == "ETD2SolverCPU"
    cpu.add_source_class(_eq(run))
    cpu.solve(dz=1e-3)
    run.backend.linear_algebra_backend = "b200"
    try:
        s = P.UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
        assert isinstance(s, B.UHECRPropagationSolverETD2)
        s.add_source_class(_eq(run))
        s.solve(dz=1e-3)
    finally:
        run.backend.linear_algebra_backend = "scipy"
    assert rel_err_on_support(s.state, np.asarray(cpu.state), _blocks(run)) < TOL
    z, _, _ = light_network()
    assert rel_err_on_support(s.state, z["state_plain"], _blocks(run)) < TOL
    # the result container on the reference's grid object
    g_ref, f_ref = cpu.res.get_solution_group("CR", epow=3)
    g, f = s.res.get_solution_group("CR", epow=3)
    np.testing.assert_allclose(g, g_ref, rtol=1e-14)
    np.testing.assert_allclose(f, f_ref, rtol=1e-9, atol=1e-12 * np.abs(f_ref).max())


def test_reference_multi_rhs_factory_with_reference_sources(ref):
    prince_cr, P, run = ref
    from prince_cr import cr_sources
    from prince_b200 import solvers as B

    z, _, _ = light_network()
    cols = [str(c).split(",") for c in z["multi_columns"]]
    import ast

    def source(key):
        kind = str(z[f"src_{key}_kind"])
        params = ast.literal_eval(str(z[f"src_{key}_params"]))
        m = ast.literal_eval(str(z[f"src_{key}_m"]))
        zmax = float(z[f"src_{key}_zmax"])
        src = getattr(cr_sources, kind)(run, norm=float(z[f"src_{key}_norm"]), params=params, m=m)
        if np.isfinite(zmax):   # the golden run's z_max cut (its ZmaxRigidity subclass)
            ev = src.evolution
            src.evolution = lambda zz, _ev=ev, _zm=zmax: 0.0 if zz > _zm else _ev(zz)
        return src

    run.backend.linear_algebra_backend = "b200"
    try:
        m = P.MultiRHSPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run, K=len(cols))
        assert isinstance(m, B.MultiRHSPropagationSolverETD2)
        for k, keys in enumerate(cols):
            for key in keys:
                m[k].add_source_class(source(key))
        m.solve(dz=1e-3)
    finally:
        run.backend.linear_algebra_backend = "scipy"
    assert rel_err_on_support(m.state, z["state_multi"], _blocks(run)) < TOL


def test_reference_em_run_through_the_b200_backend():
    """PriNCe's own run with the co-evolved EM cascade on its decoupled EM grid
    (276 bins, 16 per decade, native coupling) and its own CPU solver (per-window
    kinetic transfer and Bethe-Heitler shape, FP64) against the b200 backend on
    the same run object, with the transfer and shape built on the device."""
    import prince_cr.solvers.propagation as P
    from prince_cr import cr_sources
    from prince_b200 import plugin, solvers as B
    from prince_b200.em_cascade import KineticCascadeModel

    prince_cr, run = reference_env.load_light_em_run()
    plugin.register(P)
    assert run.em_grid is not None and run.em_grid.d == 276
    params = {2212: (2.0, 1e10, 1.0), 1000020040: (2.0, 1e10, 1.0)}
    run.backend.linear_algebra_backend = "scipy"
    cpu = P.UHECRPropagationSolverETD2(initial_z=0.02, final_z=0.0, prince_run=run)
    assert type(cpu).__name__ == "ETD2SolverCPU" and cpu.enable_em_cascade
    cpu.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=params))
    cpu.solve(dz=1e-3)
    ref = np.asarray(cpu.state)
    assert np.isfinite(ref).all()
    run.em_cascade_model = KineticCascadeModel(run, 1e-3)
    run.backend.linear_algebra_backend = "b200"
    try:
        s = P.UHECRPropagationSolverETD2(initial_z=0.02, final_z=0.0, prince_run=run)
        assert isinstance(s, B.UHECRPropagationSolverETD2)
        s.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=params))
        s.solve(dz=1e-3)
    finally:
        run.backend.linear_algebra_backend = "scipy"
    g = run.spec_man.pdgid2sref[22].sl
    assert np.abs(ref[g]).max() > 0
    assert rel_err_on_support(s.state, ref, _blocks(run)) < TOL
