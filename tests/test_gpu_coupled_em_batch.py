"""Parity of the coupled EM cascade at its benchmark scale (needs a B200).

The A <= 56 network with gamma and e+- on the decoupled 128-bin EM grid
(1e-3 to 1e14 GeV), the cascade transfer and the Bethe-Heitler pair shape
built on the device from CMB + the synthetic CIB, and the bench's 2048 seeded
points with z_max ~ U[0.5, 4] (seed 5000), propagated in one batch from
z = 2.5 (the columns with z_max above it inject from the start; the oracle, a
scipy restatement, needs about 70 ms per step on this network, so the range is
capped there).  Three of those columns -- the smallest z_max, the median and
the one nearest 2.5 -- are solved by the oracle on the same redshift grid with
the same per-window EM matrices, and
held to the headline criterion: relative 1e-10 per bin wherever the oracle's
flux exceeds 1e-20 of the species maximum, except on bins whose value the
oracle's own operator perturbations (four draws) move by more than that, where
the GPU must stay within the oracle's spread.  The perturbations are 2e-15
relative: the device operator differs from the oracle's by up to 1.5e-15
(CUDA's libm in the photon densities and the Bethe-Heitler rates, the DMMA
fold order), so that is the size of the differences whose effect the probe
has to cover; over the 2500 steps of this case one bin sits at a zero
crossing of the FD oscillation where 1e-15 draws move it by 4.7e-10 and the
GPU by 5.2e-10.
"""

PERTURB = 2e-15

import multiprocessing as mp

import numpy as np
import pytest

from oracle_jobs import coupled_em_oracle
from test_gpu_headline_parity import TOL, _check

pytestmark = pytest.mark.gpu


def test_coupled_em_batch_vs_oracle():
    from prince_b200.schedule import make_schedule, z_grid
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import draw_points, em_network_run, point_source

    run = em_network_run()
    pts = draw_points(run, 2048, seed=5000, z_range=(0.5, 4.0))
    zmax = np.array([p["zmax"] for p in pts])
    order = np.argsort(zmax)
    cols = [int(order[0]), int(order[1024]), int(np.argmin(np.abs(zmax - 2.5)))]
    zi = 2.5
    m = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=len(pts))
    for k, p in enumerate(pts):
        m[k].add_source_class(point_source(run, p))
    m.solve(dz=1e-3)
    X = np.asarray(m.state)
    assert np.isfinite(X).all()
    g = run.spec_man.pdgid2sref[22].sl
    assert np.abs(X[g]).max() > 0.0
    sched = make_schedule(z_grid(zi, 0.0, 1e-3), run.backend.update_rates_z_threshold)
    model = run.em_cascade_model
    table = {float(z): tuple(np.asarray(a) for a in model(float(z))) for z in sched.z_window}
    with mp.get_context("spawn").Pool(5) as pool:
        ref, *pert = pool.map(coupled_em_oracle, [(cols, zi, s, table, PERTURB) for s in (None, 0, 1, 2, 3)])
    blocks = [s.sl for s in run.spec_man.species_refs]
    rep = _check(X[:, cols], ref, pert, blocks)
    assert rep["worst_on_stable_bins"] <= TOL, rep
    assert rep["gpu_beyond_oracle_spread"] == 0, rep


@pytest.mark.skipif(not __import__("os").environ.get("PRINCE_B200_LONG"),
                    reason="about 6 minutes of oracle time; set PRINCE_B200_LONG=1")
def test_coupled_em_batch_full_range_vs_oracle():
    """The bench's own solve (all 2048 points from the largest z_max, 3,998 steps)
    against the oracle on its two deepest columns, over the whole range."""
    from prince_b200.schedule import make_schedule, z_grid
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import draw_points, em_network_run, point_source

    run = em_network_run()
    pts = draw_points(run, 2048, seed=5000, z_range=(0.5, 4.0))
    zmax = np.array([p["zmax"] for p in pts])
    order = np.argsort(zmax)
    cols = [int(order[-1]), int(order[-2])]
    zi = float(zmax.max())
    m = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=len(pts))
    for k, p in enumerate(pts):
        m[k].add_source_class(point_source(run, p))
    m.solve(dz=1e-3)
    X = np.asarray(m.state)
    sched = make_schedule(z_grid(zi, 0.0, 1e-3), run.backend.update_rates_z_threshold)
    model = run.em_cascade_model
    table = {float(z): tuple(np.asarray(a) for a in model(float(z))) for z in sched.z_window}
    with mp.get_context("spawn").Pool(5) as pool:
        ref, *pert = pool.map(coupled_em_oracle, [(cols, zi, s, table, PERTURB) for s in (None, 0, 1, 2, 3)])
    blocks = [s.sl for s in run.spec_man.species_refs]
    rep = _check(X[:, cols], ref, pert, blocks)
    assert rep["worst_on_stable_bins"] <= TOL, rep
    assert rep["gpu_beyond_oracle_spread"] == 0, rep
