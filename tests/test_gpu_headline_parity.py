"""Parity at the configurations the bench times, over their full redshift range (needs a B200).

* One column: the A <= 56 network (350 species x 96 bins), one column, H/He/N/Si/Fe
  injection, z = 1 -> 0 (1000 steps, 100 rate windows), against the oracle:
  relative 1e-10 per bin wherever the oracle's flux exceeds 1e-20 of that
  species' maximum.
* The batch: the first 16 of the bench's 512 seeded points (seed 1000,
  z_max ~ U[0.5, 1]), propagated inside the full 512-column batch exactly as
  the bench runs it, against the oracle over the full range.

Conditioning.  The FD loss stencil oscillates below steep spectral edges, and
a few bins of a large batch sit at the zero crossings of those oscillations
(~1e-8 of the species maximum between neighbours of both signs).  There the
oracle cannot define the answer to 1e-10: a relative perturbation of 1e-15 of
its own operator values (the size of the differences that another summation
order or math library makes) moves those bins by more than 1e-10.  The test
measures that sensitivity on the same case, with two perturbations, and holds
every support bin to the strict 1e-10 wherever the oracle's own spread stays
below it; on the bins where it does not, the GPU must agree with the oracle at
least as closely as the perturbed oracle does.  The assertion messages carry
the counts.
"""

import multiprocessing as mp

import numpy as np
import pytest

from oracle_jobs import headline_oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10
FLOOR = 1e-20


def _oracles(kind, cols, zi):
    """The oracle and two perturbed oracles, solved in parallel spawned processes."""
    with mp.get_context("spawn").Pool(3) as pool:
        return pool.map(headline_oracle, [(kind, cols, zi, s) for s in (None, 0, 1)])


def _per_bin(x, ref, blocks):
    """Relative error per support bin (|ref| > FLOOR x species max per column) and the support mask."""
    X, R = np.atleast_2d(x.T).T, np.atleast_2d(ref.T).T
    err = np.zeros(R.shape)
    sup = np.zeros(R.shape, dtype=bool)
    for sl in blocks:
        r = R[sl]
        m = np.abs(r).max(axis=0)
        s = (np.abs(r) > FLOOR * m[None, :]) & (m[None, :] > 0)
        e = np.zeros(r.shape)
        e[s] = np.abs(X[sl][s] - r[s]) / np.abs(r[s])
        err[sl], sup[sl] = e, s
    return err, sup


def _check(gpu, ref, perturbed, blocks):
    err, sup = _per_bin(gpu, ref, blocks)
    spread = np.max([_per_bin(p, ref, blocks)[0] for p in perturbed], axis=0)
    stable = sup & (spread <= TOL)
    shaky = sup & ~stable
    worst_stable = float(err[stable].max()) if stable.any() else 0.0
    strict_miss = int(np.count_nonzero(err[sup] > TOL))
    beyond_oracle = int(np.count_nonzero(err[shaky] > spread[shaky]))
    report = dict(support=int(sup.sum()), worst_strict=float(err[sup].max()), strict_misses=strict_miss,
                  oracle_sensitive_bins=int(shaky.sum()), worst_on_stable_bins=worst_stable,
                  worst_oracle_spread=float(spread[sup].max()), gpu_beyond_oracle_spread=beyond_oracle)
    print(report)
    return report


@pytest.fixture(scope="module")
def a56():
    from workloads import network_run
    return network_run()


def test_one_column_full_range_vs_oracle(a56):
    from prince_b200 import cr_sources
    from prince_b200.solvers import UHECRPropagationSolverETD2
    from workloads import INJECTED

    run = a56
    params = {p: (2.0, 1e10, 0.2) for p in INJECTED}
    s = UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
    s.add_source_class(cr_sources.RigdityCutoffSource(run, norm=1.0, params=params))
    s.solve(dz=1e-3)
    ref, p0, p1 = _oracles("single", None, 1.0)
    blocks = [sp.sl for sp in run.spec_man.species_refs]
    rep = _check(s.state, ref, (p0, p1), blocks)
    assert rep["worst_on_stable_bins"] < TOL, rep
    assert rep["gpu_beyond_oracle_spread"] == 0, rep
    assert rep["strict_misses"] == 0, rep    # one column: every support bin meets the strict bar


def test_bench_columns_full_range_vs_oracle(a56):
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import draw_points, point_source

    run = a56
    pts = draw_points(run, 512, seed=1000, z_range=(0.5, 1.0))
    zi = max(p["zmax"] for p in pts)
    m = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=512)
    for k, p in enumerate(pts):
        m[k].add_source_class(point_source(run, p))
    m.solve(dz=1e-3)
    cols = list(range(16))
    gpu = m.state[:, cols].copy()
    ref, p0, p1 = _oracles("batch", cols, zi)
    blocks = [sp.sl for sp in run.spec_man.species_refs]
    rep = _check(gpu, ref, (p0, p1), blocks)
    assert rep["worst_on_stable_bins"] < TOL, rep
    assert rep["gpu_beyond_oracle_spread"] == 0, rep
    assert rep["oracle_sensitive_bins"] <= 1e-4 * rep["support"], rep
