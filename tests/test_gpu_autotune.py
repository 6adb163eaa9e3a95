"""The autotuner of the batched stage (needs a B200).

``prince_b200.autotune.tune`` times every candidate (band-tile CTA warps,
bin-local prefetch depth, staging) with a short all-columns-active solve on
the live operator, keeps the fastest on the context and caches it per device
and shape.  The prefetch depth and the staging do not change the arithmetic,
so every choice with the default band CTAs gives bit-identical states; the
half-size band CTAs sum the band partials in other groups (agreement far
below the parity bar).
"""

import numpy as np
import pytest

from golden_io import local_scale_check, rel_err_on_support
from oracle import etd2_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_tuned_choice_is_fastest_cached_and_gives_the_same_states(tmp_path):
    from prince_b200 import _lib, autotune
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import draw_points, network_run, point_source
    run = network_run(max_mass=16, n_species=60, seed=5)
    blocks = [s.sl for s in run.spec_man.species_refs]
    K = 96
    pts = draw_points(run, K, seed=17, z_range=(0.02, 0.05))
    srcs = [point_source(run, p) for p in pts]
    zi = max(p["zmax"] for p in pts)
    m = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=K)
    for k, s in enumerate(srcs):
        m[k].add_source_class(s)
    ctx = m._dev.ctx
    m.solve(dz=1e-3)
    default = m.state.copy()
    path = str(tmp_path / "autotune.json")
    choice, cands = autotune.tune(m, path=path, force=True, steps=8, reps=2)
    assert len(cands) == 12
    assert choice["steps_ms"] == min(c["steps_ms"] for c in cands) < 1e299
    assert ctx.info(_lib.PB_OPT_BAND_WARPS) == choice["band_warps"]
    assert ctx.info(_lib.PB_OPT_SLAB_PREFETCH) == choice["slab_prefetch"]
    assert ctx.info(_lib.PB_OPT_TMA_STAGING) == choice["tma_staging"]
    m.solve(dz=1e-3)
    if choice["band_warps"] == 8:
        assert np.array_equal(m.state, default)
    else:
        worst, _, _ = local_scale_check(m.state, default, blocks, tol=TOL)
        assert worst < 1e-13
    # every prefetch depth and staging with the default band CTAs: identical states
    try:
        for pre in (1, 3):
            for tma in (1, 0):
                autotune.apply(ctx, dict(band_warps=8, slab_prefetch=pre, tma_staging=tma))
                m.solve(dz=1e-3)
                assert np.array_equal(m.state, default), (pre, tma)
    finally:
        autotune.apply(ctx, choice)
    again, none = autotune.tune(m, path=path)
    assert none is None and again == choice
    ref = O.OracleSolver(run, zi, 0.0, K=K, exp="cr").solve([[s] for s in srcs], dz=1e-3)
    assert rel_err_on_support(default, ref, blocks) < TOL
