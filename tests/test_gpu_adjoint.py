"""Adjoint gradients against central finite differences (needs a B200).

Parameters per source point: spectral index, log10 R_max, composition
fractions, evolution index m; plus the shared photon-density scale.  The
adjoint gradient must match central differences (step h = 1e-5) of the GPU
forward and of the CPU oracle of the reference solver to 1e-6 relative.
"""

import numpy as np
import pytest
import torch

from oracle import etd2_oracle as O
from prince_b200 import adjoint as AD
from prince_b200 import cr_sources, photonfields as pf

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _params(K, seed, nspec):
    rng = np.random.default_rng(seed)
    return dict(gamma=rng.uniform(0.5, 2.2, K), lg_rmax=rng.uniform(9.3, 10.5, K),
                frac=rng.dirichlet(np.ones(nspec), K), m=rng.uniform(-2, 4, K))


def _tensors(p):
    return {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in p.items()}


def _forward(sb, plan, t, scale):
    G = sb.grids(t["gamma"], t["lg_rmax"], t["frac"])
    coeff = sb.coefficients(t["m"])
    return AD.PropagateFunction.apply(G, coeff, scale, plan)


def _central(f, h):
    """Central difference with step h, Richardson-extrapolated with h/2 (error O(h^4))."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def _check_fd(fun, t, scale, keys, rel=TOL, h=1e-5, skip_small=1e-12):
    """Adjoint gradient of fun (via autograd) against central differences (step h)."""
    L = fun(t, scale)
    L.backward()
    worst, where = 0.0, None
    for key in keys:
        base = t[key].detach().clone()
        g = t[key].grad.detach().numpy()
        for idx in np.ndindex(base.shape):
            def f(step):
                tt = {k: v.detach().clone() for k, v in t.items()}
                tt[key][idx] += step
                with torch.no_grad():
                    return float(fun(tt, scale.detach()))
            fd = _central(f, h)
            if abs(fd) < skip_small and abs(g[idx]) < skip_small:
                continue
            err = abs(g[idx] - fd) / max(abs(fd), 1e-300)
            if not err <= worst:
                worst, where = err, (key, idx, float(g[idx]), fd)
    s0 = float(scale.detach())

    def fs(step):
        with torch.no_grad():
            tt = {k: v.detach().clone() for k, v in t.items()}
            return float(fun(tt, torch.tensor(s0 + step, dtype=torch.float64)))
    fd = _central(fs, h * s0)
    gs = float(scale.grad)
    return (worst, where), (abs(gs - fd) / abs(fd), gs, fd)


@pytest.fixture(scope="module")
def light():
    from workloads import light_run
    return light_run()


def test_adjoint_linear_functional_light(light):
    run = light
    species = [2212, 1000020040]
    K = 3
    sb = AD.SourceBatch(run, species, z_max=[0.3, 0.24, 0.17], initial_z=0.3)
    plan = sb.plan(0.3, ckpt_every=8)
    t = _tensors(_params(K, 1, len(species)))
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    # weights 1/X on bins above 1e-12 of each species' maximum, so every bin counts
    # about equally and the differences are not swamped by rounding of large bins
    with torch.no_grad():
        X0 = _forward(sb, plan, {k: v.detach() for k, v in t.items()}, scale.detach())
    w = torch.zeros_like(X0)
    for sref in run.spec_man.species_refs:
        blk = X0[sref.sl]
        mx = blk.abs().max(dim=0).values
        good = blk.abs() > 1e-12 * mx
        w[sref.sl] = torch.where(good, 1.0 / torch.where(good, blk, torch.ones_like(blk)), torch.zeros_like(blk))

    def fun(tt, sc):
        X = _forward(sb, plan, tt, sc)
        return (w * X).sum()

    (worst, where), (worst_s, gs, fds) = _check_fd(fun, t, scale, ["gamma", "lg_rmax", "frac", "m"])
    assert worst < TOL, where
    assert worst_s < TOL, (gs, fds)


def test_adjoint_flux_loss_medium_network():
    from workloads import network_run
    run = network_run(max_mass=16, n_species=60, seed=5)
    species = [2212, 1000020040, 1000070140]
    K = 3
    sb = AD.SourceBatch(run, species, z_max=[0.2, 0.15, 0.12], initial_z=0.2)
    plan = sb.plan(0.2, ckpt_every=32)
    hidden = _tensors(_params(1, 9, len(species)))
    sbh = AD.SourceBatch(run, species, z_max=[0.2], initial_z=0.2)
    ph = sbh.plan(0.2)
    with torch.no_grad():
        Xt = _forward(sbh, ph, hidden, torch.tensor(1.0, dtype=torch.float64))
        _, T = AD.group_flux(run, Xt)
    target = T[:, 0]
    t = _tensors(_params(K, 4, len(species)))
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)

    def fun(tt, sc):
        X = _forward(sb, plan, tt, sc)
        assert torch.isfinite(X).all()
        L = AD.log_ratio_loss(run, X, target, dynamic_range=1e-12).sum()
        assert torch.isfinite(L), L
        return L

    (worst, where), (worst_s, gs, fds) = _check_fd(fun, t, scale, ["gamma", "lg_rmax", "frac", "m"])
    assert worst < TOL, where
    assert worst_s < TOL, (gs, fds)


def test_adjoint_against_oracle_differences(light):
    """Gradient of the flux loss vs central differences of the CPU reference solver."""
    run = light
    species = [2212, 1000020040]
    K = 2
    zmax = [0.15, 0.1]
    sb = AD.SourceBatch(run, species, z_max=zmax, initial_z=0.15)
    plan = sb.plan(0.15, ckpt_every=16)
    p = _params(K, 5, len(species))
    t = _tensors(p)
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    target = torch.tensor(np.logspace(0, -3, 200), dtype=torch.float64)

    X = _forward(sb, plan, t, scale)
    eg, F = AD.group_flux(run, X)
    target = F[:, 0].detach() * 1.3
    L = AD.log_ratio_loss(run, X, target, dynamic_range=1e-12).sum()
    L.backward()

    def oracle_loss(pp, s):
        field = pf.ScaledPhotonField(pf.CMBPhotonSpectrum(), s)
        run.set_photon_field(field)
        try:
            srcs = []
            for k in range(K):
                params = {sp: (pp["gamma"][k], 10 ** pp["lg_rmax"][k], float(pp["frac"][k, i]))
                          for i, sp in enumerate(species)}
                srcs.append([cr_sources.RigdityCutoffSource(run, norm=1.0, params=params,
                                                            m=("simple", float(pp["m"][k])), z_max=zmax[k])])
            Xo = O.OracleSolver(run, 0.15, 0.0, K=K, exp="cr").solve(srcs, dz=1e-3)
        finally:
            run.set_photon_field(pf.CMBPhotonSpectrum())
        return float(AD.log_ratio_loss(run, torch.tensor(Xo), target, dynamic_range=1e-12).sum())

    for key in ("gamma", "lg_rmax", "m", "frac"):
        for k in range(K):
            for i in (range(len(species)) if key == "frac" else [None]):
                def f(step):
                    pp = {kk: np.array(v, dtype=np.float64) for kk, v in p.items()}
                    if i is None:
                        pp[key][k] += step
                    else:
                        pp[key][k, i] += step
                    return oracle_loss(pp, 1.0)
                fd = _central(f, 1e-5)
                g = float(t[key].grad[k] if i is None else t[key].grad[k, i])
                assert abs(g - fd) / abs(fd) < TOL, (key, k, i, g, fd)
    fd = _central(lambda st: oracle_loss(p, 1.0 + st), 1e-5)
    assert abs(float(scale.grad) - fd) / abs(fd) < TOL, (float(scale.grad), fd)


def test_blocked_and_row_kernel_adjoints_agree():
    """The bin-blocked record pass and transposed sweep against the row kernels:
    37 columns (a partial column tile) of the 60-species network, with the
    photon scale, switching on at different redshifts."""
    from prince_b200 import _lib
    from workloads import network_run
    run = network_run(max_mass=16, n_species=60, seed=5)
    species = [2212, 1000020040, 1000070140]
    K = 37
    rng = np.random.default_rng(3)
    sb = AD.SourceBatch(run, species, z_max=list(rng.uniform(0.05, 0.2, K)), initial_z=0.2)
    plan = sb.plan(0.2, ckpt_every=16)
    ctx = plan.dev.ctx
    assert ctx.info(_lib.PB_INFO_BLOCKED_LAYOUT) == 1
    seed = torch.tensor(rng.uniform(0.5, 1.5, (run.dim_states, K)), device="cuda:0")
    grads = []
    for mode in (0, 1):
        ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, mode)
        try:
            t = _tensors(_params(K, 8, len(species)))
            scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
            X = _forward(sb, plan, t, scale)
            assert ctx.info(_lib.PB_INFO_LAST_BLOCKED) == mode
            (seed * X).sum().backward()
            grads.append([t[k].grad.numpy().copy() for k in ("gamma", "lg_rmax", "frac", "m")] + [float(scale.grad)])
        finally:
            ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, 1)
    for g0, g1 in zip(grads[0], grads[1]):
        g0, g1 = np.asarray(g0), np.asarray(g1)
        np.testing.assert_allclose(g1, g0, rtol=1e-9, atol=1e-12 * np.abs(g0).max())


@pytest.mark.parametrize("mode", [1, 0])
def test_adjoint_through_the_em_cascade(mode):
    """Decoupled EM grid: a loss on the photons reaches the source parameters only
    through the Bethe-Heitler pairs and the cascade transfer (the transposed hook)."""
    from golden_io import light_network_em_decoupled
    from prince_b200 import _lib
    z, run, em, source = light_network_em_decoupled()
    species = [2212, 1000020040]
    K = 3
    sb = AD.SourceBatch(run, species, z_max=[0.2, 0.16, 0.12], initial_z=0.2)
    plan = sb.plan(0.2, ckpt_every=8)
    plan.dev.ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, mode)
    t = _tensors(_params(K, 3, len(species)))
    scale = torch.tensor(1.0, dtype=torch.float64)
    with torch.no_grad():
        X0 = _forward(sb, plan, {k: v.detach() for k, v in t.items()}, scale)
    g = run.spec_man.pdgid2sref[22].sl
    w = torch.zeros_like(X0)
    blk = X0[g]
    good = blk.abs() > 1e-12 * blk.abs().max(dim=0).values
    assert good.any()
    w[g] = torch.where(good, 1.0 / torch.where(good, blk, torch.ones_like(blk)), torch.zeros_like(blk))
    p = run.spec_man.pdgid2sref[2212].sl
    w[p] = 1e-3 / X0[p].abs().max()

    def fun(tt, sc):
        return (w * _forward(sb, plan, tt, sc)).sum()

    L = fun(t, scale)
    L.backward()
    worst, where = 0.0, None
    for key in ["gamma", "lg_rmax", "frac", "m"]:
        gr = t[key].grad.detach().numpy()
        for idx in np.ndindex(t[key].shape):
            def f(step):
                tt = {k: v.detach().clone() for k, v in t.items()}
                tt[key][idx] += step
                with torch.no_grad():
                    return float(fun(tt, scale))
            fd = _central(f, 1e-5)
            err = abs(gr[idx] - fd) / max(abs(fd), 1e-300)
            if not err <= worst:
                worst, where = err, (key, idx, float(gr[idx]), fd)
    plan.dev.ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, 1)
    assert worst < TOL, where


def test_adjoint_without_the_photon_scale_records_factors_only(light):
    """A scale that needs no gradient skips the state recompute of the sweep: the
    operator factors alone are recorded, and the source gradients are unchanged."""
    run = light
    species = [2212, 1000020040]
    K = 3
    sb = AD.SourceBatch(run, species, z_max=[0.3, 0.24, 0.17], initial_z=0.3)
    plan = sb.plan(0.3, ckpt_every=8)
    grads = []
    for want in (True, False):
        t = _tensors(_params(K, 7, len(species)))
        scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=want)
        X = _forward(sb, plan, t, scale)
        (X.sum() / X.detach().abs().max()).backward()
        assert (scale.grad is not None) == want
        grads.append({k: v.grad.detach().numpy().copy() for k, v in t.items()})
    for k in grads[0]:
        np.testing.assert_allclose(grads[1][k], grads[0][k], rtol=1e-13, atol=0)


def test_sweep_staging_wait_gives_up_cleanly_and_the_next_gradient_is_exact():
    """The transposed sweep's bin-local kernel stages by TMA behind a bounded
    wait.  With its poll limit at 0 (and no photon-scale gradient, so that the
    sweep's staging is the backward's first wait) the backward raises
    RuntimeError (PB_ERR_DEVICE); with the limit restored the same context
    returns the gradient of a clean run bit for bit."""
    from prince_b200 import _lib
    from workloads import network_run
    run = network_run(max_mass=16, n_species=60, seed=5)
    species = [2212, 1000020040, 1000070140]
    K = 37
    rng = np.random.default_rng(4)
    sb = AD.SourceBatch(run, species, z_max=list(rng.uniform(0.05, 0.2, K)), initial_z=0.2)
    plan = sb.plan(0.2, ckpt_every=16)
    ctx = plan.dev.ctx
    seed = torch.tensor(rng.uniform(0.5, 1.5, (run.dim_states, K)), device="cuda:0")
    scale = torch.tensor(1.0, dtype=torch.float64)

    def gradient():
        t = _tensors(_params(K, 9, len(species)))
        (seed * _forward(sb, plan, t, scale)).sum().backward()
        return [t[k].grad.numpy().copy() for k in ("gamma", "lg_rmax", "frac", "m")]

    ref = gradient()
    assert ctx.info(_lib.PB_INFO_LAST_BLOCKED) == 1
    t = _tensors(_params(K, 9, len(species)))
    X = _forward(sb, plan, t, scale)
    ctx.set_option(_lib.PB_OPT_STAGING_WAIT_TRIES, 0)
    try:
        with pytest.raises(RuntimeError, match="gave up waiting"):
            (seed * X).sum().backward()
    finally:
        ctx.set_option(_lib.PB_OPT_STAGING_WAIT_TRIES, -1)
    again = gradient()
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
