"""Differentiable batched propagation: a ``torch.autograd.Function`` over the C ABI.

``PropagateFunction.apply(G, coeff, scale, plan)`` propagates K columns and
returns the z = 0 states ``X`` (n x K).  Its backward runs the device adjoint
(``pb_adjoint``: checkpointed recomputation, the ETD2 step reversed with the
transposed operator) and returns gradients for

* ``G``      -- injection grids on the injected state rows (n_rows x n_src),
* ``coeff``  -- per-step source coefficients norm * evolution(z_k) (n_steps x n_src),
* ``scale``  -- the photon-density scale shared by the rate fold and the
  Bethe-Heitler loss (a 0-d tensor).

With the co-evolved EM cascade (``run.enable_em_cascade``) the backward also
runs the transposed EM hook after every step (Bethe-Heitler pairs from the
charged nuclei, ``T_gamma`` / ``T_electron`` on gamma and e+-), so a loss on
the photon flux reaches the source parameters; the photon scale then gets no
gradient (the transfer's own dependence on the photon field is not
differentiated).

``SourceBatch`` builds ``G`` and ``coeff`` from per-point parameters with torch
operations (spectral index, log10 rigidity cutoff, five composition fractions,
evolution index), so ``torch.autograd`` carries the gradient back to them.
``group_flux`` is the all-particle flux on the common total-energy grid of
``UHECRPropagationResult.get_solution_group`` (``propagation.py:135-167``),
written with torch operations so a flux loss can be differentiated.

The reference has no adjoint; its gradient is obtained by differencing the
forward solver.  The forward here is the same device solve as
``MultiRHSPropagationSolverETD2``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import constants as C
from .photonfields import device_components, device_table
from .schedule import make_schedule, z_grid
from .solvers import DeviceRun, run_em_windows

FLAGS_ALL = (_lib.PB_ADIABATIC | _lib.PB_PAIRPROD | _lib.PB_PHOTOHAD | _lib.PB_INJECTION
             | _lib.PB_PARTIAL_DIFF)


class Plan:
    """Fixed part of a differentiable solve: run, schedule, injected rows, column order."""

    def __init__(self, run, initial_z, n_cols, rows, src_col, first_active, dz=1e-3, device=0,
                 ckpt_every=32, flags=FLAGS_ALL):
        self.run = run
        self.dev = DeviceRun.of(run, device)
        self.sched = make_schedule(z_grid(initial_z, 0.0, dz), run.backend.update_rates_z_threshold)
        self.em = bool(getattr(run, "enable_em_cascade", False))
        if self.em:
            self.dev.ensure_em()
            flags |= _lib.PB_EM_CASCADE
            self.em_windows = run_em_windows(run, self.sched, dz)
        self.K = int(n_cols)
        self.rows = np.asarray(rows, dtype=np.int32)
        self.src_col = np.asarray(src_col, dtype=np.int64)       # user column of each source
        self.ckpt_every = int(ckpt_every)
        self.flags = int(flags)
        first = np.asarray(first_active, dtype=np.int64)         # first active step per user column
        self.perm = np.argsort(first, kind="stable")             # device column j <- user column perm[j]
        self.inv = np.empty(self.K, dtype=np.int64)
        self.inv[self.perm] = np.arange(self.K)
        self.n_active = np.searchsorted(np.sort(first), np.arange(self.sched.n_steps), side="right").astype(np.int32)
        self.src_order = np.argsort(self.inv[self.src_col], kind="stable")
        self.dev_src_col = self.inv[self.src_col][self.src_order].astype(np.int32)
        self.device = int(device)
        self.last_args = None


class PropagateFunction(torch.autograd.Function):
    """X(z=0) = propagate(G, coeff, scale) with a device adjoint as backward.

    ``X`` is returned as a tensor on the plan's GPU, written there by the solve
    (no host round trip), and the backward hands the incoming gradient of
    ``X`` to the adjoint as a device pointer.  ``G`` and ``coeff`` (a few MB at
    the A <= 56 network) are staged through the host; their gradients are
    returned on ``G``'s device.
    """

    @staticmethod
    def forward(ctx, G, coeff, scale, plan):
        ctx_dev = plan.dev.ctx
        Gd = G.detach().cpu().numpy()[:, plan.src_order]
        cd = coeff.detach().cpu().numpy()[:, plan.src_order]
        ctx_dev.set_injection(plan.dev.dev_rows(plan.rows), np.ascontiguousarray(Gd), plan.dev_src_col, plan.K)
        ctx_dev.set_photon_field(device_components(plan.run.photon_field),
                                 table=device_table(plan.run.photon_field))
        if plan.em:
            ctx_dev.set_em_windows(*plan.em_windows)
            plan.dev.em_key = None   # the solvers' resident windows are replaced
        dev = torch.device("cuda", plan.device)
        X = torch.empty((plan.run.dim_states, plan.K), dtype=torch.float64, device=dev)  # caller's column order
        s = float(scale.detach().cpu().item())
        plan.last_args = (np.ascontiguousarray(cd), s)
        torch.cuda.current_stream(dev).synchronize()
        _solve(ctx_dev, plan, cd, X, s)   # returns after the library stream completed
        ctx.plan = plan
        ctx.in_device = G.device
        # the photon-scale gradient needs the recorded state sensitivities; without
        # it the adjoint records only the operator factors (no state recompute)
        ctx.want_scale = bool(ctx.needs_input_grad[2]) and not plan.em
        return X

    @staticmethod
    def backward(ctx, grad_X):
        plan = ctx.plan
        dev = torch.device("cuda", plan.device)
        seed = grad_X.detach().to(device=dev, dtype=torch.float64).contiguous()  # caller's column order
        torch.cuda.current_stream(dev).synchronize()
        cd, s = plan.last_args
        gG, gc, gs = _adjoint(plan.dev.ctx, plan, cd, s, seed, ctx.want_scale)
        gG_user = np.empty_like(gG)
        gG_user[:, plan.src_order] = gG
        gc_user = np.empty_like(gc)
        gc_user[:, plan.src_order] = gc
        out = ctx.in_device
        g_scale = None if gs is None else torch.tensor(float(gs.sum()), dtype=torch.float64, device=out)
        return torch.from_numpy(gG_user).to(out), torch.from_numpy(gc_user).to(out), g_scale, None


def _args(plan, coeff, scale, state):
    """Solve arguments; ``state`` is a host array or a CUDA tensor (written in place)."""
    import ctypes as Cc

    keep = []

    def f(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(Cc.POINTER(Cc.c_double))

    def i(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return a.ctypes.data_as(Cc.POINTER(Cc.c_int32))

    sc = plan.sched
    args = _lib.SolveArgs()
    args.n_steps = sc.n_steps
    args.n_windows = len(sc.z_window)
    args.n_cols = plan.K
    args.flags = plan.flags
    args.photon_scale = float(scale)
    args.z_window = f(sc.z_window)
    args.window = i(sc.window)
    args.h = f(sc.h)
    args.dldz = f(sc.dldz)
    args.hc = f(sc.hc)
    args.finj = f(sc.finj)
    args.coeff = f(coeff)
    args.n_active = i(plan.n_active)
    if isinstance(state, torch.Tensor):
        args.state = Cc.cast(Cc.c_void_p(state.data_ptr()), Cc.POINTER(Cc.c_double))
        args.state_on_device = 1
    else:
        args.state = state.ctypes.data_as(Cc.POINTER(Cc.c_double))
        args.state_on_device = 0
    args.init_state = 0
    args.ckpt_every = plan.ckpt_every
    args.out_cols = i(plan.perm)  # solve column -> caller column, for the states and the seed
    return args, keep


def _solve(ctx, plan, coeff, out, scale):
    import ctypes as Cc

    args, keep = _args(plan, coeff, scale, out)
    ctx._check(ctx.lib.pb_solve(ctx.h, Cc.byref(args)), "pb_solve")


def _adjoint(ctx, plan, coeff, scale, seed, want_scale=True):
    """Device adjoint; ``seed`` is a contiguous CUDA tensor (n x K, caller's column order).
    The photon-scale gradient (``want_scale``) is None for EM runs or when not wanted."""
    import ctypes as Cc

    dummy = np.zeros(1)  # the adjoint reads no state through args
    args, keep = _args(plan, coeff, scale, dummy)
    n_src = plan.dev_src_col.size
    gG = np.zeros((plan.rows.size, n_src))
    gc = np.zeros((plan.sched.n_steps, n_src))
    gs = np.zeros(plan.K) if (want_scale and not plan.em) else None
    P = lambda a: None if a is None else a.ctypes.data_as(Cc.POINTER(Cc.c_double))
    seed_p = Cc.cast(Cc.c_void_p(seed.data_ptr()), Cc.POINTER(Cc.c_double))
    ctx._check(ctx.lib.pb_adjoint(ctx.h, Cc.byref(args), seed_p, 1, P(gG), P(gc), P(gs)), "pb_adjoint")
    return gG, gc, gs


class SourceBatch:
    """K rigidity-cutoff sources as torch functions of their parameters.

    Per point: ``gamma`` (spectral index), ``lg_rmax`` (log10 R_max / V),
    ``frac`` (composition weights of ``species``), ``m`` (evolution (1+z)^m),
    ``z_max`` (fixed, not differentiated).  The spectrum of species (A, Z) on
    the per-nucleon grid E is ``f A (A E / 1 GeV)^-gamma exp(1 - A E/(Z R_max))``
    -- ``RigdityCutoffSource`` (``cr_sources.py:182-198``).
    """

    def __init__(self, run, species, z_max, initial_z, dz=1e-3):
        self.run = run
        self.species = [int(p) for p in species]
        self.z_max = np.asarray(z_max, dtype=np.float64)
        sm = run.spec_man
        self.rows = np.concatenate([np.arange(sm.pdgid2sref[p].lidx(), sm.pdgid2sref[p].uidx())
                                    for p in self.species]).astype(np.int32)
        E = run.cr_grid.grid
        self.E = torch.tensor(np.tile(E, len(self.species)), dtype=torch.float64)
        self.A = torch.tensor(np.repeat([float(sm.pdgid2sref[p].A) for p in self.species], E.size),
                              dtype=torch.float64)
        self.Z = torch.tensor(np.repeat([float(sm.pdgid2sref[p].Z) for p in self.species], E.size),
                              dtype=torch.float64)
        self.sidx = torch.tensor(np.repeat(np.arange(len(self.species)), E.size))
        zg = z_grid(initial_z, 0.0, dz)
        self.zs = torch.tensor(zg[:-1], dtype=torch.float64)
        K = self.z_max.size
        live = zg[:-1][:, None] <= self.z_max[None, :]
        self.live = torch.tensor(live.astype(np.float64))
        self.first_active = np.array([np.flatnonzero(live[:, k])[0] if live[:, k].any() else zg.size - 1
                                      for k in range(K)])

    def grids(self, gamma, lg_rmax, frac):
        """G (n_rows x K) from per-point tensors gamma (K), lg_rmax (K), frac (K x n_species)."""
        ek = self.A[:, None] * self.E[:, None]
        rmax = 10.0 ** lg_rmax
        f = frac.t()[self.sidx]                                   # (rows, K)
        return f * self.A[:, None] * (ek / 1e9) ** (-gamma[None, :]) * torch.exp(
            1.0 - ek / (self.Z[:, None] * rmax[None, :]))

    def coefficients(self, m, norm=1.0):
        """coeff (n_steps x K): norm (1+z_k)^m where z_k <= z_max, else 0."""
        return norm * (1.0 + self.zs[:, None]) ** m[None, :] * self.live

    def plan(self, initial_z, dz=1e-3, device=0, ckpt_every=32):
        K = self.z_max.size
        return Plan(self.run, initial_z, K, self.rows, np.arange(K), self.first_active, dz=dz,
                    device=device, ckpt_every=ckpt_every)


def group_flux(run, X, egrid=None):
    """All-particle flux of the nuclei on the common total-energy grid (torch, differentiable).

    The reference's ``get_solution_group("CR", epow=3)`` (``propagation.py:103-167``)
    for every column of ``X`` (n x K) at once, through the batched projector of
    ``prince_b200.results``: positive bins interpolated in log-log, zero outside
    each species' positive span.  Returns ``(common grid, flux (G x K))``.
    """
    from .results import GroupProjector, common_energy_grid, select_species

    sm = run.spec_man
    species = select_species(sm, "CR")
    if egrid is None:
        egrid = common_energy_grid(run.cr_grid, max(s.A for s in sm.species_refs))
    key = ("_b200_group_projector", tuple(species), len(egrid), float(egrid[0]), float(egrid[-1]))
    cache = run.__dict__.setdefault("_b200_projectors", {})
    if key not in cache:
        cache[key] = GroupProjector(sm, run.cr_grid.grid, species, egrid)
    pr = cache[key]
    F = pr(X, 3).sum(dim=0)
    return torch.as_tensor(pr.com, dtype=X.dtype, device=X.device), F


def log_ratio_loss(run, X, target, e_min=10 ** 9.5, dynamic_range=0.0):
    """sum over bins with E > e_min of ln(F_k(E) / T(E))^2, per column (K).

    ``F_k`` is the all-particle flux of column k (``group_flux``).  Bins where
    the target is zero or below ``dynamic_range`` of its maximum, and bins where
    the column's flux is zero (beyond the span of the spectra), are left out,
    so the loss stays finite.
    """
    egrid, F = group_flux(run, X)
    T = torch.as_tensor(target, dtype=F.dtype, device=F.device)
    sel = (egrid > e_min) & (T > 0) & (T > dynamic_range * T.max())
    Fs, Ts = F[sel], T[sel][:, None]
    ok = Fs > 0
    r = torch.log(torch.where(ok, Fs, torch.ones_like(Fs))) - torch.log(Ts)
    return torch.where(ok, r * r, torch.zeros_like(r)).sum(dim=0)


def photon_log_ratio_loss(run, X, target, e_min=1e-1, e_max=1e3, dynamic_range=1e-30):
    """sum over photon bins with e_min <= E <= e_max of ln(n_k(E) / T(E))^2, per column.

    ``n_k`` is column k's z = 0 photon spectrum on the photon's home grid (the
    decoupled EM grid when the run has one) and ``T`` a target spectrum on the
    same grid.  Bins where the target is zero or below ``dynamic_range`` of its
    maximum, and bins where the column's spectrum is not positive, are left out.
    """
    s = run.spec_man.pdgid2sref[22]
    grid = (run.em_grid if s.grid_tag != "default" else run.cr_grid).grid
    E = torch.as_tensor(grid, dtype=X.dtype, device=X.device)
    n = X[s.lidx():s.uidx()]
    T = torch.as_tensor(target, dtype=X.dtype, device=X.device)
    sel = (E >= e_min) & (E <= e_max) & (T > 0) & (T > dynamic_range * T.max())
    ns, Ts = n[sel], T[sel][:, None]
    ok = ns > 0
    r = torch.log(torch.where(ok, ns, torch.ones_like(ns))) - torch.log(Ts)
    return torch.where(ok, r * r, torch.zeros_like(r)).sum(dim=0)
