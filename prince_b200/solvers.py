"""Propagation solvers and the result container (reference API, B200 backend).

``UHECRPropagationSolverETD2`` and ``MultiRHSPropagationSolverETD2`` keep the
constructor signature, ``add_source_class``, ``solve``, ``state`` and ``res``
of the reference solvers (``src/prince_cr/solvers/propagation.py:195-890,
2344-2562``).  The redshift stepping, the photon field, the pair-loss
vectors, the rate fold, the operator split and the ETD2 steps all run on the
GPU through the C ABI; the host evaluates only the scalar schedule (z grid,
windows, dl/dz, source evolution) and moves the state.

The result container ``UHECRPropagationResult`` lives in
``prince_b200.results`` and is re-exported here.
"""

from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sp

from .data import is_decoupled

from . import _lib
from . import constants as C
from .cosmology import H as _H
from .cosmology import dldz as _dldz
from .operators import run_fd_loss_operator, split_diagonal
from .photonfields import device_components, device_table
from .results import UHECRPropagationResult  # noqa: F401  (reference API location)
from .schedule import make_schedule, z_grid


# ---------------------------------------------------------------------------
# device state of one run
# ---------------------------------------------------------------------------
def _dense_kernel(bm):
    if sp.issparse(bm):
        bm = bm.toarray()
    return np.ascontiguousarray(bm, dtype=np.float64)


def device_order(run):
    """``(dev2run, n_blocks)``: the device's row order of the run's state.

    On a shared grid the device keeps the run's layout (``dev2run`` None).
    With species on other grids (gamma and e+- on a decoupled EM grid) the
    device puts the species blocks of the cosmic-ray grid first, in
    ``princeidx`` order, then the other species: device row i holds run row
    ``dev2run[i]`` and rows ``[0, n_blocks)`` are blocks of ``cr_grid.d``
    bins, the layout of the bin-blocked kernels.
    """
    sm = run.spec_man
    if not is_decoupled(sm):
        return None, run.dim_states
    refs = sorted(sm.species_refs, key=lambda x: x.princeidx)
    blocks = [s for s in refs if s.grid_tag == "default"]
    tail = [s for s in refs if s.grid_tag != "default"]
    dev2run = np.concatenate([np.arange(s.lidx(), s.uidx()) for s in blocks + tail]).astype(np.int64)
    return dev2run, sum(s.uidx() - s.lidx() for s in blocks)


def permute_csr(M, dev2run):
    """``(M_dev, order)``: ``M`` with rows and columns in device order (sorted
    CSR) and, for every entry of ``M_dev``, the index of that entry in ``M``'s
    CSR order."""
    M = sp.csr_matrix(M)
    if dev2run is None:
        return M, np.arange(M.nnz)
    n = M.shape[0]
    run2dev = np.empty(n, dtype=np.int64)
    run2dev[dev2run] = np.arange(n)
    rows = np.repeat(np.arange(n), np.diff(M.indptr))
    r, c = run2dev[rows], run2dev[M.indices]
    order = np.lexsort((c, r))
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, r + 1, 1)
    indptr = np.cumsum(indptr)
    M_dev = sp.csr_matrix((np.asarray(M.data)[order], c[order], indptr), shape=M.shape)
    return M_dev, order


class DeviceRun:
    """The run's constant operators resident on one GPU (one C context).

    Uploaded once per (run, device): the coupling pattern, the FP64 fold
    kernel, the photon grid, the FD loss operator, the loss inputs and (if the
    run carries one) the explicit-decay operator, all in the device's row
    order (``device_order``); the solves read and write states in the run's
    order through the context's row map.
    """

    def __init__(self, run, device=0):
        self.run = run
        self.ctx = _lib.Context(device)
        n = run.dim_states
        ir = run.int_rates
        self.n = n
        self.dev2run, n_blocks = device_order(run)
        p = self.dev2run
        self.run2dev = None
        if p is not None:
            self.run2dev = np.empty(n, dtype=np.int64)
            self.run2dev[p] = np.arange(n)
        cm, order = permute_csr(ir.coupling_mat, p)
        self.ctx.set_coupling(n, cm.indptr, cm.indices)
        if p is None:
            self.ctx.set_layout(run.spec_man.nspec and n // run.spec_man.nspec)
        else:
            self.ctx.set_layout(run.cr_grid.d, n_blocks)
            self.ctx.set_row_map(p)
        spec = getattr(ir, "kernel_spec", None)
        if spec is not None:   # expanded on the device, in coupling-CSR order
            self.ctx.build_fold_kernel(spec, np.asarray(spec.chan)[ir.sortidx][order])
        else:
            bm = _dense_kernel(ir._batch_matrix)
            self.ctx.set_fold_kernel(bm if p is None else np.ascontiguousarray(bm[order]))
        self.ctx.set_photon_grid(ir.e_photon.grid)
        D, _ = permute_csr(run_fd_loss_operator(run), p)
        self.D_diag, self.D_off = split_diagonal(D)
        self.ctx.set_fd_operator(self.D_off, self.D_diag)
        pl = run.pair_loss_rates_grid
        pair_bin = np.full(n, -1, dtype=np.int32)
        for s in run.spec_man.species_refs:
            if s.is_nucleus:
                pair_bin[s.lidx():s.uidx()] = np.arange(s.uidx() - s.lidx())
        self.ctx.set_losses(self.dev_vec(run.adia_loss_rates_grid.energy_vector), self.dev_vec(pl.scale_vec),
                            self.dev_vec(pair_bin), pl.xi, pl.phi_xi2, pl.photon_grid)
        self.has_decay = False
        dec = getattr(run, "decay_operator", None)
        if dec is not None:
            diag, off = dec
            self.ctx.set_decay(self.dev_vec(diag), None if off is None else permute_csr(off, p)[0])
            self.has_decay = True

    def dev_vec(self, v):
        """A per-state vector of the run in device order."""
        v = np.asarray(v)
        return v if self.dev2run is None else np.ascontiguousarray(v[self.dev2run])

    def dev_rows(self, rows):
        """Run state rows as device rows."""
        rows = np.asarray(rows)
        return rows if self.run2dev is None else self.run2dev[rows].astype(rows.dtype)

    def ensure_em(self):
        """Upload the EM-cascade layout once: gamma / e+- blocks and the charged
        nuclei feeding Bethe-Heitler pairs (``propagation.py:270-305``)."""
        if getattr(self, "_em_ready", False):
            return
        run = self.run
        sm = run.spec_man
        if 22 not in sm.pdgid2sref:
            raise ValueError("enable_em_cascade needs the photon (22) among the run's species")
        g = sm.pdgid2sref[22]

        def off(s):  # device row of the species block's first bin
            return int(self.dev_rows(np.array([s.lidx()]))[0])

        for p in (11, -11):
            if p in sm.pdgid2sref and sm.pdgid2sref[p].grid_tag != g.grid_tag:
                raise ValueError("gamma and e+- must share one grid")
        lep = [off(sm.pdgid2sref[p]) if p in sm.pdgid2sref else -1 for p in (11, -11)]
        bh = [(off(s), float(s.A)) for s in sm.species_refs if s.is_nucleus and abs(s.charge) >= 1]
        E = run.cr_grid.grid
        with np.errstate(divide="ignore"):
            inv_E = np.where(E > 0, 1.0 / E, 0.0)
        self.ctx.set_em(g.uidx() - g.lidx(), off(g), lep[0], lep[1], E.size,
                        np.array([b[0] for b in bh], dtype=np.int64), np.array([b[1] for b in bh]),
                        inv_E, np.gradient(E))
        self._em_ready = True

    @classmethod
    def of(cls, run, device=0):
        cache = getattr(run, "_b200_device_runs", None)
        if cache is None:
            cache = {}
            try:
                run._b200_device_runs = cache
            except AttributeError:
                return cls(run, device)
        if device not in cache:
            cache[device] = cls(run, device)
        return cache[device]


# ---------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------
def run_em_windows(run, sched, dz):
    """Per-window ``(T_gamma, T_electron, R_BH, dl_step)`` of a run's
    ``em_cascade_model`` at the windows' redshifts (the solvers' ``_em_windows``
    without their override points)."""
    model = getattr(run, "em_cascade_model", None)
    if model is None:
        raise NotImplementedError("enable_em_cascade needs the run's em_cascade_model(z) -> (T_gamma, T_electron, R_BH)")
    if hasattr(model, "prefetch"):
        model.prefetch([float(zw) for zw in sched.z_window])
    out = [model(float(zw)) for zw in sched.z_window]
    dl = [C.PRINCE_UNITS.c * abs(dz) / ((1.0 + float(zw)) * _H(float(zw))) for zw in sched.z_window]
    return (np.stack([np.asarray(o[0], dtype=np.float64) for o in out]),
            np.stack([np.asarray(o[1], dtype=np.float64) for o in out]),
            np.stack([np.asarray(o[2], dtype=np.float64) for o in out]), np.array(dl))


def _host_buffer(shape):
    """A page-locked float64 host array for a solve's states (the device-to-host
    copy runs at the link's rate instead of through a staging buffer); a plain
    array when pinned memory is not available.  torch's caching host allocator
    reuses the blocks of released results."""
    try:
        import torch

        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        return np.empty(shape)


def _other_grids(run):
    """Energies of the run's home grids other than the shared one, by tag."""
    return {t: g.grid for t, g in getattr(run, "grids", {}).items() if t != "default"}


def _coefficients(sources, zs):
    """(n_steps, n_src) table of norm * evolution(z_k) per source."""
    if not sources:
        return np.zeros((zs.size, 0))
    cols = []
    for s in sources:
        if hasattr(s, "evolution_array"):
            ev = s.evolution_array(zs)
        else:
            ev = np.array([s.evolution(z) for z in zs])
        cols.append(s.norm * np.asarray(ev, dtype=np.float64))
    return np.stack(cols, axis=1)


class UHECRPropagationSolverETD2:
    """ETD2 (Cox-Matthews) redshift integrator of the transport equation on one GPU.

    Same constructor and flags as the reference solver
    (``propagation.py:196-209``); ``device`` selects the GPU.
    """

    def __init__(self, initial_z, final_z, prince_run, enable_adiabatic_losses=True,
                 enable_pairprod_losses=True, enable_photohad_losses=True, enable_injection_jacobian=True,
                 enable_partial_diff_jacobian=True, enable_decay=False, enable_decay_jacobian=True,
                 z_offset=0.0, device=0):
        self.initial_z = initial_z + z_offset
        self.final_z = final_z + z_offset
        self.z_offset = z_offset
        self.prince_run = prince_run
        self.backend = prince_run.backend
        self.recomp_z_threshold = self.backend.update_rates_z_threshold
        self.spec_man = prince_run.spec_man
        self.egrid = prince_run.cr_grid.grid
        self.ebins = prince_run.cr_grid.bins
        self.widths = prince_run.cr_grid.widths
        self.enable_adiabatic_losses = enable_adiabatic_losses
        self.enable_pairprod_losses = enable_pairprod_losses
        self.enable_photohad_losses = enable_photohad_losses
        self.enable_injection_jacobian = enable_injection_jacobian
        self.enable_partial_diff_jacobian = enable_partial_diff_jacobian
        self.enable_decay = enable_decay
        self.enable_decay_jacobian = enable_decay_jacobian
        self.dim_states = prince_run.dim_states
        self.state = np.zeros(self.dim_states)
        self.result = None
        self.list_of_sources = []
        self.device = device
        self._dev = DeviceRun.of(prince_run, device)
        self.last_timing = None
        self.enable_em_cascade = bool(getattr(prince_run, "enable_em_cascade", False))
        if self.enable_em_cascade:
            self._dev.ensure_em()
        if enable_decay and not self._dev.has_decay:
            unstable = [s for s in self.spec_man.species_refs if np.isfinite(getattr(s, "lifetime", np.inf))]
            if unstable:
                raise NotImplementedError(
                    "enable_decay=True needs the run's explicit-decay operator: attach "
                    "run.decay_operator = (Lambda_diag, Lambda_off_csr) before creating the solver")

    # -- reference API ---------------------------------------------------
    @property
    def known_species(self):
        return self.spec_man.known_species

    @property
    def res(self):
        if self.result is None:
            self.result = UHECRPropagationResult(self.state, self.egrid, self.spec_man, self.prince_run.cr_grid,
                                                 _other_grids(self.prince_run))
        return self.result

    def add_source_class(self, source_instance):
        self.list_of_sources.append(source_instance)

    def dldz(self, z):
        return _dldz(z)

    def injection(self, dz, z):
        f = self.dldz(z) * dz * C.PRINCE_UNITS.cm2sec
        if len(self.list_of_sources) > 1:
            return f * np.sum([s.injection_rate(z) for s in self.list_of_sources], axis=0)
        return f * self.list_of_sources[0].injection_rate(z)

    def close(self):
        """Reference API (``propagation.py:708``).  The device buffers belong to the
        run's ``DeviceRun`` (shared by every solver of the run on that device and
        released with it), so a solver holds nothing to free."""

    # -- co-evolved EM cascade (propagation.py:540-665) --------------------
    def _em_model(self, z):
        model = getattr(self.prince_run, "em_cascade_model", None)
        if model is None:
            raise NotImplementedError(
                "enable_em_cascade needs the run's em_cascade_model(z) -> (T_gamma, T_electron, R_BH), "
                "or overrides of _em_transfer_at / _em_bh_at")
        return model(z)

    def _em_transfer_at(self, z):
        """(T_gamma, T_electron) of the cascade transfer at redshift z."""
        return tuple(self._em_model(z)[:2])

    def _em_bh_at(self, z):
        """Bethe-Heitler e+- pair shape R_BH at redshift z."""
        return self._em_model(z)[2]

    def _em_windows(self, sched, dz):
        """Per-window T_gamma, T_electron, R_BH and dl_step = c |dz| / ((1+z) H(z)),
        all at the window's redshift (``_refresh_z_caches`` and
        ``_inject_bh_pairs``, ``propagation.py:620-665``)."""
        Tg, Te, R, dl = [], [], [], []
        model = getattr(self.prince_run, "em_cascade_model", None)
        if hasattr(model, "prefetch"):   # build every window's matrices in one device call
            model.prefetch([float(zw) for zw in sched.z_window])
        for zw in sched.z_window:
            zw = float(zw)
            tg, te = self._em_transfer_at(zw)
            Tg.append(np.asarray(tg, dtype=np.float64))
            Te.append(np.asarray(te, dtype=np.float64))
            R.append(np.asarray(self._em_bh_at(zw), dtype=np.float64))
            dl.append(C.PRINCE_UNITS.c * abs(dz) / ((1.0 + zw) * _H(zw)))
        return np.stack(Tg), np.stack(Te), np.stack(R), np.array(dl)

    # -- solve -----------------------------------------------------------
    def _flags(self):
        f = 0
        if self.enable_adiabatic_losses:
            f |= _lib.PB_ADIABATIC
        if self.enable_pairprod_losses:
            f |= _lib.PB_PAIRPROD
        if self.enable_photohad_losses:
            f |= _lib.PB_PHOTOHAD
        if self.enable_injection_jacobian:
            f |= _lib.PB_INJECTION
        if self.enable_partial_diff_jacobian:
            f |= _lib.PB_PARTIAL_DIFF
        if self.enable_decay and self._dev.has_decay:
            f |= _lib.PB_DECAY
        if self.enable_em_cascade:
            f |= _lib.PB_EM_CASCADE
        return f

    def _column_sources(self):
        return [list(self.list_of_sources)]

    def _photon_scale(self):
        return float(getattr(self.prince_run.photon_field, "scale", 1.0))

    def _prepare(self, dz):
        """Host-side schedule, injection basis and column order of one solve."""
        zg = z_grid(self.initial_z, self.final_z, dz)
        sched = make_schedule(zg, self.recomp_z_threshold)
        cols = self._column_sources()
        K = len(cols)
        srcs = [s for c in cols for s in c]
        owner = np.array([k for k, c in enumerate(cols) for _ in c], dtype=np.int64)
        zs = zg[:-1]
        coeff = _coefficients(srcs, zs) if srcs else np.zeros((zs.size, 0))
        grids = [np.asarray(s.injection_grid, dtype=np.float64) for s in srcs]
        # injected states of each source (sources of this package record them when they build their grid)
        support = [s.injection_support if getattr(s, "injection_support", None) is not None else np.flatnonzero(g)
                   for s, g in zip(srcs, grids)]
        use_inj = self.enable_injection_jacobian and len(srcs) > 0
        # first step at which each column receives a non-zero injection
        first = np.full(K, sched.n_steps, dtype=np.int64)
        if use_inj:
            injects = np.array([sp.size > 0 for sp in support])
            live = (coeff != 0.0) & injects[None, :]
            has = live.any(axis=0)
            first_src = np.where(has, live.argmax(axis=0), sched.n_steps)
            np.minimum.at(first, owner, first_src)
        perm = np.argsort(first, kind="stable")          # device column j <- user column perm[j]
        inv = np.empty(K, dtype=np.int64)
        inv[perm] = np.arange(K)
        n_active = np.searchsorted(np.sort(first), np.arange(sched.n_steps), side="right").astype(np.int32)
        src_order = np.argsort(inv[owner], kind="stable") if srcs else np.zeros(0, dtype=np.int64)
        src_col = inv[owner][src_order].astype(np.int32)
        if srcs:
            rows = np.unique(np.concatenate(support)).astype(np.int32)
            G = np.stack([grids[si][rows] for si in src_order], axis=1)
        else:
            rows, G = np.zeros(0, np.int32), np.zeros((0, 0))
        return sched, K, coeff[:, src_order] if srcs else coeff, rows, G, src_col, n_active, perm, use_inj

    def solve(self, dz=1e-3, verbose=False, summary=False, progressbar=False):
        start = time.time()
        sched, K, coeff, rows, G, src_col, n_active, perm, use_inj = self._prepare(dz)
        ctx = self._dev.ctx
        flags = self._flags()
        if use_inj:
            ctx.set_injection(self._dev.dev_rows(rows), G, src_col, K)
        else:
            flags &= ~_lib.PB_INJECTION
        self._set_field(ctx)
        if flags & _lib.PB_EM_CASCADE:
            # the window matrices stay on the device while the windows, the
            # model, its photon field and the solver's hooks are the same
            model = getattr(self.prince_run, "em_cascade_model", None)
            cacheable = (hasattr(model, "prefetch") and "_em_transfer_at" not in self.__dict__
                         and "_em_bh_at" not in self.__dict__)
            key = (tuple(float(z) for z in sched.z_window), float(dz), id(model),
                   id(self.prince_run.photon_field), type(self)._em_transfer_at, type(self)._em_bh_at)
            if not cacheable or getattr(self._dev, "em_key", None) != key:
                ctx.set_em_windows(*self._em_windows(sched, dz))
                self._dev.em_key = key if cacheable else None
        state = _host_buffer((self.dim_states, K)) if K > 1 else np.empty((self.dim_states, K))
        ctx.solve(sched, flags, K, coeff if use_inj else None, n_active, state, photon_scale=self._photon_scale(),
                  out_cols=perm)
        self.last_timing = ctx.last_timing()
        self._store(state)
        self.result = None
        if summary or verbose:
            print("ETD2 summary:")
            print(f"  steps: {sched.n_steps}")
            print(f"  initial z: {self.initial_z} → final z: {self.final_z}")
            print(f"  wall time: {time.time() - start:.3f} s")

    def _set_field(self, ctx):
        f = self.prince_run.photon_field
        ctx.set_photon_field(device_components(f), table=device_table(f))

    def _store(self, state):
        self.state = state[:, 0].copy()

    def operator_pattern(self):
        """M_off pattern (indptr, indices) of the last solve's first window."""
        return self._dev.ctx.operator_pattern(self.dim_states)

    def window_values(self, w):
        ip, ix = self.operator_pattern()
        return self._dev.ctx.window_values(w, self.dim_states, ix.size)


class _MultiRHSView:
    """Column k of a multi-RHS solver: its own sources and result."""

    def __init__(self, parent, k):
        self.parent = parent
        self.k = k
        self.list_of_sources = []

    def add_source_class(self, source_instance):
        self.list_of_sources.append(source_instance)

    @property
    def state(self):
        s = self.parent.state
        return s[:, self.k] if s.ndim == 2 else s

    @property
    def res(self):
        return UHECRPropagationResult(self.state, self.parent.egrid, self.parent.spec_man,
                                      self.parent.prince_run.cr_grid, _other_grids(self.parent.prince_run))


class MultiRHSPropagationSolverETD2(UHECRPropagationSolverETD2):
    """K independent right-hand sides sharing one operator (one SpMM per stage).

    Columns whose sources are still switched off (zero injection so far) are
    exactly zero and are skipped; columns are processed in the order in which
    they switch on, which keeps the active set a prefix of the device tile.
    """

    def __init__(self, *args, K, **kwargs):
        if K < 1:
            raise ValueError(f"K must be >= 1, got {K!r}")
        super().__init__(*args, **kwargs)
        self._K = int(K)
        self._views = [_MultiRHSView(self, k) for k in range(self._K)]
        self.state = np.zeros((self.dim_states, self._K))

    def __len__(self):
        return self._K

    def __getitem__(self, k):
        return self._views[k]

    @property
    def K(self):
        return self._K

    def add_source_class(self, source_instance):
        raise TypeError(
            "MultiRHSPropagationSolverETD2 expects per-RHS sources via "
            "solver[k].add_source_class(...). The k-th view's sources drive "
            "the k-th column of the multi-RHS state.")

    @property
    def res(self):
        raise TypeError("MultiRHSPropagationSolverETD2.res is per-view: use solver[k].res for the k-th RHS.")

    def injection(self, dz, z):
        f = self.dldz(z) * dz * C.PRINCE_UNITS.cm2sec
        out = np.zeros((self.dim_states, self._K))
        for k, view in enumerate(self._views):
            srcs = view.list_of_sources
            if not srcs:
                continue
            col = np.sum([s.injection_rate(z) for s in srcs], axis=0) if len(srcs) > 1 else srcs[0].injection_rate(z)
            out[:, k] = f * col
        return out

    def _column_sources(self):
        return [list(v.list_of_sources) for v in self._views]

    def _store(self, state):
        self.state = state
