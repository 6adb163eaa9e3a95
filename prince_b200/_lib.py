"""ctypes binding of the C ABI in ``include/prince_b200.h``.

The shared library ``prince_b200/libprince_b200.so`` is built in-tree by
``prince_b200.build.build()`` (nvcc, sm_100a).  Loading fails loudly when the
library is missing: there is no CPU implementation behind this package.

``Context`` owns one ``pb_context`` (one device, one stream).  Non-zero
status codes become exceptions: ``PB_ERR_ARG`` -> ``ValueError``, everything
else -> ``RuntimeError``, with the library's message.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libprince_b200.so")

PB_OK, PB_ERR_ARG, PB_ERR_STATE, PB_ERR_CUDA, PB_ERR_DEVICE = 0, 1, 2, 3, 4
PB_ADIABATIC, PB_PAIRPROD, PB_PHOTOHAD, PB_INJECTION, PB_PARTIAL_DIFF, PB_DECAY = 1, 2, 4, 8, 16, 32
PB_EM_CASCADE = 64
PB_OPT_BATCHED_KERNELS, PB_INFO_BLOCKED_LAYOUT, PB_INFO_LAST_BLOCKED, PB_INFO_BAND_SPECIES = 1, 2, 3, 4
PB_INFO_BAND_ENTRIES, PB_INFO_SLAB_ENTRIES, PB_INFO_SLAB_ROWS, PB_INFO_FD_DENSE = 5, 6, 7, 8
PB_OPT_TMA_STAGING, PB_INFO_LAST_TMA = 9, 10
PB_OPT_STAGING_WAIT_TRIES = 11
PB_OPT_BAND_WARPS = 12
PB_OPT_SLAB_PREFETCH = 13

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_vp = C.c_void_p


class SolveArgs(C.Structure):
    _fields_ = [
        ("n_steps", C.c_int64),
        ("n_windows", C.c_int32),
        ("n_cols", C.c_int32),
        ("flags", C.c_uint32),
        ("photon_scale", C.c_double),
        ("z_window", _d),
        ("window", _i32),
        ("h", _d),
        ("dldz", _d),
        ("hc", _d),
        ("finj", _d),
        ("coeff", _d),
        ("n_active", _i32),
        ("state", _d),
        ("init_state", C.c_int32),
        ("state_on_device", C.c_int32),
        ("ckpt_every", C.c_int32),
        ("out_cols", _i32),
    ]


class KernelSpecArgs(C.Structure):
    """``pb_kernel_spec``: the fold kernel as per-channel response samples."""

    _fields_ = [
        ("d", C.c_int32),
        ("dph", C.c_int32),
        ("f_mo", _d),
        ("dE", _d),
        ("n_resp", C.c_int32),
        ("resp", _d),
        ("n_ddr", C.c_int32),
        ("ddr", _d),
        ("n_sep", C.c_int32),
        ("sep_a", _d),
        ("sep_b", _d),
        ("n_channels", C.c_int32),
        ("channels", _i32),
        ("entry_channel", _i32),
    ]


class EmTransferArgs(C.Structure):
    """``pb_em_transfer_args``."""

    _fields_ = [
        ("n", C.c_int32), ("E", _d), ("n_z", C.c_int32), ("z", _d), ("dl_step", _d),
        ("n_eps", C.c_int32), ("eps", _d), ("n_eps_o", C.c_int32), ("eps_o", _d),
        ("n_mu", C.c_int32), ("mu", _d), ("n_E1", C.c_int32), ("photon_scale", C.c_double),
        ("cool_floor_frac", C.c_double), ("max_scatter", C.c_int32), ("tol", C.c_double),
        ("m_electron", C.c_double), ("r_electron", C.c_double), ("c_cm", C.c_double),
        ("T_gamma", _d), ("T_electron", _d), ("iterations", C.POINTER(C.c_int32)),
    ]


class BhShapeArgs(C.Structure):
    """``pb_bh_shape_args``."""

    _fields_ = [
        ("n_e", C.c_int32), ("E_e", _d), ("n_p", C.c_int32), ("E_p", _d), ("n_eps", C.c_int32), ("eps", _d),
        ("n_z", C.c_int32), ("z", _d), ("photon_scale", C.c_double), ("e_p_min", C.c_double),
        ("m_electron", C.c_double), ("m_proton", C.c_double), ("R", _d),
    ]


class TuneChoice(C.Structure):
    _fields_ = [("band_warps", C.c_int32), ("slab_prefetch", C.c_int32), ("tma_staging", C.c_int32),
                ("steps_ms", C.c_double)]


# name -> (restype, argtypes)
_PROTOS = {
    "pb_abi_version": (C.c_int, []),
    "pb_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "pb_destroy": (None, [_vp]),
    "pb_last_error": (C.c_char_p, [_vp]),
    "pb_global_error": (C.c_char_p, []),
    "pb_set_coupling": (C.c_int, [_vp, C.c_int64, C.c_int64, _i64, _i32]),
    "pb_set_fold_kernel": (C.c_int, [_vp, C.c_int64, C.c_int32, _d]),
    "pb_set_photon_grid": (C.c_int, [_vp, C.c_int32, _d]),
    "pb_set_photon_field": (C.c_int, [_vp, C.c_int32, _i32, _d]),
    "pb_set_photon_table": (C.c_int, [_vp, C.c_int32, C.c_int32, _d, _d, _d]),
    "pb_build_fold_kernel": (C.c_int, [_vp, C.POINTER(KernelSpecArgs)]),
    "pb_autotune": (C.c_int, [_vp, C.POINTER(SolveArgs), C.c_int32, C.c_int32, C.POINTER(TuneChoice),
                              C.POINTER(C.c_int32)]),
    "pb_get_fold_kernel": (C.c_int, [_vp, C.c_int64, C.c_int32, _d]),
    "pb_em_transfer": (C.c_int, [_vp, C.POINTER(EmTransferArgs)]),
    "pb_bh_shape": (C.c_int, [_vp, C.POINTER(BhShapeArgs)]),
    "pb_set_fd_operator": (C.c_int, [_vp, C.c_int64, _i64, _i32, _d, _d]),
    "pb_set_losses": (C.c_int, [_vp, _d, _d, _i32, C.c_int32, C.c_int32, _d, _d, _d]),
    "pb_set_decay": (C.c_int, [_vp, _d, C.c_int64, _i64, _i32, _d]),
    "pb_set_injection": (C.c_int, [_vp, C.c_int32, C.c_int32, _i32, _d, C.c_int32, _i32]),
    "pb_set_layout": (C.c_int, [_vp, C.c_int32]),
    "pb_set_layout_rows": (C.c_int, [_vp, C.c_int32, C.c_int64]),
    "pb_set_row_map": (C.c_int, [_vp, _i32]),
    "pb_set_option": (C.c_int, [_vp, C.c_int32, C.c_int64]),
    "pb_get_info": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int64)]),
    "pb_profile_stage": (C.c_int, [_vp, C.c_int64, C.c_int32, C.c_int32, _d]),
    "pb_fp64_peak": (C.c_int, [_vp, _d]),
    "pb_set_em": (C.c_int, [_vp, C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32, _i64, _d, _d,
                            _d]),
    "pb_set_em_windows": (C.c_int, [_vp, C.c_int32, _d, _d, _d, _d]),
    "pb_solve": (C.c_int, [_vp, C.POINTER(SolveArgs)]),
    "pb_adjoint": (C.c_int, [_vp, C.POINTER(SolveArgs), _d, C.c_int32, _d, _d, _d]),
    "pb_get_operator_pattern": (C.c_int, [_vp, _i64, _i64, _i32]),
    "pb_get_window": (C.c_int, [_vp, C.c_int32, _d, _d, _d]),
    "pb_integrate_const": (C.c_int, [_vp, C.c_int64, _d, C.c_int64, _i64, _i32, _d, C.c_int64, _d, _d]),
    "pb_integrate_const_noalloc": (C.c_int, [_vp, C.c_int64, _vp, C.c_int64, _vp, _vp, _vp, C.c_int64, _vp,
                                              _vp]),
    "pb_eval_exp": (C.c_int, [_vp, C.c_int64, _d, _d]),
    "pb_last_timing": (C.c_int, [_vp, _d, _d, _d, _i64]),
}

_LIB = None


def exported_symbols():
    """Names of the C ABI functions this binding expects."""
    return list(_PROTOS)


def load():
    """Load the in-tree shared library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA extension first "
            "(python -c 'import __graft_entry__ as g; g.build()' or "
            "python -m prince_b200.build). There is no CPU fallback."
        )
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32a(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _i64a(a):
    return np.ascontiguousarray(a, dtype=np.int64)


class Context:
    """One device context of the C library."""

    def __init__(self, device=0):
        self.lib = load()
        h = _vp()
        rc = self.lib.pb_create(int(device), C.byref(h))
        if rc != PB_OK:
            msg = self.lib.pb_global_error().decode()
            raise (ValueError if rc == PB_ERR_ARG else RuntimeError)(f"pb_create: {msg}")
        self.h = h
        self.device = int(device)

    def _check(self, rc, what):
        if rc != PB_OK:
            msg = self.lib.pb_last_error(self.h).decode()
            raise (ValueError if rc == PB_ERR_ARG else RuntimeError)(f"{what}: {msg}")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.pb_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ---------------------------------------------------------
    def set_coupling(self, n, indptr, indices):
        indptr, indices = _i64a(indptr), _i32a(indices)
        self._check(self.lib.pb_set_coupling(self.h, int(n), int(indices.size), _ptr(indptr, C.c_int64),
                                             _ptr(indices, C.c_int32)), "pb_set_coupling")

    def set_fold_kernel(self, kernel):
        kernel = _f64(kernel)
        self._check(self.lib.pb_set_fold_kernel(self.h, int(kernel.shape[0]), int(kernel.shape[1]),
                                                _ptr(kernel, C.c_double)), "pb_set_fold_kernel")

    def build_fold_kernel(self, spec, entry_channel):
        """Build the fold kernel on the device from a ``KernelSpec``; ``entry_channel``
        is the channel of each coupling entry in CSR order."""
        keep = []

        def f(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _ptr(a, C.c_double)

        def i(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return _ptr(a, C.c_int32)

        k = KernelSpecArgs()
        k.d, k.dph = int(spec.d), int(spec.dph)
        k.f_mo, k.dE = f(spec.f_mo), f(spec.dE)
        k.n_resp, k.resp = int(spec.resp.shape[0]), f(spec.resp if spec.resp.size else np.zeros(1))
        k.n_ddr, k.ddr = int(spec.ddr.shape[0]), f(spec.ddr if spec.ddr.size else np.zeros(1))
        k.n_sep = int(spec.sep_a.shape[0])
        k.sep_a = f(spec.sep_a if spec.sep_a.size else np.zeros(1))
        k.sep_b = f(spec.sep_b if spec.sep_b.size else np.zeros(1))
        k.n_channels, k.channels = int(spec.channels.shape[0]), i(spec.channels)
        k.entry_channel = i(entry_channel if np.size(entry_channel) else np.zeros(1))
        self._check(self.lib.pb_build_fold_kernel(self.h, C.byref(k)), "pb_build_fold_kernel")

    def fold_kernel(self, R, dph):
        """The device fold kernel (R x dph, coupling-CSR order)."""
        out = np.empty((int(R), int(dph)))
        self._check(self.lib.pb_get_fold_kernel(self.h, int(R), int(dph), _ptr(out, C.c_double)),
                    "pb_get_fold_kernel")
        return out

    def em_transfer(self, E, zs, dl_step, eps, eps_o, mu, n_E1=400, photon_scale=1.0, cool_floor_frac=0.1,
                    max_scatter=4000, tol=1e-4):
        """Device kinetic cascade transfer on the context's photon field:
        ``(T_gamma, T_electron, passes)`` with the matrices ``(n_z, n, n)``."""
        from .constants import PRINCE_UNITS as U

        keep = [_f64(E), _f64(zs), _f64(dl_step), _f64(eps), _f64(eps_o), _f64(mu)]
        E_, z_, dl_, eps_, epso_, mu_ = keep
        n, nz = E_.size, z_.size
        Tg = np.empty((nz, n, n))
        Te = np.empty((nz, n, n))
        it = C.c_int32(0)
        a = EmTransferArgs()
        a.n, a.E = n, _ptr(E_, C.c_double)
        a.n_z, a.z, a.dl_step = nz, _ptr(z_, C.c_double), _ptr(dl_, C.c_double)
        a.n_eps, a.eps = eps_.size, _ptr(eps_, C.c_double)
        a.n_eps_o, a.eps_o = epso_.size, _ptr(epso_, C.c_double)
        a.n_mu, a.mu = mu_.size, _ptr(mu_, C.c_double)
        a.n_E1, a.photon_scale = int(n_E1), float(photon_scale)
        a.cool_floor_frac, a.max_scatter, a.tol = float(cool_floor_frac), int(max_scatter), float(tol)
        a.m_electron, a.r_electron, a.c_cm = U.m_electron, U.r_electron, U.c
        a.T_gamma, a.T_electron = _ptr(Tg, C.c_double), _ptr(Te, C.c_double)
        a.iterations = C.pointer(it)
        self._check(self.lib.pb_em_transfer(self.h, C.byref(a)), "pb_em_transfer")
        return Tg, Te, it.value

    def bh_shape(self, E_e, E_p, eps, zs, e_p_min=1e5, photon_scale=1.0):
        """Device Bethe-Heitler pair shapes on the context's photon field: ``(n_z, n_e, n_p)``."""
        from .constants import PRINCE_UNITS as U

        Ee, Ep, ep, z = _f64(E_e), _f64(E_p), _f64(eps), _f64(np.atleast_1d(zs))
        R = np.empty((z.size, Ee.size, Ep.size))
        a = BhShapeArgs()
        a.n_e, a.E_e, a.n_p, a.E_p = Ee.size, _ptr(Ee, C.c_double), Ep.size, _ptr(Ep, C.c_double)
        a.n_eps, a.eps, a.n_z, a.z = ep.size, _ptr(ep, C.c_double), z.size, _ptr(z, C.c_double)
        a.photon_scale, a.e_p_min = float(photon_scale), float(e_p_min)
        a.m_electron, a.m_proton = U.m_electron, U.m_proton
        a.R = _ptr(R, C.c_double)
        self._check(self.lib.pb_bh_shape(self.h, C.byref(a)), "pb_bh_shape")
        return R

    def set_photon_grid(self, energies):
        e = _f64(energies)
        self._check(self.lib.pb_set_photon_grid(self.h, int(e.size), _ptr(e, C.c_double)), "pb_set_photon_grid")

    def set_photon_field(self, components, table=None):
        """Field components ``(kind, p0, p1, p2)``; ``table = (z, log10 E, log10 dn/de)`` for kind 3."""
        if table is not None:
            tz, tle, tv = _f64(table[0]), _f64(table[1]), _f64(table[2])
            self._check(self.lib.pb_set_photon_table(self.h, int(tz.size), int(tle.size), _ptr(tz, C.c_double),
                                                     _ptr(tle, C.c_double), _ptr(tv, C.c_double)),
                        "pb_set_photon_table")
        kinds = _i32a([c[0] for c in components])
        pars = _f64([list(c[1:4]) for c in components]).reshape(-1)
        self._check(self.lib.pb_set_photon_field(self.h, int(kinds.size), _ptr(kinds, C.c_int32),
                                                 _ptr(pars, C.c_double)), "pb_set_photon_field")

    def set_fd_operator(self, off, diag):
        ip, ix, v, dg = _i64a(off.indptr), _i32a(off.indices), _f64(off.data), _f64(diag)
        self._check(self.lib.pb_set_fd_operator(self.h, int(v.size), _ptr(ip, C.c_int64), _ptr(ix, C.c_int32),
                                                _ptr(v, C.c_double), _ptr(dg, C.c_double)), "pb_set_fd_operator")

    def set_losses(self, adia_energy, pair_scale, pair_bin, xi, phi_xi2, pair_photon_grid):
        ae, ps, pb_ = _f64(adia_energy), _f64(pair_scale), _i32a(pair_bin)
        xi, ph, pg = _f64(xi), _f64(phi_xi2), _f64(pair_photon_grid)
        self._check(self.lib.pb_set_losses(self.h, _ptr(ae, C.c_double), _ptr(ps, C.c_double),
                                           _ptr(pb_, C.c_int32), int(pg.shape[0]), int(xi.size),
                                           _ptr(xi, C.c_double), _ptr(ph, C.c_double), _ptr(pg, C.c_double)),
                    "pb_set_losses")

    def set_decay(self, diag, off=None):
        dg = None if diag is None else _f64(diag)
        if off is None or off.nnz == 0:
            self._check(self.lib.pb_set_decay(self.h, _ptr(dg, C.c_double), 0, None, None, None), "pb_set_decay")
            return
        ip, ix, v = _i64a(off.indptr), _i32a(off.indices), _f64(off.data)
        self._check(self.lib.pb_set_decay(self.h, _ptr(dg, C.c_double), int(v.size), _ptr(ip, C.c_int64),
                                          _ptr(ix, C.c_int32), _ptr(v, C.c_double)), "pb_set_decay")

    def set_injection(self, rows, grids, src_col, n_cols):
        rows, grids, src_col = _i32a(rows), _f64(grids), _i32a(src_col)
        self._check(self.lib.pb_set_injection(self.h, int(src_col.size), int(rows.size), _ptr(rows, C.c_int32),
                                              _ptr(grids, C.c_double), int(n_cols), _ptr(src_col, C.c_int32)),
                    "pb_set_injection")

    def set_layout(self, d, n_blocks=None):
        if n_blocks is None:
            self._check(self.lib.pb_set_layout(self.h, int(d)), "pb_set_layout")
        else:
            self._check(self.lib.pb_set_layout_rows(self.h, int(d), int(n_blocks)), "pb_set_layout_rows")

    def set_row_map(self, caller_row):
        """Device row i holds the caller's row ``caller_row[i]`` (None: identity)."""
        if caller_row is None:
            self._check(self.lib.pb_set_row_map(self.h, None), "pb_set_row_map")
            return
        m = _i32a(caller_row)
        self._check(self.lib.pb_set_row_map(self.h, _ptr(m, C.c_int32)), "pb_set_row_map")

    def set_option(self, key, value):
        self._check(self.lib.pb_set_option(self.h, int(key), int(value)), "pb_set_option")

    def info(self, key):
        v = C.c_int64(0)
        self._check(self.lib.pb_get_info(self.h, int(key), C.byref(v)), "pb_get_info")
        return int(v.value)

    def profile_stage(self, step, stage, reps=5):
        """Per-kernel milliseconds of one stage of the last solve: (fd, slab, band, band_finish)."""
        out = np.zeros(4)
        self._check(self.lib.pb_profile_stage(self.h, int(step), int(stage), int(reps), _ptr(out, C.c_double)),
                    "pb_profile_stage")
        return tuple(float(v) for v in out)

    def fp64_peak(self):
        v = np.zeros(1)
        self._check(self.lib.pb_fp64_peak(self.h, _ptr(v, C.c_double)), "pb_fp64_peak")
        return float(v[0])

    def set_em(self, n_em, gamma_off, em_off, ep_off, n_cr, bh_off, bh_A, inv_E, dE):
        bo, ba, ie, de = _i64a(bh_off), _f64(bh_A), _f64(inv_E), _f64(dE)
        self._check(self.lib.pb_set_em(self.h, int(n_em), int(gamma_off), int(em_off), int(ep_off), int(n_cr),
                                       int(bo.size), _ptr(bo, C.c_int64), _ptr(ba, C.c_double),
                                       _ptr(ie, C.c_double), _ptr(de, C.c_double)), "pb_set_em")

    def set_em_windows(self, Tg, Te, R, dl_step):
        Tg, Te, R, dl = _f64(Tg), _f64(Te), _f64(R), _f64(dl_step)
        self._check(self.lib.pb_set_em_windows(self.h, int(dl.size), _ptr(Tg, C.c_double), _ptr(Te, C.c_double),
                                               _ptr(R, C.c_double), _ptr(dl, C.c_double)), "pb_set_em_windows")

    # -- solve ----------------------------------------------------------
    def solve(self, sched, flags, n_cols, coeff, n_active, state, photon_scale=1.0, init_state=False,
              state_ptr=None, out_cols=None):
        """Run one solve.  ``state`` is an (n, K) float64 host array (in/out)
        unless ``state_ptr`` (a device pointer) is given.  ``out_cols`` (solve
        column -> output column) orders the returned columns."""
        args, keep = self._solve_args(sched, flags, n_cols, coeff, n_active, state, photon_scale, init_state,
                                      state_ptr, out_cols)
        self._check(self.lib.pb_solve(self.h, C.byref(args)), "pb_solve")

    def autotune(self, sched, flags, n_cols, coeff, n_active, state, reps=3, photon_scale=1.0):
        """Search the batched stage's tile parameters on this solve; the fastest stays set.
        Returns the candidates as dicts, the chosen one first."""
        args, keep = self._solve_args(sched, flags, n_cols, coeff, n_active, state, photon_scale, False, None, None)
        out = (TuneChoice * 32)()
        n = C.c_int32(0)
        self._check(self.lib.pb_autotune(self.h, C.byref(args), int(reps), 32, out, C.byref(n)), "pb_autotune")
        return [dict(band_warps=o.band_warps, slab_prefetch=o.slab_prefetch, tma_staging=o.tma_staging,
                     steps_ms=o.steps_ms) for o in out[: n.value]]

    def _solve_args(self, sched, flags, n_cols, coeff, n_active, state, photon_scale, init_state, state_ptr,
                    out_cols):
        keep = []

        def f(a):
            a = _f64(a)
            keep.append(a)
            return _ptr(a, C.c_double)

        def i(a):
            a = _i32a(a)
            keep.append(a)
            return _ptr(a, C.c_int32)

        args = SolveArgs()
        args.n_steps = int(sched.n_steps)
        args.n_windows = int(len(sched.z_window))
        args.n_cols = int(n_cols)
        args.flags = int(flags)
        args.photon_scale = float(photon_scale)
        args.z_window = f(sched.z_window)
        args.window = i(sched.window)
        args.h = f(sched.h)
        args.dldz = f(sched.dldz)
        args.hc = f(sched.hc)
        args.finj = f(sched.finj)
        args.coeff = f(coeff) if coeff is not None else None
        args.n_active = i(n_active)
        if state_ptr is not None:
            args.state = C.cast(C.c_void_p(int(state_ptr)), _d)
            args.state_on_device = 1
        else:
            assert state.dtype == np.float64 and state.flags["C_CONTIGUOUS"]
            args.state = _ptr(state, C.c_double)
            args.state_on_device = 0
        args.init_state = 1 if init_state else 0
        if out_cols is not None:
            args.out_cols = i(out_cols)
        return args, keep

    def operator_pattern(self, n):
        nnz = C.c_int64(0)
        self._check(self.lib.pb_get_operator_pattern(self.h, C.byref(nnz), None, None), "pb_get_operator_pattern")
        ip = np.zeros(n + 1, dtype=np.int64)
        ix = np.zeros(max(nnz.value, 1), dtype=np.int32)
        self._check(self.lib.pb_get_operator_pattern(self.h, C.byref(nnz), _ptr(ip, C.c_int64), _ptr(ix, C.c_int32)),
                    "pb_get_operator_pattern")
        return ip, ix[: nnz.value]

    def window_values(self, w, n, nnz):
        off = np.zeros(max(nnz, 1))
        dg = np.zeros(n)
        kp = np.zeros(n)
        self._check(self.lib.pb_get_window(self.h, int(w), _ptr(off, C.c_double), _ptr(dg, C.c_double),
                                           _ptr(kp, C.c_double)), "pb_get_window")
        return off[:nnz], dg, kp

    def integrate_const(self, d, L_off, z_grid, state):
        d = _f64(d)
        x = np.array(state, dtype=np.float64)
        zg = _f64(z_grid)
        n = d.size
        if L_off is None or L_off.nnz == 0:
            rc = self.lib.pb_integrate_const(self.h, n, _ptr(d, C.c_double), 0, None, None, None,
                                             int(zg.size - 1), _ptr(zg, C.c_double), _ptr(x, C.c_double))
        else:
            ip, ix, v = _i64a(L_off.indptr), _i32a(L_off.indices), _f64(L_off.data)
            rc = self.lib.pb_integrate_const(self.h, n, _ptr(d, C.c_double), int(v.size), _ptr(ip, C.c_int64),
                                             _ptr(ix, C.c_int32), _ptr(v, C.c_double), int(zg.size - 1),
                                             _ptr(zg, C.c_double), _ptr(x, C.c_double))
        self._check(rc, "pb_integrate_const")
        return x

    def integrate_const_noalloc(self, n, d_ptr, nnz, indptr_ptr, indices_ptr, values_ptr, n_steps, z_ptr,
                                state_ptr):
        """Allocation-free constant-operator integration; all pointers are device addresses (ints)."""
        vp = lambda v: None if v is None else C.c_void_p(int(v))
        self._check(self.lib.pb_integrate_const_noalloc(self.h, int(n), vp(d_ptr), int(nnz), vp(indptr_ptr),
                                                        vp(indices_ptr), vp(values_ptr), int(n_steps), vp(z_ptr),
                                                        vp(state_ptr)), "pb_integrate_const_noalloc")

    def eval_exp(self, x):
        """The device exp of the phi functions on ``x`` (float64 array)."""
        x = _f64(x)
        y = np.empty_like(x)
        self._check(self.lib.pb_eval_exp(self.h, int(x.size), _ptr(x, C.c_double), _ptr(y, C.c_double)),
                    "pb_eval_exp")
        return y

    def last_timing(self):
        """(solve_ms, device_ms, steps_ms, launches) of the last solve."""
        a, d, b, n = C.c_double(), C.c_double(), C.c_double(), C.c_int64()
        self._check(self.lib.pb_last_timing(self.h, C.byref(a), C.byref(d), C.byref(b), C.byref(n)),
                    "pb_last_timing")
        return a.value, d.value, b.value, n.value
