"""Autotuning of the batched stage's tile parameters, cached per device and shape.

The bin-blocked batched stage has three tunable choices (``pb_autotune``):
the warps of a band-tile CTA (8: a CTA per SM; 4: half the registers and
shared memory, so it runs beside the bin-local gather), the bin-local
kernel's prefetch depth (1, 2 or 3 row quartets) and its staging (TMA tensor
maps or ``cp.async``).  ``tune(solver)`` times every candidate on the
solver's live operator with a short solve that has all K columns active
(the states are discarded), keeps the fastest on the device context and
records it in a JSON cache keyed by (GPU name, states, coupling entries, K),
so later runs of the same shape apply it without searching.

The cache file is ``$PRINCE_B200_CACHE/autotune.json`` (default
``~/.cache/prince_b200/autotune.json``).
"""

from __future__ import annotations

import json
import os

import numpy as np

from . import _lib
from .schedule import make_schedule, z_grid


def cache_path():
    base = os.environ.get("PRINCE_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "prince_b200"))
    return os.path.join(base, "autotune.json")


def _device_name(device):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def shape_key(solver):
    run = solver.prince_run
    return (f"{_device_name(solver.device)}|n={run.dim_states}|entries={run.int_rates.coupling_mat.nnz}"
            f"|K={len(solver._column_sources())}")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def apply(ctx, choice):
    ctx.set_option(_lib.PB_OPT_BAND_WARPS, int(choice["band_warps"]))
    ctx.set_option(_lib.PB_OPT_SLAB_PREFETCH, int(choice["slab_prefetch"]))
    ctx.set_option(_lib.PB_OPT_TMA_STAGING, int(choice["tma_staging"]))


def tune(solver, steps=16, reps=3, dz=1e-3, path=None, force=False):
    """Pick the stage's tile parameters for ``solver`` (a multi-RHS solver with its
    sources added).  Returns ``(choice, candidates)``; ``candidates`` is ``None``
    when the choice came from the cache."""
    path = path or cache_path()
    key = shape_key(solver)
    table = _load(path)
    ctx = solver._dev.ctx
    if not force and key in table:
        try:  # a choice cached by an older build may name a value this build refuses
            apply(ctx, table[key])
            return table[key], None
        except (RuntimeError, KeyError, TypeError, ValueError):
            pass
    # a short schedule at the end of the solve range, where every column is active
    zg = z_grid(solver.final_z + steps * dz, solver.final_z, dz)
    sched = make_schedule(zg, solver.recomp_z_threshold)
    cols = solver._column_sources()
    K = len(cols)
    srcs = [s for c in cols for s in c]
    if not srcs:
        raise ValueError("add the sources before tuning")
    owner = np.array([k for k, c in enumerate(cols) for _ in c])
    grids = [np.asarray(s.injection_grid, dtype=np.float64) for s in srcs]
    rows = np.unique(np.concatenate([np.flatnonzero(g) for g in grids])).astype(np.int32)
    G = np.stack([g[rows] for g in grids], axis=1)
    order = np.argsort(owner, kind="stable")
    ctx.set_injection(solver._dev.dev_rows(rows), G[:, order], owner[order].astype(np.int32), K)
    solver._set_field(ctx)
    if solver._flags() & _lib.PB_EM_CASCADE:   # the short schedule's own EM windows
        ctx.set_em_windows(*solver._em_windows(sched, dz))
        solver._dev.em_key = None
    coeff = np.ones((sched.n_steps, len(srcs)))
    state = np.empty((solver.dim_states, K))
    cands = ctx.autotune(sched, solver._flags(), K, coeff, np.full(sched.n_steps, K, dtype=np.int32), state,
                         reps=reps)
    choice = {k: cands[0][k] for k in ("band_warps", "slab_prefetch", "tma_staging", "steps_ms")}
    table = _load(path)
    table[key] = choice
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return choice, cands
