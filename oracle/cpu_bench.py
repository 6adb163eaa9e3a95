"""Timed CPU samples of the reference algorithm -- TEST/BENCH INFRASTRUCTURE ONLY.

Used by ``bench.py`` for its ``cpu_baseline`` entry and for the reference
arm (``--impl reference``): the oracle restatement of the reference CPU
solver (scipy CSR SpMM per ETD2 stage, numpy GEMV fold per window) is run on
a bounded sample of the workload and extrapolated to a full solve.

The sample of one measurement: ``k_sample`` source columns, ``s_sample``
redshift steps starting at the top of the grid (their windows' folds
included).  The per-step cost of the SpMM path grows linearly with the
number of columns, the per-window fold does not, so a full solve of ``K``
columns over ``S`` steps and ``W`` windows is extrapolated as

    t_full = S * t_step(k_sample) * K / k_sample + W * t_fold.

``processes > 1`` runs that many independent samples in spawned worker
processes (each one its own column subset and fold) and reports the
aggregate throughput, which is how the reference solver uses several cores.
"""

from __future__ import annotations

import os
import time

import numpy as np


def _sample(args):
    """Run one bounded oracle sample in this process; returns timing components."""
    (run_builder, points, zi, dz, s_sample, thr) = args
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import etd2_oracle as O
    import workloads

    run = getattr(workloads, run_builder)()
    srcs = [[workloads.point_source(run, p)] for p in points]
    o = O.OracleSolver(run, zi, zi - s_sample * dz, K=len(srcs), thr=thr)
    # time the fold of one window separately
    t0 = time.perf_counter()
    o._refresh(zi, first=True)
    t_fold = time.perf_counter() - t0
    o.trace.windows.clear()
    t0 = time.perf_counter()
    o.solve(srcs, dz=dz)
    t_all = time.perf_counter() - t0
    n_win = len(o.trace.windows)
    t_steps = max(t_all - n_win * t_fold, 1e-9)
    return dict(t_fold=t_fold, t_step=t_steps / s_sample, n_win=n_win, k=len(points))


def measure(run_builder, points, zi, dz, s_sample, thr, processes=1):
    """Time ``processes`` parallel samples; each gets ``len(points) // processes`` columns."""
    if processes <= 1:
        return [_sample((run_builder, points, zi, dz, s_sample, thr))]
    import multiprocessing as mp

    chunks = [c for c in np.array_split(np.arange(len(points)), processes) if c.size]
    jobs = [(run_builder, [points[i] for i in c], zi, dz, s_sample, thr) for c in chunks]
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(jobs)) as pool:
        return pool.map(_sample, jobs)


def extrapolate(samples, K_total, n_steps, n_windows):
    """Spectra per second of a full solve from per-process samples."""
    P = len(samples)
    k_per = K_total / P
    t = max(n_steps * s["t_step"] * k_per / s["k"] + n_windows * s["t_fold"] for s in samples)
    return K_total / t, t
