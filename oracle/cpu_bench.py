"""Timed CPU samples of the reference algorithm -- TEST/BENCH INFRASTRUCTURE ONLY.

Used by ``bench.py`` for its ``cpu_baseline`` entry and for the reference arm
(``--impl reference``); both call :func:`sample_rate` with the same
arguments, so the two CPU figures of one bench run come from one sampler.

The timed work is the oracle restatement of the reference CPU solver
(``_MultiRHSETD2SolverCPU``: scipy CSR SpMM per ETD2 stage, numpy GEMV fold
per rate window), one solver per worker process, the way several cores run
the reference: the K source columns are split evenly over P worker processes
(64 columns each at K = 512 and P = 8).  One sample advances every worker's
columns ``s_sample`` redshift steps from the top of the grid; the time of each
window refresh (the fold) is measured directly and separated from the time of
the steps.  The full solve of one worker is then

    t_full = S * t_step + W * t_fold,

with S steps and W windows of the real schedule (an extrapolation in steps
and windows only: every column of the workload is in the sample), and the
throughput is K / max over workers of t_full.

Workers are spawned (never forked: the caller may already hold a CUDA
context) and build the run once; samples after the first reuse them.
"""

from __future__ import annotations

import os
import time

import numpy as np

_W = {}


def _init(run_builder, points, dz, thr):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import workloads

    run = getattr(workloads, run_builder)()
    _W.update(run=run, srcs=[[workloads.point_source(run, p)] for p in points], dz=dz, thr=thr)


def _task(job):
    """One worker's sample: its columns, ``s_sample`` steps from ``zi``."""
    cols, zi, s_sample = job
    from oracle import etd2_oracle as O

    run, dz = _W["run"], _W["dz"]
    srcs = [_W["srcs"][i] for i in cols]
    o = O.OracleSolver(run, zi, zi - s_sample * dz, K=len(srcs), thr=_W["thr"])
    fold = []
    refresh = o._refresh

    def timed_refresh(z, first):
        t0 = time.perf_counter()
        refresh(z, first)
        fold.append(time.perf_counter() - t0)

    o._refresh = timed_refresh
    t0 = time.perf_counter()
    o.solve(srcs, dz=dz)
    t_all = time.perf_counter() - t0
    t_fold = float(np.mean(fold))
    t_step = (t_all - float(np.sum(fold))) / s_sample
    return dict(k=len(cols), t_step=t_step, t_fold=t_fold, n_win=len(fold), wall=t_all)


def default_processes(per_process_gb=3.0):
    """Worker count: every host core, up to the memory each worker's run needs
    (the A <= 56 fold kernel alone is 2 GB per worker)."""
    n = os.cpu_count() or 1
    try:
        import psutil

        n = min(n, max(1, int(psutil.virtual_memory().available / (per_process_gb * 2 ** 30))))
    except Exception:
        n = min(n, 8)
    return max(1, n)


class Sampler:
    """A pool of spawned workers holding the run; ``sample()`` times one bounded sample."""

    def __init__(self, run_builder, points, zi, dz, thr, processes):
        import multiprocessing as mp

        os.environ.setdefault("OMP_NUM_THREADS", "1")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        self.K = len(points)
        self.zi = zi
        self.P = max(1, min(int(processes), self.K))
        self.chunks = [c.tolist() for c in np.array_split(np.arange(self.K), self.P) if c.size]
        self.pool = mp.get_context("spawn").Pool(len(self.chunks), initializer=_init,
                                                   initargs=(run_builder, points, dz, thr))

    def sample(self, s_sample):
        jobs = [(c, self.zi, s_sample) for c in self.chunks]
        t0 = time.perf_counter()
        res = self.pool.map(_task, jobs, chunksize=1)
        return res, time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def extrapolate(samples, n_steps, n_windows):
    """(spectra per second, seconds) of a full solve of all sampled columns."""
    K = sum(s["k"] for s in samples)
    t = max(n_steps * s["t_step"] + n_windows * s["t_fold"] for s in samples)
    return K / t, t


def describe(sampler, s_sample, n_steps, n_windows, t_full):
    k = sampler.chunks[0].__len__()
    return (f"CPU oracle of the reference multi-RHS solver (scipy SpMM per stage + numpy fold per window), "
            f"{len(sampler.chunks)} spawned processes x {k} columns (all {sampler.K} columns), "
            f"{s_sample} steps from z={sampler.zi:.3f} with every window refresh timed separately; "
            f"extrapolated in steps and windows to {n_steps} steps and {n_windows} windows "
            f"(t_full={t_full:.1f} s)")
