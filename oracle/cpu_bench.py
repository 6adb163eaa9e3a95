"""Timed CPU samples of the reference algorithm -- TEST/BENCH INFRASTRUCTURE ONLY.

Used by ``bench.py`` for its ``cpu_baseline`` entry and for the reference arm
(``--impl reference``); both call the same sampler with the same arguments,
so the two CPU figures of one bench run come from one measurement method.

What runs (``kind``):

* ``"reference"`` -- PriNCe's own ``MultiRHSPropagationSolverETD2`` (its scipy
  CPU backend, ``_MultiRHSETD2SolverCPU``), imported from the reference
  installed in ``baseline/_ref``, on this workload's run object (which
  provides the reference's run contract: ``get_hadr_jacobian``,
  ``build_split_fold`` / ``fold_split``, the loss objects);
* ``"port"`` -- the restatement in ``oracle/etd2_oracle.py`` when the
  reference is not installed.

One solver per worker process, the way several cores run the reference: the
K source columns are split evenly over P spawned workers.  One sample
advances every worker's columns ``s_sample`` redshift steps from the top of
the grid; each window refresh (the fold) is timed directly and kept apart
from the steps; the first refresh (which also builds the reference's
row-subset fold kernels) separately from the later ones.  A worker's full
solve is then

    t_full = S * t_step + t_first + (W - 1) * t_fold,

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


def reference_available():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return os.path.isdir(os.path.join(root, "baseline", "_ref", "prince_cr"))


def _init(run_builder, points, dz, thr, kind):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import workloads

    run = getattr(workloads, run_builder)()
    if kind == "reference":
        import reference_env

        config = reference_env.load_package()
        config.linear_algebra_backend = "scipy"
        run.backend.linear_algebra_backend = "scipy"
    _W.update(run=run, srcs=[[workloads.point_source(run, p)] for p in points], dz=dz, thr=thr, kind=kind)


def _timed(fn, log):
    def wrapped(*a, **k):
        t0 = time.perf_counter()
        out = fn(*a, **k)
        log.append(time.perf_counter() - t0)
        return out
    return wrapped


def _task(job):
    """One worker's sample: its columns, ``s_sample`` steps from ``zi``."""
    cols, zi, s_sample = job
    run, dz = _W["run"], _W["dz"]
    srcs = [_W["srcs"][i] for i in cols]
    fold = []
    if _W["kind"] == "reference":
        from prince_cr.solvers import MultiRHSPropagationSolverETD2 as RefMulti

        solver = RefMulti(initial_z=zi, final_z=zi - s_sample * dz, prince_run=run, K=len(srcs))
        solver.recomp_z_threshold = _W["thr"]
        for k, src in enumerate(srcs):
            for s in src:
                solver[k].add_source_class(s)
        solver._refresh_z_caches = _timed(solver._refresh_z_caches, fold)
        t0 = time.perf_counter()
        solver.solve(dz=dz)
        t_all = time.perf_counter() - t0
    else:
        from oracle import etd2_oracle as O

        o = O.OracleSolver(run, zi, zi - s_sample * dz, K=len(srcs), thr=_W["thr"])
        o._refresh = _timed(o._refresh, fold)
        t0 = time.perf_counter()
        o.solve(srcs, dz=dz)
        t_all = time.perf_counter() - t0
    t_first = fold[0]
    t_fold = float(np.mean(fold[1:])) if len(fold) > 1 else t_first
    t_step = (t_all - float(np.sum(fold))) / s_sample
    return dict(k=len(cols), t_step=t_step, t_first=t_first, t_fold=t_fold, n_win=len(fold), wall=t_all)


def default_processes(per_process_gb=6.0):
    """Worker count: every host core, up to the memory each worker's run needs
    (the A <= 56 fold kernel is 2 GB per worker, the reference's row-subset
    copy of it another 2 GB)."""
    n = os.cpu_count() or 1
    try:
        import psutil

        n = min(n, max(1, int(psutil.virtual_memory().available / (per_process_gb * 2 ** 30))))
    except Exception:
        n = min(n, 8)
    return max(1, n)


class Sampler:
    """A pool of spawned workers holding the run; ``sample()`` times one bounded sample."""

    def __init__(self, run_builder, points, zi, dz, thr, processes, kind=None):
        import multiprocessing as mp

        os.environ.setdefault("OMP_NUM_THREADS", "1")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        self.kind = kind or ("reference" if reference_available() else "port")
        self.K = len(points)
        self.zi = zi
        self.P = max(1, min(int(processes), self.K))
        self.chunks = [c.tolist() for c in np.array_split(np.arange(self.K), self.P) if c.size]
        self.pool = mp.get_context("spawn").Pool(len(self.chunks), initializer=_init,
                                                   initargs=(run_builder, points, dz, thr, self.kind))

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
    t = max(n_steps * s["t_step"] + s["t_first"] + (n_windows - 1) * s["t_fold"] for s in samples)
    return K / t, t


def describe(sampler, s_sample, n_steps, n_windows, t_full):
    k = sampler.chunks[0].__len__()
    what = ("PriNCe's own MultiRHSPropagationSolverETD2 (scipy CPU backend, installed reference)"
            if sampler.kind == "reference" else
            "CPU restatement of the reference multi-RHS solver (scipy SpMM per stage + numpy fold per window)")
    return (f"{what}, {len(sampler.chunks)} spawned processes x {k} columns (all {sampler.K} columns), "
            f"{s_sample} steps from z={sampler.zi:.3f} with every window refresh timed separately; "
            f"extrapolated in steps and windows to {n_steps} steps and {n_windows} windows "
            f"(t_full={t_full:.1f} s)")
