#!/usr/bin/env python
"""Throughput of the B200 ETD2 propagation core on the A<=56 workload.

One bench step is one batched solve: 512 seeded source-parameter points
(spectral index U[-1.5, 2.5], log10 Rmax/V U[9, 11], H/He/N/Si/Fe fractions
~ Dirichlet(1), evolution (1+z)^m with m ~ U[-3, 5], z_max ~ U[0.5, 1])
propagated from z_max to z = 0 with dz = 1e-3 on the A <= 56 network
(350 species x 96 bins = 33,600 FP64 states, CMB + synthetic CIB).

Prints one JSON line (rank 0):
  value  -- spectra/s with the operator resident on the device, CUDA events
            around each solve on the library stream (photon field, pair
            losses, fold, split and all ETD2 steps);
  e2e    -- spectra/s through the public solver API (host schedule, pinned
            host->device uploads, device->host copy of the result states);
  roofline -- the dominant stage kernel (re-run alone between CUDA events) against
              its measured peak; roofline_kernels lists every stage kernel;
  cpu_baseline -- the CPU oracle of the reference algorithm on a bounded sample;
  plain  -- the one-spectrum-per-launch path on the same operator.

``--impl reference`` times the CPU restatement of the reference solver on the
same workload (bounded samples, extrapolated) and prints its line.

Multi-GPU (torchrun): every rank propagates its own 512 points (weak scaling,
replicas of the operator, no collective in the data path); the reported time
is the maximum over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "A<=56 spectra/s batched vs plain on 1 B200 at 1e-10 rel err; adjoint/forward time"
WORKLOAD = ("A<=56 network: 350 species x 96 bins = 33,600 FP64 states, CMB + 40 K grey-body CIB; "
            "512 source points per batch, z_max~U[0.5,1] -> z=0, dz=1e-3, rate windows every 0.01 in z")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


def _dist(backend=None):
    """(dist, rank, world size, local rank) under torchrun; (None, 0, 1, 0) alone.
    The backend is NCCL on GPUs (gloo for host-side tests)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    backend = backend or os.environ.get("PB_DIST_BACKEND", "nccl")
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=timedelta(seconds=60))
    return dist, rank, ws, local


def _max_over_ranks(dist, local, vals):
    """Element-wise maximum over ranks (the device times of the slowest rank)."""
    if dist is None:
        return vals
    import torch

    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def step_bytes(n, nnz_m, n_inj, n_act):
    """Algorithmic HBM bytes of one ETD2 step (both stages) with n_act columns:
    state traffic 48 n K (read x, write a and F(x); read a and F(x), write x),
    the operator twice (8 B value + 4 B column per entry, 4 B row pointer),
    8 per-row FP64 vectors and the injection rows read in both stages."""
    return 48.0 * n * n_act + 2 * (12.0 * nnz_m + 4.0 * (n + 1)) + 8.0 * n * 8 + 16.0 * n_inj * n_act


def rank_points(run, points, rank, z_range):
    """The source points of one rank: every rank propagates its own seeded batch."""
    from workloads import draw_points

    return draw_points(run, points, seed=1000 + rank, z_range=z_range)


def workload_config(run, sched, points, ws, nnz_m):
    """The ``config`` object of both arms' lines."""
    return {
        "workload": WORKLOAD,
        "points_per_gpu": points,
        "n_states": run.dim_states,
        "coupling_entries": int(run.int_rates._batch_matrix.shape[0]),
        "offdiag_nnz": int(nnz_m),
        "n_steps": sched.n_steps,
        "n_windows": int(len(sched.z_window)),
        "parallelism": f"replicas x{ws} (columns sharded, no collective)",
        "l2": "state buffers 3 x 138 MB exceed the 126 MB L2 between solves",
    }


def run_b200(args, dist, rank, ws, local):
    import torch
    from prince_b200.solvers import MultiRHSPropagationSolverETD2, UHECRPropagationSolverETD2
    from workloads import draw_points, network_run, point_source

    torch.cuda.set_device(local)
    run = network_run()
    pts = rank_points(run, args.points, rank, args.z_range)
    zi = max(p["zmax"] for p in pts)
    solver = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=args.points, device=local)
    for k, p in enumerate(pts):
        solver[k].add_source_class(point_source(run, p))
    tuned = None
    if args.band_warps:
        from prince_b200 import _lib
        solver._dev.ctx.set_option(_lib.PB_OPT_BAND_WARPS, args.band_warps)
    elif args.autotune:
        import tempfile
        from prince_b200 import autotune
        # a fresh search on this box (a scratch cache), reported beside the line
        with tempfile.TemporaryDirectory() as tdir:
            choice, cands = autotune.tune(solver, path=os.path.join(tdir, "autotune.json"), force=True)
        default = next((c for c in cands if c["band_warps"] == 8 and c["slab_prefetch"] == 2
                        and c["tma_staging"] == 1), None)
        tuned = {"choice": {k: choice[k] for k in ("band_warps", "slab_prefetch", "tma_staging")},
                 "tuned_steps_ms": choice["steps_ms"],
                 "default_steps_ms": default["steps_ms"] if default else None,
                 "candidates": len(cands), "search": "16 fully active steps per candidate, fastest of 3"}

    for _ in range(args.warmup):
        solver.solve(dz=1e-3)
    # bytes model inputs from the warm solve
    sched, K, coeff, rows, G, src_col, n_active, perm, use_inj = solver._prepare(1e-3)
    ip, ix = solver.operator_pattern()
    nnz_m = int(ix.size)
    n = run.dim_states
    bytes_solve = sum(step_bytes(n, nnz_m, rows.size, int(a)) for a in n_active if a > 0)
    step_launches = 2 * sum(1 for a in n_active if a > 0)

    clocks = Clocks(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_ms, steps_ms, wall, launches = [], [], [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        solver.solve(dz=1e-3)
        wall.append(time.perf_counter() - t0)
        solve_ms, device_ms, s_ms, nl = solver.last_timing
        dev_ms.append(device_ms)
        steps_ms.append(s_ms)
        launches += nl
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    t_dev = sum(dev_ms) / 1e3
    t_wall = sum(wall)
    t_dev, t_wall = _max_over_ranks(dist, local, [t_dev, t_wall])
    spectra = args.points * args.steps * ws
    value = spectra / t_dev
    e2e = spectra / t_wall

    # per-kernel rooflines (re-runs the last batched solve's final step)
    kern = kernel_rooflines(solver, run, sched, n_active, rows.size)

    # plain path: one spectrum per launch on the same operator
    plain = None
    if args.plain > 0:
        ps = UHECRPropagationSolverETD2(initial_z=pts[0]["zmax"], final_z=0.0, prince_run=run, device=local)
        ps.add_source_class(point_source(run, pts[0]))
        for _ in range(2):
            ps.solve(dz=1e-3)
        pm = []
        for i in range(args.plain):
            p = pts[i % len(pts)]
            ps.initial_z = p["zmax"]
            ps.list_of_sources = [point_source(run, p)]
            ps.solve(dz=1e-3)
            pm.append(ps.last_timing[1])
        plain = len(pm) / (sum(pm) / 1e3)

    adj = adjoint_timing(run, pts, zi, local) if args.adjoint else None
    cem = None
    if args.coupled_em and ws == 1:   # one GPU only: the other ranks would wait for it at the final barrier
        del solver
        cem = coupled_em_timing(local, adjoint=bool(args.adjoint))

    pk, pk_kind = _peaks()
    avg_steps_ms = statistics.mean(steps_ms)
    achieved = bytes_solve / (avg_steps_ms / 1e3) / 1e9
    h2d = (sched.n_steps * (4 * 8 + 2 * 4) + len(sched.z_window) * 8 + coeff.size * 8 + G.size * 8
           + rows.size * 4 + src_col.size * 4)
    d2h = n * K * 8
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "spectra/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded synthetic photo-nuclear model and source points)",
        "config": workload_config(run, sched, args.points, ws, nnz_m),
        "e2e": {"value": e2e, "unit": "spectra/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": kern["dominant"] if kern else None,
        "roofline_kernels": kern["kernels"] if kern else None,
        "step_stream": {"bytes_per_solve": bytes_solve, "steps_ms_per_solve": avg_steps_ms,
                        "achieved_gbs": achieved, "peak_gbs": pk, "peak_source": pk_kind,
                        "note": "whole step loop (all stage kernels, both streams) against the HBM copy peak"},
        "gpu_launches": int(launches),
        "plain_spectra_per_s": plain,
        "batched_over_plain": (value / ws / plain) if plain else None,
    }
    if adj:
        fwd_wall = t_wall / args.steps
        adj["forward_s"] = fwd_wall
        adj["adjoint_over_forward"] = adj["adjoint_s"] / fwd_wall
        adj["gradient_over_forward"] = adj["gradient_s"] / fwd_wall
        adj["gradient_source_params_only_over_forward"] = adj["gradient_source_params_only_s"] / fwd_wall
        line["adjoint"] = adj
    if tuned:
        line["autotune"] = tuned
    if cem:
        line["coupled_em"] = cem
    if clk:
        line["clocks"] = clk
    return line, run, pts, zi, sched


def ncu_traffic():
    """DRAM bytes per launch of each kernel at K = 512, read from the committed ncu
    summaries under ``profiles/`` (the tables' "DRAM traffic per launch (MB)" /
    "DRAM bytes per launch (MB)" rows, one column per kernel)."""
    import glob
    import re

    out = {}
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*_512pts_*.md"))):
        header = None
        for line in open(path):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if line.startswith("| metric"):
                header = cells
            elif header and re.match(r"DRAM (traffic|bytes) per launch \(MB\)", cells[0]):
                for name, val in zip(header[1:], cells[1:]):
                    try:
                        out.setdefault(name.split("<")[0].strip(), float(val) * 1e6)
                    except ValueError:
                        pass
    return out


def kernel_rooflines(solver, run, sched, n_active, n_inj):
    """Per-kernel rooflines of the bin-blocked stage at full activity.

    The last step of the solve has every column active.  Each kernel of its
    two stages is re-run alone between CUDA events on the library stream
    (``pb_profile_stage``); achieved = algorithmic bytes (or useful FP64 flops)
    per launch / mean launch time.  Algorithmic bytes per launch, K columns,
    n states, ns bin-local rows, E entries of the bin-local rows:
      k_fd_dense    read v and kappa, write D_off (kappa v):  16 n K + 8 n
                    (k_fd, the table-driven form, where the stencil does not fit)
      k_slab        read v (all rows), entries (12 E), FD term, row factors;
                    stage 1 writes a and F(x), stage 2 reads F(x), writes x:
                    8 n K + 12 E + 24 ns K + 24 ns
      k_band        useful flops 2 nnz_band K on the FP64 tensor pipe (DMMA)
      k_band_finish read the group partials and the band rows' inputs.
    """
    from prince_b200 import _lib

    ctx = solver._dev.ctx
    if not ctx.info(_lib.PB_INFO_LAST_BLOCKED):
        return None
    K = int(n_active[-1])
    step = int(sched.n_steps - 1)
    n = run.dim_states
    ns = ctx.info(_lib.PB_INFO_SLAB_ROWS)
    nent = ctx.info(_lib.PB_INFO_SLAB_ENTRIES)
    nnz_band = ctx.info(_lib.PB_INFO_BAND_ENTRIES)
    t1 = ctx.profile_stage(step, 1, reps=5)
    t2 = ctx.profile_stage(step, 2, reps=5)
    ms = [(a + b) / 2 for a, b in zip(t1, t2)]
    hbm, hbm_kind = _peaks()
    fp64 = ctx.fp64_peak()
    fd_name = "k_fd_dense" if ctx.info(_lib.PB_INFO_FD_DENSE) else "k_fd"
    kb = {
        fd_name: 16.0 * n * K + 8.0 * n,
        "k_slab": 8.0 * n * K + 12.0 * nent + 24.0 * ns * K + 24.0 * ns,
    }
    traffic = ncu_traffic() if K == 512 else {}
    kernels = []
    for name, t in ((fd_name, ms[0]), ("k_slab", ms[1])):
        if t > 0:
            a = kb[name] / (t * 1e-3) / 1e9
            kernels.append({"kernel": name, "bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                            "frac": a / hbm, "traffic": traffic.get(name),
                            "launch_us": t * 1e3,
                            "algorithmic_bytes": kb[name], "peak_source": hbm_kind})
    if ms[2] > 0:
        a = 2.0 * nnz_band * K / (ms[2] * 1e-3) / 1e12
        kernels.append({"kernel": "k_band", "bound": "tensor", "achieved": a, "peak": fp64, "unit": "TFLOP/s",
                        "frac": a / fp64, "traffic": traffic.get("k_band_tma", traffic.get("k_band")),
                        "traffic_unit": "bytes", "launch_us": ms[2] * 1e3,
                        "algorithmic_flops": 2.0 * nnz_band * K,
                        "peak_source": "measured FP64 DMMA peak (pb_fp64_peak, register-only kernel)"})
    if ms[3] > 0:
        kernels.append({"kernel": "k_band_finish", "launch_us": ms[3] * 1e3})
    timed = [k for k in kernels if "frac" in k]
    dominant = dict(max(timed, key=lambda k: k["launch_us"]))
    dominant["share_of_stage"] = dominant["launch_us"] / (sum(ms) * 1e3)
    return {"dominant": dominant, "kernels": kernels}


def adjoint_timing(run, pts, zi, device):
    """Gradient of the flux loss of all points: the squared log-ratio of
    each point's z = 0 all-particle flux to a target flux from one hidden
    parameter point, summed over bins above 10^9.5 GeV.  Timed: the
    forward with checkpoints every 32 steps (parameters -> grids on the host,
    states on the device), the loss on the device, and the backward (device
    adjoint plus the parameter chain rule), against the plain forward time."""
    import torch
    from prince_b200 import adjoint as AD
    from workloads import draw_points

    species = [p for p in pts[0]["species"]]

    def tensors(ps, grad=True):
        return {"gamma": torch.tensor([p["gamma"] for p in ps], requires_grad=grad),
                "lg_rmax": torch.tensor([np.log10(p["rmax"]) for p in ps], requires_grad=grad),
                "frac": torch.tensor(np.array([p["frac"] for p in ps]), requires_grad=grad),
                "m": torch.tensor([p["m"] for p in ps], requires_grad=grad)}

    hidden = draw_points(run, 1, seed=4242, z_range=(1.0, 1.0))
    sbh = AD.SourceBatch(run, species, z_max=[hidden[0]["zmax"]], initial_z=hidden[0]["zmax"])
    th = tensors(hidden, grad=False)
    with torch.no_grad():
        Xh = AD.PropagateFunction.apply(sbh.grids(th["gamma"], th["lg_rmax"], th["frac"]),
                                        sbh.coefficients(th["m"]), torch.tensor(1.0, dtype=torch.float64),
                                        sbh.plan(hidden[0]["zmax"], device=device))
        target = AD.group_flux(run, Xh)[1][:, 0]
    sb = AD.SourceBatch(run, species, z_max=[p["zmax"] for p in pts], initial_z=zi)
    plan = sb.plan(zi, device=device, ckpt_every=32)
    t = tensors(pts)
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    fwd, bwd, tot = [], [], []
    for rep in range(2):
        for v in list(t.values()) + [scale]:
            v.grad = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G = sb.grids(t["gamma"], t["lg_rmax"], t["frac"])
        coeff = sb.coefficients(t["m"])
        X = AD.PropagateFunction.apply(G, coeff, scale, plan)
        loss = AD.log_ratio_loss(run, X, target).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        fwd.append(t1 - t0)
        bwd.append(t2 - t1)
        tot.append(t2 - t0)
    grads_finite = all(bool(torch.isfinite(v.grad).all()) for v in list(t.values()) + [scale])
    # the same loss differentiated with respect to the 8 source parameters only
    # (the photon scale held fixed): the sweep records the operator factors
    # without recomputing the states
    t2s = tensors(pts)
    fixed = torch.tensor(1.0, dtype=torch.float64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X = AD.PropagateFunction.apply(sb.grids(t2s["gamma"], t2s["lg_rmax"], t2s["frac"]), sb.coefficients(t2s["m"]),
                                   fixed, plan)
    AD.log_ratio_loss(run, X, target).sum().backward()
    torch.cuda.synchronize()
    src_only = time.perf_counter() - t0
    return {"points": len(pts), "ckpt_every": 32, "loss": "sum_k sum_{E>10^9.5 GeV} ln(F_k/T)^2",
            "forward_ckpt_s": fwd[-1], "adjoint_s": bwd[-1], "gradient_s": tot[-1],
            "params_per_point": 8, "with_photon_scale": True, "grads_finite": grads_finite,
            "gradient_source_params_only_s": src_only}


def coupled_em_timing(device, points=2048, adjoint=True):
    """The coupled EM cascade at scale: the A <= 56 network with the co-evolved EM cascade -- gamma and
    e+- on the decoupled 128-bin EM grid (1e-3 to 1e14 GeV), pair production and
    inverse Compton on CMB + the synthetic CIB (transfer and Bethe-Heitler
    shape built on the device for every rate window) -- over 2048 seeded
    points with z_max ~ U[0.5, 4].  Timed: the EM build of all windows, one
    forward solve (device events and wall clock), and the gradient of a loss
    on the z = 0 all-particle flux and photon spectrum with respect to the
    8 source parameters of every point (the adjoint through the EM hook)."""
    import torch
    from prince_b200 import adjoint as AD
    from prince_b200.schedule import make_schedule, z_grid
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import draw_points, em_network_run, point_source

    t0 = time.perf_counter()
    run = em_network_run()
    pts = draw_points(run, points, seed=5000, z_range=(0.5, 4.0))
    zi = max(p["zmax"] for p in pts)
    sched = make_schedule(z_grid(zi, 0.0, 1e-3), run.backend.update_rates_z_threshold)
    solver = MultiRHSPropagationSolverETD2(initial_z=zi, final_z=0.0, prince_run=run, K=points, device=device)
    for k, p in enumerate(pts):
        solver[k].add_source_class(point_source(run, p))
    setup_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run.em_cascade_model.prefetch([float(z) for z in sched.z_window])
    torch.cuda.synchronize()
    em_build_s = time.perf_counter() - t0
    solver.solve(dz=1e-3)   # warm-up: operator set-up and graph capture
    t0 = time.perf_counter()
    solver.solve(dz=1e-3)
    wall = time.perf_counter() - t0
    solve_ms, device_ms, steps_ms, launches = solver.last_timing
    sched_, K, coeff, rows, G, src_col, n_active, perm, use_inj = solver._prepare(1e-3)
    col_steps = int(np.sum(n_active))
    out = {"workload": "A<=56 network + gamma/e+- on a 128-bin EM grid (1e-3-1e14 GeV), CMB + synthetic CIB, "
                       "2048 points, z_max ~ U[0.5,4], dz = 1e-3",
           "n_states": run.dim_states, "em_bins": run.em_grid.d, "points": points, "steps": int(sched.n_steps),
           "windows": len(sched.z_window), "column_steps": col_steps,
           "setup_s": setup_s, "em_build_s": em_build_s, "em_build_windows": len(sched.z_window),
           "forward_device_s": device_ms / 1e3, "forward_steps_s": steps_ms / 1e3, "forward_wall_s": wall,
           "spectra_per_s": points / (device_ms / 1e3), "spectra_per_s_e2e": points / wall,
           "gpu_launches": int(launches)}
    if adjoint:
        species = list(pts[0]["species"])
        hidden = draw_points(run, 1, seed=4243, z_range=(2.0, 2.0))

        def tensors(ps, grad=True):
            return {"gamma": torch.tensor([p["gamma"] for p in ps], requires_grad=grad),
                    "lg_rmax": torch.tensor([np.log10(p["rmax"]) for p in ps], requires_grad=grad),
                    "frac": torch.tensor(np.array([p["frac"] for p in ps]), requires_grad=grad),
                    "m": torch.tensor([p["m"] for p in ps], requires_grad=grad)}

        one = torch.tensor(1.0, dtype=torch.float64)
        sbh = AD.SourceBatch(run, species, z_max=[hidden[0]["zmax"]], initial_z=hidden[0]["zmax"])
        th = tensors(hidden, grad=False)
        with torch.no_grad():
            Xh = AD.PropagateFunction.apply(sbh.grids(th["gamma"], th["lg_rmax"], th["frac"]),
                                            sbh.coefficients(th["m"]), one,
                                            sbh.plan(hidden[0]["zmax"], device=device))
            tgt_cr = AD.group_flux(run, Xh)[1][:, 0]
            g = run.spec_man.pdgid2sref[22]
            tgt_g = Xh[g.lidx():g.uidx(), 0]
        sb = AD.SourceBatch(run, species, z_max=[p["zmax"] for p in pts], initial_z=zi)
        ck = 128
        plan = sb.plan(zi, device=device, ckpt_every=ck)
        t = tensors(pts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        X = AD.PropagateFunction.apply(sb.grids(t["gamma"], t["lg_rmax"], t["frac"]), sb.coefficients(t["m"]),
                                       one, plan)
        loss = (AD.log_ratio_loss(run, X, tgt_cr) + AD.photon_log_ratio_loss(run, X, tgt_g)).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out["adjoint"] = {"loss": "sum_k [sum_{E>10^9.5} ln(F_k/T)^2 + sum_{0.1<=E<=1e3 GeV} ln(n_gamma,k/T_gamma)^2]",
                          "ckpt_every": ck, "params_per_point": 8, "with_photon_scale": False,
                          "forward_ckpt_s": t1 - t0, "adjoint_s": t2 - t1, "gradient_s": t2 - t0,
                          "gradient_over_forward": (t2 - t0) / wall,
                          "grads_finite": all(bool(torch.isfinite(v.grad).all()) for v in t.values())}
    return out


CPU_SAMPLE_STEPS = 20   # two rate windows at dz = 1e-3 and the 0.01 refresh threshold


def cpu_line(pts, zi, sched, processes=None, sampler=None):
    """The CPU oracle of the reference solver on a bounded sample of this workload."""
    from oracle import cpu_bench

    own = sampler is None
    if own:
        sampler = cpu_bench.Sampler("network_run", pts, zi, 1e-3, 0.01,
                                    processes or cpu_bench.default_processes())
    try:
        samples, wall = sampler.sample(CPU_SAMPLE_STEPS)
    finally:
        if own:
            sampler.close()
    rate, t_full = cpu_bench.extrapolate(samples, sched.n_steps, len(sched.z_window))
    return {"value": rate, "unit": "spectra/s", "cores": len(sampler.chunks), "kind": sampler.kind,
            "sample": cpu_bench.describe(sampler, CPU_SAMPLE_STEPS, sched.n_steps, len(sched.z_window), t_full),
            "sample_wall_s": wall}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--points", type=int, default=512)
    ap.add_argument("--plain", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--adjoint", type=int, default=1, help="also time the adjoint gradient (1/0)")
    ap.add_argument("--coupled-em", type=int, default=1,
                    help="also time the coupled EM cascade workload, forward and gradient (1/0)")
    ap.add_argument("--autotune", type=int, default=1, help="search the stage's tile choices before timing (1/0)")
    ap.add_argument("--band-warps", type=int, default=0, choices=[0, 4, 8],
                    help="warps of a band-tile CTA (0: the library default)")
    ap.add_argument("--z-range", default="0.5,1.0",
                    help="z_max range of the source points (smaller cases for profiling)")
    args = ap.parse_args()
    args.z_range = tuple(float(v) for v in args.z_range.split(","))

    if args.impl == "reference":
        return reference_arm(args)

    dist, rank, ws, local = _dist()
    line, run, pts, zi, sched = run_b200(args, dist, rank, ws, local)
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_line(pts, zi, sched)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def reference_arm(args):
    """The reference's CPU algorithm (its restatement in ``oracle/``) on the host cores.

    Each step is one bounded sample of the workload (every column, 20 redshift
    steps, window refreshes timed apart) by the same sampler as the GPU arm's
    ``cpu_baseline``; ``value`` is the mean extrapolated full-solve throughput
    over the timed steps and ``ms_per_step`` the mean wall time of one sample.
    """
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from prince_b200.schedule import make_schedule, z_grid
    from workloads import network_run
    from oracle import cpu_bench

    from oracle import etd2_oracle as O

    run = network_run()
    pts = rank_points(run, args.points, 0, args.z_range)
    zi = max(p["zmax"] for p in pts)
    sched = make_schedule(z_grid(zi, 0.0, 1e-3), run.backend.update_rates_z_threshold)
    probe = O.OracleSolver(run, zi, 0.0, K=1)
    probe._refresh(zi, first=True)    # the off-diagonal pattern of the first window
    config = workload_config(run, sched, args.points, ws, probe.M_off.nnz)
    del run, probe
    sampler = cpu_bench.Sampler("network_run", pts, zi, 1e-3, 0.01, cpu_bench.default_processes())
    vals, walls = [], []
    try:
        for i in range(args.warmup + args.steps):
            samples, wall = sampler.sample(CPU_SAMPLE_STEPS)
            rate, t_full = cpu_bench.extrapolate(samples, sched.n_steps, len(sched.z_window))
            if i >= args.warmup:
                vals.append(rate)
                walls.append(wall)
    finally:
        sampler.close()
    value = statistics.mean(vals)
    line = {
        "metric": METRIC, "value": value, "unit": "spectra/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(walls) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded synthetic photo-nuclear model and source points)",
        "config": config,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "spectra/s", "cores": len(sampler.chunks), "kind": sampler.kind,
                         "sample": "per step: " + cpu_bench.describe(sampler, CPU_SAMPLE_STEPS, sched.n_steps,
                                                                     len(sched.z_window), t_full),
                         "spread": [min(vals), max(vals)]},
        "e2e": {"value": value, "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_note": "a step is one bounded CPU sample; ms_per_step is its wall time",
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
