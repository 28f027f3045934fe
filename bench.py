#!/usr/bin/env python
"""Benchmark: implicit time steps of the 3D lens problem on B200 (plain FP64 path by default).

A step is one implicit-Euler time step (dt = 250 s): a full Newton solve (ECFV+AD linearization,
BiCGStab + red-black block ILU(0), FP64 update) of the 256 x 256 x 128 lens problem (8.39 M
cells), starting from the hydrostatic state. W warm-up steps advance the simulation, then K steps
are timed with CUDA events on the library's stream, bracketed by a barrier and a synchronize.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--precision mixed]

Prints one JSON line. value = Mcells per second of implicit time steps (cells x steps / time);
ms_per_step and s_per_step carry the time per step. Under torchrun every rank runs its own
permeability realization (independent problems, no data-path collective: weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ewoms-numerics_b200"))

import numpy as np  # noqa: E402

METRIC = "s per implicit time step, plain FP64 vs learned+mixed (same Newton tol); Mcells/s"
FALLBACK_HBM_GBS = 6650.0
# The reference's own CPU step on the 256x256x128 workload is composed from timed phases (an
# 8.39 M-cell implicit step of the sequential natural-order ILU(0) BiCGStab takes over an hour).
# Its iteration counts: Newton per step as measured on the device for this workload (steps 4-6 of
# the plain path: 11, 11, 10; the oracle takes the same Newton counts as the device in every
# parity test), and BiCGStab per step = the device's box-8-colour count (3556, 3512, 3133) times
# the natural order's share of it, 2163 / 2461 = 0.879 (the oracle's first implicit step of the
# 128x128x64 lens in both orders).
NATURAL_OVER_BOX8 = 2163.0 / 2461.0
REF_NEWTON_PER_STEP = (11 + 11 + 10) / 3.0
REF_BICGSTAB_PER_STEP = (3556 + 3512 + 3133) / 3.0 * NATURAL_OVER_BOX8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--ensemble-members", type=int, default=64)
    ap.add_argument("--ensemble-steps", type=int, default=3)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-scheduler", default="device", choices=["device", "host"],
                    help="device: Newton / step decisions on the device, supersteps in a CUDA graph WHILE node")
    ap.add_argument("--no-vcfv", action="store_true")
    ap.add_argument("--no-conv", action="store_true")
    ap.add_argument("--conv", action="store_true", help="time only the guess network's tensor-core convolutions")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# distributed plumbing


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# clocks


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# algorithmic bytes per kernel launch (FP64 s = 8, FP32 s = 4)


def mixed_opts(ewg):
    """The mixed-precision form: FP32 Jacobian, ILU(0) and BiCGStab solve each Newton correction
    to a relative 1e-3 (the reference's default LinearSolverTolerance); the FP64 defect check
    accepts the correction once the FP64 defect is reduced by 1e-2 (at most 3 FP32 passes).
    Residual, update and the Newton test (1e-8) stay FP64: Newton is the defect correction."""
    return ewg.default_solve_opts(precision=ewg.PRECISION_MIXED, linear_solver_tolerance=1e-2,
                                  inner_tolerance=1e-3, max_defect_iterations=3, linear_solver_max_iterations=5000)


def geometry(n):
    nx, ny, nz = n
    N = nx * ny * nz
    F = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)
    return N, F


def cross_box_faces(n):
    """Interior faces between two 2x2x2 boxes of the box-8-colour order (the rest lie inside a box)."""
    nx, ny, nz = n
    return (nx // 2 - 1) * ny * nz + nx * (ny // 2 - 1) * nz + nx * ny * (nz // 2 - 1)


def kernel_bytes(name, N, F, s_mat=8, s_vec=8, b8=False, Fx=None):
    """Bytes a launch must move at minimum in the band layout (no index arrays): every matrix
    block and vector entry it needs read once, every output written once. b8: the solve runs its
    ILU(0) in the box-8-colour order (Fx = faces between boxes): per sweep eight colour launches,
    and the SpMV after a preconditioner application reads only the earlier neighbours' blocks."""
    Nh = N // 2
    blk, vec = 4 * s_mat, 2 * s_vec
    if b8:
        Fx = F // 2 if Fx is None else Fx
        table8 = {
            # forward, per launch (a sweep is 8 colour launches): L blocks of the earlier
            # neighbours, d in, w out, the earlier neighbours' w across box faces (within a box they
            # stay in registers)
            "b8_forward": (F * blk + N * vec * 2 + Fx * vec) / 8,
            # backward, per launch: blocks of the later neighbours, inverted pivots, w in, y out, the
            # later neighbours' y across box faces
            "b8_backward": (F * blk + N * blk + N * vec * 2 + Fx * vec) / 8,
            # v = relax w + E y + sum of the earlier neighbours' blocks times y; r0hat (or s) for
            # the dot products
            "bicg_spmv_alpha": F * blk + N * blk + N * vec * 4,
            "bicg_spmv_omega": F * blk + N * blk + N * vec * 4,
            # the Jacobian into box-8 order (7 bands) and a vector conversion
            "b8_layout": None,
        }
        if name in table8:
            return table8[name]
    table = {
        # linearization: x, lens flag in; the neighbours' intensive quantities out (p_c, lambda_w,
        # lambda_n); the 3D assembly evaluates its own cell's
        "intensive": N * (16 + 1) + N * 24,
        # x, S_old, K, lens, the cached p_c / lambda_w / lambda_n in; r and the Jacobian column
        # (diag + 2 per face) out
        "assemble": N * (16 + 16 + 8 + 1 + 24) + N * (16 + 32) + F * 64,
        # black rows: own d, red d, L blocks (one per face), Dinv; y_b out
        "ilu_black_apply": Nh * (vec + blk + vec) + Nh * vec + F * blk,
        # red rows: own d, black y, A_rb blocks (one per face), Dinv; y_r out
        "ilu_red_apply": Nh * (vec + blk + vec) + Nh * vec + F * blk,
        "jacobi_apply": N * (vec + blk + vec),
        # v = A y (all blocks, y) + r0hat for the dot; v out
        "bicg_spmv_alpha": (N + 2 * F) * blk + N * vec * 3,
        "bicg_spmv_omega": (N + 2 * F) * blk + N * vec * 3,
        "spmv": (N + 2 * F) * blk + N * vec * 2,
        "bicg_p": N * vec * 4,
        "bicg_hs": N * vec * 6,
        "bicg_xr": N * vec * 7,
        "bicg_init": N * vec * 6,
        "newton_update": N * 16 * 3,
        "diag_inverse": N * blk * 2,
        "ilu_black_factor": Nh * (2 * blk) + F * blk * 3 + Nh * blk,
    }
    return table.get(name)


def lin_bytes(N, F, s=8):
    """B_lin of the linearization (both kernels): N (2s x + 2s S_old + 8 K + 1 + 2s r + 4s J_ii)
    + F (2 x 4s J_ij)."""
    return N * (2 * s + 2 * s + 8 + 1 + 2 * s + 4 * s) + F * (8 * s)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ncu DRAM bytes (read + write) per launch of the FP64 kernels at the full 256x256x128 workload:
# the --set full capture of the 128x128x64 case (profiles/kernels_lens3d_128x128x64_fp64_ncu.md)
# scaled by the cell count (x 8); the traffic of these streaming kernels grows in proportion.
NCU_TRAFFIC = {
    "bicg_spmv_omega": (281.86e6 + 17.78e6) * 8,
    "bicg_spmv_alpha": (281.20e6 + 14.63e6) * 8,
    "ilu_black_apply": (133.48e6 + 4.35e6) * 8,
    "ilu_red_apply": (133.50e6 + 4.21e6) * 8,
    "bicg_xr": (83.93e6 + 3.81e6) * 8,
}
# with the box-8-colour ILU(0): ncu dram__bytes_read.sum + dram__bytes_write.sum of the 192x192x96
# case (3,538,944 cells; profiles/traffic_lens3d_192x192x96_fp64_box8.md) scaled by the cell count
# (x 2.370); the sweeps' figures are a sweep's traffic over its 8 colour launches, like their
# algorithmic bytes (a written colour stays in L2 for the next launches to read)
NCU_TRAFFIC_B8 = {
    "b8_backward": 594.6e6 / 8 * 2.370,
    "b8_forward": 479.6e6 / 8 * 2.370,
    "bicg_spmv_alpha": 734.6e6 * 2.370,
    "bicg_spmv_omega": 737.1e6 * 2.370,
    "bicg_xr": 358.1e6 * 2.370,
    "bicg_hs": 285.6e6 * 2.370,
    "bicg_p": 195.7e6 * 2.370,
}


# ---------------------------------------------------------------------------------------------
# CPU baseline: the oracle restatement on the host cores


def cpu_vcfv_linearization(n=32, seed=0):
    """The oracle's vertex-centred linearization on an n^3-element sample of the 3D lens problem
    at the bench's drained-top state: the element loop runs on one thread (its scatter into shared
    vertex rows is what the reference serialises with its linearization lock)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ewg
    import oracle
    oracle.build()
    case = ewg.vcfv_case(ewg.lens3d_case(n, n, n, seed=seed), seed=seed)
    o = oracle.VcfvOracle(case, nthreads=os.cpu_count() or 1)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.default_rng(seed)
    top = ewg.vertex_positions(case.grid)[1] > 0.8 * case.grid.ly
    x[top, 1] = 1.0 - rng.uniform(0.0, 0.4, int(top.sum()))
    o.set_solution(0, x)
    t0 = time.perf_counter()
    o.linearize(250.0, 1)
    el = time.perf_counter() - t0
    return {"mvertices_per_s": o.n / el / 1e6, "s_per_linearization": el, "cores": 1,
            "sample": f"oracle vertex-centred AD linearization, {n}^3 elements ({o.n} vertices)"}


def cpu_phases_full(case, x, dt=250.0, its=8):
    """The oracle on the bench's own problem and state: one AD linearization with the element loop
    on all host cores (the reference's ThreadsPerProcess tasklets), and natural-order block ILU(0)
    + BiCGStab (sequential, as one reference rank runs dune-istl): a solve capped at 1 iteration
    and one capped at 1 + its iterations give the factorization time and the time per iteration."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ewg
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    o = oracle.Oracle(case, nthreads=cores)
    o.set_solution(1, x)
    o.set_solution(0, x)
    o.linearize(dt, 0)  # first iteration of the step: the storage cache of solution(1)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.linearize(dt, 1)
    t_lin = time.perf_counter() - t0
    capped = dict(linear_solver_tolerance=1e-30, linear_solver_abs_tolerance=0.0, restart_on_breakdown=1,
                  verify_true_residual=0)
    t0 = time.perf_counter()
    o.solve(ewg.default_solve_opts(linear_solver_max_iterations=1, **capped))
    t_1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    rc, _, it, _ = o.solve(ewg.default_solve_opts(linear_solver_max_iterations=1 + its, **capped))
    t_k = time.perf_counter() - t0
    o.close()
    t_it = (t_k - t_1) / its
    return {"cores": cores, "threads_linearization": cores, "threads_solve": 1,
            "s_per_linearization": t_lin, "s_per_bicgstab_iteration": t_it,
            "s_ilu_factorization": max(t_1 - t_it, 0.0), "s_context_setup": t_setup,
            "iterations_timed": it}


def cpu_baseline_block(case, x, gpu, steps_its):
    """cpu_baseline on the bench workload itself (same grid, permeability and state): per-phase CPU
    times, the GPU/CPU ratio of each phase, and a time step composed from them with the Newton and
    BiCGStab iteration counts of the timed GPU steps."""
    N = case.n_cells
    ph = cpu_phases_full(case, x)
    n_newton = float(np.mean([a for a, _ in steps_its]))
    # the timed steps ran the box-8-colour ILU(0); the reference's natural order needs fewer
    n_bicg = float(np.mean([b for _, b in steps_its])) * NATURAL_OVER_BOX8
    # a step: one linearization and one ILU(0) factorization per Newton iteration, one BiCGStab
    # iteration per counted iteration (the last linearization of a step is not solved)
    s_step = n_newton * ph["s_per_linearization"] + (n_newton - 1) * ph["s_ilu_factorization"] + \
        n_bicg * ph["s_per_bicgstab_iteration"]
    value = N / s_step / 1e6
    phases = {
        "linearization": {"cpu_mcells_per_s": N / ph["s_per_linearization"] / 1e6,
                          "gpu_mcells_per_s": gpu.get("lin_mcells_per_s"),
                          "gpu_over_cpu": (gpu["lin_mcells_per_s"] / (N / ph["s_per_linearization"] / 1e6))
                          if gpu.get("lin_mcells_per_s") else None},
        "bicgstab_iteration": {"cpu_iterations_per_s": 1.0 / ph["s_per_bicgstab_iteration"],
                               "cpu_cell_iterations_per_s": N / ph["s_per_bicgstab_iteration"],
                               "gpu_iterations_per_s": gpu.get("bicg_iterations_per_s"),
                               "gpu_over_cpu": (gpu["bicg_iterations_per_s"] * ph["s_per_bicgstab_iteration"])
                               if gpu.get("bicg_iterations_per_s") else None},
    }
    return {"value": value, "unit": "Mcells/s", "cores": ph["cores"], "kind": "port",
            "sample": (f"oracle (CPU restatement of the reference path) on the same {case.grid.nx}x{case.grid.ny}x"
                       f"{case.grid.nz} problem and state as the timed GPU steps: one AD linearization "
                       f"(element loop on {ph['cores']} threads) and {ph['iterations_timed'] - 1} + 1 "
                       f"natural-order block-ILU(0) BiCGStab iterations (sequential, as one reference rank); "
                       f"value = cells / composed step time, the step composed of {n_newton:.1f} "
                       f"linearizations, {n_newton - 1:.1f} ILU(0) factorizations and {n_bicg:.0f} BiCGStab "
                       f"iterations (the means of the timed GPU steps; their box-8-colour BiCGStab count times "
                       f"{NATURAL_OVER_BOX8:.3f}, the natural order's share measured by the oracle at 128x128x64)"),
            "s_per_step_composed": s_step, "phases": ph, "gpu_over_cpu": phases,
            "vcfv_linearization": cpu_vcfv_linearization()}


# ---------------------------------------------------------------------------------------------


def run_reference(args, rank, world, pg):
    """The reference's CPU path on the bench's own workload (the 256x256x128 lens, seed 0): the
    oracle restatement on the host cores (the reference itself needs DUNE / ewoms-material, absent
    here). A timed step is a bounded sample of an implicit step: one AD linearization with the element
    loop on all cores (the reference's ThreadsPerProcess tasklets) and one natural-order block-ILU(0)
    factorization + BiCGStab iteration (sequential, as one reference rank runs dune-istl); the step
    time is composed from the sampled phase times with REF_NEWTON_PER_STEP linearizations and
    factorizations and REF_BICGSTAB_PER_STEP iterations, the per-iteration time measured once
    before the timed steps on a solve capped at 1 + 8 iterations."""
    if rank != 0:
        return
    import ewg
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    case = ewg.lens3d_case(args.nx, args.ny, args.nz, seed=0)
    cores = os.cpu_count() or 1
    dt = 250.0
    o = oracle.Oracle(case, nthreads=cores)
    o.apply_initial_solution()
    o.linearize(dt, 0)  # the first iteration of a step fills the storage cache of solution(1)
    capped = dict(linear_solver_tolerance=1e-30, linear_solver_abs_tolerance=0.0, restart_on_breakdown=1,
                  verify_true_residual=0)
    its = 8
    t0 = time.perf_counter()
    o.solve(ewg.default_solve_opts(linear_solver_max_iterations=1, **capped))
    t_1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.solve(ewg.default_solve_opts(linear_solver_max_iterations=1 + its, **capped))
    t_it = (time.perf_counter() - t0 - t_1) / its
    for _ in range(args.warmup):
        o.linearize(dt, 1)
    samples = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.linearize(dt, 1)
        t_lin = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.solve(ewg.default_solve_opts(linear_solver_max_iterations=1, **capped))
        t_fact = max(time.perf_counter() - t0 - t_it, 0.0)
        samples.append(REF_NEWTON_PER_STEP * t_lin + (REF_NEWTON_PER_STEP - 1) * t_fact + REF_BICGSTAB_PER_STEP * t_it)
    o.close()
    s_step = float(np.mean(samples))
    value = case.n_cells / s_step / 1e6
    sample = (f"oracle (CPU restatement of the reference path) on the {args.nx}x{args.ny}x{args.nz} lens, hydrostatic "
              f"initial state: per timed step one AD linearization (element loop on {cores} threads) and one "
              f"natural-order block-ILU(0) factorization + BiCGStab iteration (sequential, as one reference rank); "
              f"step = {REF_NEWTON_PER_STEP:.2f} x (linearization + factorization) - 1 factorization + "
              f"{REF_BICGSTAB_PER_STEP:.0f} x {t_it:.3f} s per BiCGStab iteration")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mcells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": s_step * 1e3, "s_per_step": s_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded log-normal permeability, hydrostatic initial state)",
        "config": {"workload": f"lens3d {args.nx}x{args.ny}x{args.nz} ({case.n_cells} cells) plain FP64 path, implicit "
                               f"Euler dt=250 s, Newton tol 1e-8, BiCGStab+ILU0 rel 1e-10",
                   "cells": case.n_cells, "precision": "fp64", "ilu_ordering": "natural (the reference's)"},
        "phases": {"s_per_bicgstab_iteration": t_it, "s_per_step_samples": samples,
                   "newton_per_step": REF_NEWTON_PER_STEP, "bicgstab_per_step": REF_BICGSTAB_PER_STEP},
        "cpu_baseline": {"value": value, "unit": "Mcells/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ensemble_cases(ewg, members, seed=3, sizes=(32, 48, 64, 96, 128)):
    """Batched-ensemble workload: seeded lens realizations with cube grids drawn from
    {32, 48, 64, 96, 128}^3, sigma in [0.5, 1.5], correlation length in [4, 12] cells and
    dt in {100, 250, 500} s."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(list(sizes), size=members)
    cases, dts = [], []
    for m in range(members):
        n = int(sizes[m])
        cases.append(ewg.lens3d_case(n, n, n, seed=seed * 1000 + m, sigma=float(rng.uniform(0.5, 1.5)),
                                     corr_cells=float(rng.uniform(4.0, 12.0))))
        dts.append(float(rng.choice([100.0, 250.0, 500.0])))
    return cases, dts


def vcfv_lin_bytes(nv, dim=3):
    """Algorithmic bytes of one vertex-centred linearization: per vertex x (16), old storage (16),
    K (8), lens flag (1), residual (16) and the 27 (9) Jacobian blocks of its row (32 each)."""
    return nv * (16 + 16 + 8 + 1 + 16 + (27 if dim == 3 else 9) * 32)


def run_vcfv(args, rank, pg, torch, ewg):
    """The vertex-centred discretization: linearization of the bench grid (the same 3D lens with
    the permeability field drawn on the vertex grid) at a state with a partly drained top fifth,
    and one implicit step of a 64^3-element member (BiCGStab + block ILU(0) in the parity-colour
    order at the reference's linear tolerance 1e-3)."""
    case = ewg.vcfv_case(ewg.lens3d_case(args.nx, args.ny, args.nz, seed=rank), seed=rank)
    g = ewg.VcfvContext(case)
    g.apply_initial_solution()
    x = g.get_solution(0)
    rng = np.random.default_rng(rank)
    y = ewg.vertex_positions(case.grid)[1]
    top = y > 0.8 * case.grid.ly
    xp = x.copy()
    xp[top, 1] = 1.0 - rng.uniform(0.0, 0.4, int(top.sum()))
    g.set_solution(1, x)
    g.set_solution(0, xp)
    for _ in range(3):
        g.linearize(250.0)
    torch.cuda.synchronize()
    barrier(pg)
    reps = 10
    l0 = g.launches
    t0 = time.perf_counter()
    for _ in range(reps):
        g.linearize(250.0)
    t1 = time.perf_counter()
    launches = g.launches - l0
    ms = max_over_ranks(pg, (t1 - t0) / reps * 1e3)
    nv = g.n
    peak, _ = measured_peak()
    lb = vcfv_lin_bytes(nv)
    # the finite-difference local linearizer (lens_immiscible_vcfv_fd) on the same state
    g.set_local_linearizer(ewg.LOCAL_LINEARIZER_FD, 1)
    g.linearize(250.0)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    for _ in range(3):
        g.linearize(250.0)
    fd_ms = max_over_ranks(pg, (time.perf_counter() - t2) / 3 * 1e3)
    g.set_local_linearizer(ewg.LOCAL_LINEARIZER_AD, 1)
    out = {"grid": f"{args.nx}x{args.ny}x{args.nz} elements, {nv} vertices",
           "fd_forward_ms_per_linearization": fd_ms,
           "ms_per_linearization": ms, "mvertices_per_s": nv / (ms * 1e-3) / 1e6,
           "algorithmic_bytes": lb, "achieved_gbs": lb / (ms * 1e-3) / 1e9, "frac": lb / (ms * 1e-3) / 1e9 / peak,
           "launches_per_linearization": launches / reps,
           "timing": "host clock around synchronous ewg_vcfv_linearize calls (two kernels and a 12-byte read-back each)"}
    g.close()
    small = ewg.vcfv_case(ewg.lens3d_case(64, 64, 64, seed=rank), seed=rank)
    g = ewg.VcfvContext(small)
    g.apply_initial_solution()
    so = ewg.default_solve_opts(precond=ewg.PRECOND_ILU0, linear_solver_tolerance=1e-3,
                                linear_solver_max_iterations=2000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st, its, lin, err = g.newton_apply(250.0, None, so)
    t1 = time.perf_counter()
    out["step_64cubed"] = {"status": int(st), "newton_its": its, "linear_its": lin, "s_per_step": t1 - t0,
                           "vertices": g.n}
    g.close()
    return out


def run_ensemble(args, rank, pg, torch, ewg):
    """The batched ensemble form: every member advances one implicit step per timed step (its own
    dt, FP64 residual / update / Newton test, FP32 Jacobian, ILU(0) and BiCGStab), all members in
    the same launches with the BiCGStab iteration replayed from a CUDA graph. Under torchrun the
    one ensemble is sharded: every rank draws the same member list and advances the members the
    greedy cost balance assigns to it (shard.py); only the timing and the counts are reduced."""
    import shard
    world = pg.get_world_size() if pg is not None else 1
    all_cases, all_dts = ensemble_cases(ewg, args.ensemble_members, seed=3)
    costs = [shard.member_cost(c.n_cells, dt) for c, dt in zip(all_cases, all_dts)]
    assignment = shard.assign_members(costs, world)
    mine = assignment[rank]
    cases, dts = [all_cases[m] for m in mine], [all_dts[m] for m in mine]
    so = ewg.default_solve_opts(precision=ewg.PRECISION_MIXED, linear_solver_tolerance=1e-3,
                                verify_true_residual=0)
    ens = ewg.Ensemble(cases, precision=ewg.PRECISION_MIXED)
    ens.apply_initial_solution()
    t0 = time.perf_counter()
    shapes = ens.autotune(dts, so)
    tune_s = time.perf_counter() - t0
    ens.apply_initial_solution()
    dev = args.ensemble_scheduler == "device"
    ens.advance(1, dts, sopts=so, device=dev)  # warm-up step
    stream = torch.cuda.ExternalStream(ens.stream)
    torch.cuda.synchronize()
    barrier(pg)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # every member advances ensemble_steps steps at its own pace
    st, reps, sts = ens.advance(args.ensemble_steps, dts, sopts=so, device=dev)
    e1.record(stream)
    torch.cuda.synchronize()
    stats = [(reps, sts)]
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    cells = ens.total_cells
    total = sum_over_ranks(pg, float(cells))
    all_cells = sum(c.n_cells for c in all_cases)
    newton = [r.newton_iterations / args.ensemble_steps for reps, _ in stats for r in reps]
    out = {
        "workload": f"{len(all_cases)} lens realizations, cube grids from {{32,48,64,96,128}}^3, {all_cells} cells, "
                    f"dt from {{100,250,500}} s, mixed precision (FP32 inner BiCGStab to rel 1e-3, Newton tol 1e-8)",
        "members": len(all_cases), "cells": all_cells, "steps": args.ensemble_steps,
        "sharding": {"ranks": world, "members_per_rank": [len(a) for a in assignment],
                     "cost_imbalance": shard.imbalance(costs, assignment),
                     "scaling": "strong (one ensemble split across the ranks by cost)"},
        "s_per_step": ms / args.ensemble_steps / 1e3,
        "mcells_steps_per_s": total * args.ensemble_steps / (ms * 1e-3) / 1e6,
        "newton_iterations_per_step_mean": float(np.mean(newton)),
        "newton_iterations_per_step_max": float(np.max(newton)),
        "halvings": int(sum(r.halvings for reps, _ in stats for r in reps)),
        "scheduler": ("device: every decision on the device, supersteps inside a CUDA graph WHILE node"
                      if dev else "host: decisions on the host between supersteps"),
        "rounds": [s.rounds for _, s in stats], "linear_iterations": [s.linear_iterations for _, s in stats],
        "supersteps": [s.supersteps for _, s in stats],
        # BiCGStab work actually done: cells x iterations summed over members, per second of BiCGStab
        # time (host scheduler) or of the whole advance (device scheduler: phases not timed apart)
        "bicgstab_cell_iterations_per_s": sum(s.cell_iterations for _, s in stats) / sum(s.t_solve for _, s in stats),
        "phase_s": ({"advance": sum(s.t_solve for _, s in stats) / len(stats)} if dev else
                    {"linearize": sum(s.t_linearize for _, s in stats) / len(stats),
                     "solve": sum(s.t_solve for _, s in stats) / len(stats),
                     "update": sum(s.t_update for _, s in stats) / len(stats)}),
        "launch_shapes": shapes, "autotune_s": tune_s,
    }
    ens.close()
    return out


def run_conv(torch, ewg, shape=(1, 128, 256, 256), reps=10):
    """The guess network's tensor-core convolution (ewg_net_conv3d, tcgen05.mma + TMA) on a volume
    of the bench grid's size: both layer widths (16 -> 32 and 32 -> 32 channels, bias + ReLU), CUDA
    events around reps calls after 3 warm-up calls; FLOPs = 2 x 27 x Cin x 32 per voxel."""
    import ctypes as C
    lib = ewg.load()
    fn = lib.ewg_net_conv3d
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32] * 6 + [C.c_void_p] * 6
    B, D, H, W = shape
    V = B * D * H * W
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        pass
    out = {"volume": list(shape), "voxels": V, "peak_bf16_tflops": peak,
           "peak_kind": "measured burst (MEASURED_PEAKS.json bf16_tflops)" if peak else None}
    g = torch.Generator(device="cuda").manual_seed(0)
    for cin in (16, 32):
        x = torch.randn(V * cin, device="cuda", generator=g).to(torch.bfloat16)
        w = (torch.randn(27 * 32 * cin, device="cuda", generator=g) * 0.05).to(torch.bfloat16)
        b = torch.zeros(32, device="cuda")
        y = torch.empty(V * 32, dtype=torch.bfloat16, device="cuda")
        s = torch.cuda.current_stream()
        args = (cin, 0, B, D, H, W, C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()), C.c_void_p(b.data_ptr()),
                None, C.c_void_p(y.data_ptr()), C.c_void_p(s.cuda_stream))
        for _ in range(3):
            if fn(*args) != 0:
                raise RuntimeError("ewg_net_conv3d failed")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            if fn(*args) != 0:
                raise RuntimeError("ewg_net_conv3d failed")
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = 2.0 * 27 * cin * 32 * V / (ms * 1e-3) / 1e12
        out[f"cin{cin}"] = {"ms": ms, "tflops": tf, "frac": tf / peak if peak else None}
        del x, w, y
    return out


def run_ours(args, rank, world, local, pg):
    import torch

    import ewg
    dev = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(dev)
    nx, ny, nz = args.nx, args.ny, args.nz
    case = ewg.lens3d_case(nx, ny, nz, seed=rank)
    N, F = geometry((nx, ny, nz))
    mixed = args.precision == "mixed"
    # the graded linear tolerance (rel. 1e-10) needs more than the reference's default 1000
    # BiCGStab iterations on this grid in some Newton iterations; a linear-solver failure would
    # halve the time step and change the workload, so the limit is raised for every form
    max_its = 5000
    sopts = ewg.default_solve_opts(precision=ewg.PRECISION_MIXED if mixed else ewg.PRECISION_FP64,
                                   linear_solver_max_iterations=max_its)
    nopts = ewg.default_newton_opts()
    ctx = ewg.Context(case)
    ctx.apply_initial_solution()

    guess_log = []

    halvings = []

    def one_step(dt=250.0, sopts=sopts, net=None):
        h = dt
        for attempt in range(10):
            if attempt:
                halvings.append(h)
            if net is not None:
                # the learned initial guess replaces solution(0) only if its residual is smaller
                used, rg, rp = net.predict_guess(ctx, h)
                guess_log.append((used, rg, rp))
            st, rep = ctx.newton_apply(h, nopts, sopts)
            if st == ewg.EWG_OK:
                ctx.advance_time_level()
                return rep
            ctx.restore_time_level()
            h /= 2
        raise RuntimeError("time step failed after 10 halvings")

    for _ in range(args.warmup):
        one_step()
    # the end-to-end pass below replays the same K steps from this state
    snap0, snap1 = ctx.get_solution(0), ctx.get_solution(1)
    stream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    ctx.profile_reset()
    # every 31st launch of each kernel class is bracketed by CUDA events (all launches counted): 31
    # is prime to the 8 colour launches of a box-8 sweep, so every colour is sampled alike, and an
    # event pair (which also ends the programmatic launch overlap of its kernel) lands on one in
    # 31 launches, so the sampling costs the timed steps little
    ctx.profile_enable(True, period=31)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps = []
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            reps.append(one_step())
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    ms_local = ev0.elapsed_time(ev1)
    prof = ctx.profile()
    ctx.profile_enable(False)
    x_plain = ctx.get_solution(0)
    ms = max_over_ranks(pg, ms_local)
    total_cells = sum_over_ranks(pg, float(N))
    value = total_cells * args.steps / (ms * 1e-3) / 1e6

    # ---- the other forms on the same K steps (replayed from the snapshot) ----
    forms = {}
    if not args.no_forms:
        net = ewg.GuessNet(seed=0)
        net.load_file(os.path.join(ROOT, "ewoms-numerics_b200", "data", "guess_net_lens3d.npz"))
        variants = {
            # the reference's own default linear tolerance (LinearSolverTolerance 1e-3,
            # fvbasediscretization.hh:249) with the FP64 solver
            "fp64_reference_linear_tol": (ewg.default_solve_opts(linear_solver_tolerance=1e-3,
                                                                 linear_solver_max_iterations=max_its), None),
            # FP32 Jacobian / ILU / BiCGStab, FP64 residual, update and Newton test
            "mixed": (mixed_opts(ewg), None),
            # the same with the learned Newton initial guess (kept only where it lowers the residual)
            "learned_mixed": (mixed_opts(ewg), net),
        }
        for fname, (fo, fnet) in variants.items():
            ctx.set_solution(1, snap1)
            ctx.set_solution(0, snap0)
            guess_log.clear()
            torch.cuda.synchronize()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            freps = [one_step(sopts=fo, net=fnet) for _ in range(args.steps)]
            f1.record(stream)
            torch.cuda.synchronize()
            f_ms = max_over_ranks(pg, f0.elapsed_time(f1))
            xf = ctx.get_solution(0)
            forms[fname] = {"s_per_step": f_ms / args.steps / 1e3,
                            "mcells_per_s": total_cells * args.steps / (f_ms * 1e-3) / 1e6,
                            "newton_its": [r.iterations for r in freps],
                            "linear_its": [r.linear_iterations for r in freps],
                            "max_rel_dpw_vs_plain": float(np.max(np.abs(xf[:, 0] - x_plain[:, 0])) / np.max(np.abs(x_plain[:, 0]))),
                            "max_abs_dSn_vs_plain": float(np.max(np.abs(xf[:, 1] - x_plain[:, 1]))),
                            "speedup_vs_plain": ms / f_ms}
            if fnet is not None:
                forms[fname]["guess_used"] = [bool(u) for u, _, _ in guess_log]
                forms[fname]["guess_residual_ratio"] = [rg / rp if rp > 0 else None for _, rg, rp in guess_log]
        net.close()
        ctx.set_solution(1, x_plain)
        ctx.set_solution(0, x_plain)

    # ---- the local linearizers on the final state: AD (the timed path) and finite differences ----
    linearizers = {}
    if not args.no_forms:
        peak_l, _ = measured_peak()
        lb_l = lin_bytes(N, F, 8)
        # one short FP64 Newton pass selects the FP64 Jacobian (the forms above end in FP32)
        ctx.newton_apply(250.0, ewg.default_newton_opts(newton_max_iterations=1),
                         ewg.default_solve_opts(linear_solver_tolerance=1e-3))
        ctx.restore_time_level()
        ctx.set_solution(1, x_plain)
        ctx.set_solution(0, x_plain)
        for lname, kind, method in (("ad", ewg.LOCAL_LINEARIZER_AD, 1), ("fd_forward", ewg.LOCAL_LINEARIZER_FD, 1),
                                    ("fd_central", ewg.LOCAL_LINEARIZER_FD, 0)):
            ctx.set_local_linearizer(kind, method)
            ctx.linearize(250.0)
            torch.cuda.synchronize()
            l0 = torch.cuda.Event(enable_timing=True)
            l1 = torch.cuda.Event(enable_timing=True)
            l0.record(stream)
            for _ in range(10):
                ctx.linearize(250.0)
            l1.record(stream)
            torch.cuda.synchronize()
            l_ms = max_over_ranks(pg, l0.elapsed_time(l1)) / 10
            linearizers[lname] = {"ms_per_linearization": l_ms, "mcells_per_s": N / (l_ms * 1e-3) / 1e6,
                                  "frac_of_lin_bytes": lb_l / (l_ms * 1e-3) / 1e9 / peak_l}
        ctx.set_local_linearizer(ewg.LOCAL_LINEARIZER_AD, 1)

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        xh = torch.empty((N, 2), dtype=torch.float64, pin_memory=True)
        xn = xh.numpy()
        xn[:] = snap0
        assert np.array_equal(snap0, snap1)
        barrier(pg)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.set_solution(1, xn)
            ctx.set_solution(0, xn)
            h = 250.0
            for _ in range(10):
                st, _rep = ctx.newton_apply(h, nopts, sopts)
                if st == ewg.EWG_OK:
                    break
                ctx.restore_time_level()
                h /= 2
            ctx.get_solution(0, out=xn)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(pg)
        e_ms = max_over_ranks(pg, e0.elapsed_time(e1))
        e2e = {"value": total_cells * args.steps / (e_ms * 1e-3) / 1e6, "unit": "Mcells/s",
               "h2d_bytes_per_step": 2 * N * 16, "d2h_bytes_per_step": N * 16,
               "ms_per_step": e_ms / args.steps}

    ensemble = None
    if not args.no_ensemble:
        ensemble = run_ensemble(args, rank, pg, torch, ewg)

    vcfv = None
    if not args.no_vcfv:
        vcfv = run_vcfv(args, rank, pg, torch, ewg)

    conv = None
    if not args.no_conv:
        conv = run_conv(torch, ewg, (1, nz, ny, nx))

    if rank != 0:
        ctx.close()
        return
    # ---- roofline of the dominant kernel ----
    peak, peak_kind = measured_peak()
    s = 4 if mixed else 8
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dname, (dms, dn) = dom
    b8 = "b8_forward" in prof
    Fx = cross_box_faces((nx, ny, nz))
    db = kernel_bytes(dname, N, F, s_mat=s, s_vec=s, b8=b8, Fx=Fx)
    avg_ms = dms / dn
    achieved = db / (avg_ms * 1e-3) / 1e9 if db else None
    traffic = (NCU_TRAFFIC_B8 if b8 else NCU_TRAFFIC).get(dname) if not mixed else None
    roofline = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": traffic,
                "algorithmic_bytes_per_launch": db, "avg_launch_ms": avg_ms, "launches": dn,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback"}
    # linearization and BiCGStab-iteration rooflines
    t_lin = sum(prof.get(k, (0, 0))[0] for k in ("intensive", "assemble"))
    n_lin = prof.get("assemble", (0, 0))[1]
    lin = None
    if n_lin:
        lin_avg = t_lin / n_lin
        lb = lin_bytes(N, F, 8)
        lin = {"ms_per_linearization": lin_avg, "mcells_per_s": N / (lin_avg * 1e-3) / 1e6,
               "algorithmic_bytes": lb, "achieved_gbs": lb / (lin_avg * 1e-3) / 1e9,
               "frac": lb / (lin_avg * 1e-3) / 1e9 / peak, "launches": n_lin}
    it_kernels = ("bicg_p", "ilu_black_apply", "ilu_red_apply", "jacobi_apply", "b8_forward", "b8_backward",
                  "bicg_spmv_alpha", "bicg_hs", "bicg_spmv_omega", "bicg_xr")
    n_it = prof.get("bicg_xr", (0, 0))[1]
    bicg = None
    if n_it:
        t_it = sum(prof.get(k, (0, 0))[0] for k in it_kernels) / n_it
        b_it = sum((kernel_bytes(k, N, F, s, s, b8=b8, Fx=Fx) or 0) * prof.get(k, (0, 0))[1]
                   for k in it_kernels) / n_it
        bicg = {"ms_per_iteration": t_it, "iterations_per_s": 1e3 / t_it, "algorithmic_bytes": b_it,
                "achieved_gbs": b_it / (t_it * 1e-3) / 1e9, "frac": b_it / (t_it * 1e-3) / 1e9 / peak,
                "iterations": n_it}
    launches = int(sum(v[1] for v in prof.values()))
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        gpu_phase = {"lin_mcells_per_s": lin["mcells_per_s"] if lin else None,
                     "bicg_iterations_per_s": bicg["iterations_per_s"] if bicg else None}
        cpu = cpu_baseline_block(case, x_plain, gpu_phase, [(r.iterations, r.linear_iterations) for r in reps])
    line = {
        "metric": METRIC, "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "s_per_step": ms / args.steps / 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if not mixed else "f64/f32",
        "data": "synthetic (seeded log-normal permeability per rank, hydrostatic initial state)",
        "config": {"workload": f"lens3d {nx}x{ny}x{nz} ({N} cells) plain {'FP64' if not mixed else 'mixed'} path, "
                               f"implicit Euler dt=250 s, Newton tol 1e-8, BiCGStab+ILU0 rel 1e-10",
                   "cells": N, "interior_faces": F, "precision": args.precision,
                   "ilu_ordering": "box-8-colour (2x2x2 boxes in 8 colours)" if b8 else "red-black",
                   "l2": "working set (> 4 GB) larger than L2 (126 MB); no flush needed"},
        "newton_its": [r.iterations for r in reps], "linear_its": [r.linear_iterations for r in reps],
        "time_step_halvings": len(halvings),
        "phase_s": {"linearize": sum(r.t_linearize for r in reps) / len(reps),
                    "solve": sum(r.t_solve for r in reps) / len(reps),
                    "update": sum(r.t_update for r in reps) / len(reps)},
        "roofline": roofline, "linearization": lin, "linearizers": linearizers, "bicgstab": bicg,
        "kernels": {k: {"ms": v[0], "launches": v[1]} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "gpu_launches": launches, "e2e": e2e, "forms": forms, "ensemble": ensemble, "vcfv": vcfv,
        "guess_conv": conv, "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.impl == "reference":
        # the host-core reference arm: rank 0 alone runs it, other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, int(os.environ.get("WORLD_SIZE", "1")), None)
        return
    if args.conv:
        import torch
        import ewg
        print(json.dumps({"guess_conv": run_conv(torch, ewg, (1, args.nz, args.ny, args.nx))}), flush=True)
        return
    rank, world, local, pg = dist_init(args)
    try:
        run_ours(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
