#!/usr/bin/env python
"""Benchmark: plain FP64 F-cycle throughput of the multigrid engine on one B200 per rank.

Workload (the reference's 513x257x129 case): u = x^3 y^2 z on [0,1]x[0,0.5]x[0,0.25],
h = 1/512, 6 levels, BoundaryCondition {N,N,N,N,D,D} (resolved by the reference to Neumann
on x, Dirichlet on y and z), FullWeighting + TrilinearInterpolation + weighted Jacobi
(omega = 6/7), nsmooth = 2, F-cycles.  One step = one iteration of PoissonSolver::solve:
one F-cycle, the fine residual with its max-norm, the norm read-back and the stopping rule.
The metric is fine-grid DOF x F-cycles per second.

  value  -- device-resident: K iterations of one solve() call, CUDA events on the engine's
            stream, max over ranks; the 4 fine arrays (4 x 143 MB) are far larger than L2.
  e2e    -- through the reference-facing API (mgp.PoissonSolver): per request
            to_device (u, u_prev, f, r + faces from pinned host memory), a 4-cycle solve and
            to_host (r, u, u_prev), timed on the same stream.
  roofline -- the dominant kernel (the level-0 Jacobi sweep) timed alone with CUDA events,
            against its algorithmic 24 B/point.
  cpu_baseline -- the reference's own OpenMP build (oracle/_ref/ref_oracle) on this host.

--impl reference runs the reference's CPU code instead (rank 0 only) with the same metric.
Multi-GPU (torchrun): each rank solves its own independent replica (no collective on the
data path): weak scaling, value = all ranks' DOF-cycles / max-over-ranks time.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "multigrid-poisson_b200"))
sys.path.insert(0, str(ROOT))

DIMS = (513, 257, 129)
LEVELS = 6
H = 1.0 / 512
BC = (1, 1, 1, 1, 0, 0)  # N S E W T B requested
NSMOOTH = 2
E2E_CYCLES = 4
REF_ARM_CYCLES = 30   # timed cycles of the reference arm (a bounded sample)
# DRAM bytes (read + write) of one level-0 Jacobi sweep launch at this size, from an ncu capture
# of the timed launch: ncu --set full --clock-control none --kernel-name-base demangled
#   -k "regex:k_stencil<double, \(int\)0, \(bool\)0, \(bool\)0>" -s 3 -c 1 python bench.py --kernels --steps 1
# (289.6 MB read + 109.7 MB written; algorithmic 408.2 MB: some of u is still in L2 from the
# launch before).
JACOBI_SWEEP_DRAM_BYTES = 399.3e6
CPU_BASELINE_CYCLES = 8
NDOF = DIMS[0] * DIMS[1] * DIMS[2]
METRIC = "F-cycle fine-grid DOF/s (FP64, 513x257x129)"
UNIT = "DOF*cycles/s"
WORKLOAD = ("fp64 F-cycle, 513x257x129 (6 levels), u=x^3 y^2 z on [0,1]x[0,.5]x[0,.25], BC {N,N,N,N,D,D}, "
            "FullWeighting + Trilinear + Jacobi(6/7), nsmooth=2; step = one solve() iteration")


def problem2(x, y, z):
    return x * x * x * y * y * z


def rhs2(x, y, z):
    return 2.0 * x * x * x * z + 6.0 * x * y * y * z


def dudx2(x, y, z):
    return 3.0 * x * x * y * y * z


def dudy2(x, y, z):
    return 2.0 * x * x * x * y * z


def dudz2(x, y, z):
    return x * x * x * y * y


# ---------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.tmp,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.tmp is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.tmp.flush()
        rows = []
        for line in Path(self.tmp.name).read_text().splitlines():
            t = [c.strip() for c in line.split(",")]
            if len(t) >= 9:
                rows.append(t)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


# ---------------------------------------------------------------------------------------
def dist_setup(n_gpus: int, backend: str | None = None):
    """One process per GPU under torchrun: (world, rank, local_rank, process group or None).
    NCCL on GPU boxes; gloo where no GPU is visible (the host-side tests of the N>1 path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if not dist.is_initialized():
            if backend == "nccl":
                torch.cuda.set_device(local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float, local: int) -> float:
    """The largest x over all ranks (times are taken as the slowest rank's)."""
    if pg is None:
        return x
    import torch

    dev = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank; the job took the slowest
    rank's time (weak scaling: replicas of the same workload)."""
    return units_per_rank * world / seconds_max


def build_solver(mgp, device: int, maxiter: int, pinned: bool, flags: int = 0):
    st = mgp.Settings(levels=LEVELS, dims=list(DIMS), maxiter=maxiter, miniter=maxiter, tolerance=0.0,
                      h=H, origin=[0.0, 0.0, 0.0], dev=device)
    bc = mgp.BoundaryCondition(*BC)
    ps = mgp.PoissonSolver(st, bc, restriction="FullWeighting", relaxation="Jacobi", dtype=mgp.F64,
                           pinned=pinned, flags=flags)
    ps.init(problem2, rhs2, dudx2, dudy2, dudz2)
    return ps


def kernel_roofline(mgp, ps, torch, stream, reps: int = 20):
    """Average duration of the dominant kernel (level-0 Jacobi sweep), CUDA events on the
    engine's stream; algorithmic bytes = 3 arrays x 8 B per shape point (read u_prev, read f,
    write u)."""
    eng = ps.engine
    for _ in range(3):
        eng.relax(0, -1.0, 1)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        eng.relax(0, -1.0, 1)
    b.record(stream)
    b.synchronize()
    sec = a.elapsed_time(b) / 1e3 / reps
    alg = 24.0 * NDOF
    return sec, alg


def run_kernels(args):
    """Each level-0 operator of the workload timed alone (CUDA events on the engine's
    stream, `args.steps` launches after 3 warm-up launches).  Also the small case for
    profiler captures: the process holds one 513x257x129 hierarchy (~0.7 GB)."""
    import torch

    import mgp

    ps = build_solver(mgp, 0, maxiter=1, pinned=False, flags=args.engine_flags)
    ps.to_device()
    eng = ps.engine
    stream = torch.cuda.ExternalStream(eng.stream_handle, device="cuda:0")
    n = NDOF
    nc = ((DIMS[0] >> 1) + 1) * ((DIMS[1] >> 1) + 1) * ((DIMS[2] >> 1) + 1)
    ops = {  # name: (callable, algorithmic bytes per launch)
        "jacobi_sweep": (lambda: eng.relax(0, -1.0, 1), 24.0 * n),
        # two sweeps in one pass: read u, f; write u2 and u1
        "jacobi_pair": (lambda: eng.relax(0, -1.0, 2), 32.0 * n),
        # two sweeps and the residual with its max-norm in one pass: read u, f; write u2, u1, r
        "pair_residual_norm": (lambda: eng.relax_residual(0, -1.0, 2, norm=True), 40.0 * n),
        "residual": (lambda: eng.residual(0), 24.0 * n),
        # the solve loop's residual with its max-norm (and the norm's read-back): read u, f; write r
        "residual_norm": (lambda: eng.relax_residual(0, -1.0, 0, norm=True), 24.0 * n),
        "restrict_fw": (lambda: eng.restrict(0), 8.0 * (n + nc)),
        "prolong_add": (lambda: eng.prolong_add(0), 8.0 * (2 * n + nc)),
        # last (the level-0 legs above come first, for profiler captures by launch order): the
        # coarse sub-cycles inside one F-cycle iteration (F(1) once, V(1) twice), launched
        # directly, not from a graph
        "fcycle_level1": (lambda: eng.fcycle(1, -1.0, NSMOOTH), 0.0),
        "vcycle_level1": (lambda: eng.vcycle(1, -1.0, NSMOOTH), 0.0),
    }
    peak, kind = measured_peaks()
    out = {}
    for name, (fn, nbytes) in ops.items():
        for _ in range(3):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        b.synchronize()
        us = a.elapsed_time(b) * 1e3 / args.steps
        gbs = nbytes / (us * 1e-6) / 1e9
        out[name] = {"us": us, "algorithmic_bytes": nbytes, "GB/s": gbs, "frac": gbs / peak} if nbytes else {"us": us}
    print(json.dumps({"kernels": out, "peak_gbs": peak, "peak_kind": kind, "workload": WORKLOAD}))
    return 0


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


def timed(torch, stream, fn):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    out = fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / 1e3, out


def _sin2pi(x, y, z):
    return np.sin(2.0 * np.pi * x) * np.sin(2.0 * np.pi * y) * np.sin(2.0 * np.pi * z)


def _sin2pi_rhs(x, y, z):
    return -12.0 * np.pi * np.pi * _sin2pi(x, y, z)


def _zero(x, y, z):
    return 0.0 * x


def _cycle_leg(mgp, torch, device, dims, levels, h, bc, restriction, relaxation, cycle, cycles, funcs, flags=0,
               tune=True):
    """`cycles` iterations of solve(cycle) through the reference-facing API after a warm-up solve
    (graphs captured): ms per cycle of the solve loop (norm read-back and stop rule included)
    and of the captured iteration alone (graph replays), kernel launches per cycle, the final
    relative residual; then the same after mgp_autotune."""
    st = mgp.Settings(levels=levels, dims=list(dims), maxiter=cycles, miniter=cycles, tolerance=0.0, h=h,
                      origin=[0.0, 0.0, 0.0], dev=device)
    ps = mgp.PoissonSolver(st, mgp.BoundaryCondition(*bc), restriction=restriction, relaxation=relaxation,
                           dtype=mgp.F64, flags=flags)
    ps.init(*funcs)
    eng = ps.engine
    stream = torch.cuda.ExternalStream(eng.stream_handle, device=f"cuda:{device}")
    out = {}

    def run(tag):
        ps.to_device()
        eng.solve(cycle, NSMOOTH)  # warm-up: captures the iteration graphs
        ps.to_device()
        sec, stt = timed(torch, stream, lambda: eng.solve(cycle, NSMOOTH))
        out[tag] = {"ms_per_cycle": 1e3 * sec / stt.cycles_run, "cycles": int(stt.cycles_run),
                    "launches_per_cycle": stt.kernel_launches / stt.cycles_run, "rel_res": stt.rel_res,
                    "dof_cycles_per_s": dims[0] * dims[1] * dims[2] * stt.cycles_run / sec}

    run("built_in")
    if tune:
        t = eng.autotune(cycle, NSMOOTH, force=True)
        run("tuned")
        out["iteration_ms_graph_replay"] = {"built_in": t["untuned_ms"], "tuned": t["tuned_ms"]}
        out["tuned_params_per_level"] = t["params"]
    eng.close()
    return out


def bench_c1(mgp, torch, device=0):
    """65^3 all-Dirichlet F-cycle, Injection + red-black SOR nu=2, 5 levels, 10 cycles from a
    zero guess, u = sin(2 pi x) sin(2 pi y) sin(2 pi z): a launch-latency-bound workload (a
    65^3 level is 2.2 MB), timed per cycle."""
    out = _cycle_leg(mgp, torch, device, (65, 65, 65), 5, 1.0 / 64, (0,) * 6, "Injection", "GaussSeidel", "Fcycle",
                     10, (_sin2pi, _sin2pi_rhs, _zero, _zero, _zero))
    out["workload"] = "65x65x65, 5 levels, all Dirichlet, Injection + Trilinear + red-black SOR (8/9), F-cycle, 10 cycles"
    out["note"] = ("right-hand side from numpy's sin on the host; the reference's own output for this case (rel_res "
                   "14.1367 after 10 cycles: it diverges) is pinned bit for bit by the golden tests, whose problem data "
                   "come from libm")
    return out


def bench_c2(mgp, torch, device=0, cycles=20, tol=1e-10):
    """513x257x129 FP64 V-cycle, FullWeighting + weighted Jacobi (6/7), 6 levels, the x^3 y^2 z
    Neumann problem: plain V-cycles (per-cycle time; the reference's cycle stalls on this
    Neumann problem, so the residual reached after `cycles` cycles is reported), and the same
    V-cycle as FP64 / FP32-correction iterative refinement to `tol`."""
    funcs = (problem2, rhs2, dudx2, dudy2, dudz2)
    out = _cycle_leg(mgp, torch, device, DIMS, LEVELS, H, BC, "FullWeighting", "Jacobi", "Vcycle", cycles, funcs)
    for name, flag in (("refined_fp64", mgp.FLAG_REFINE_F64), ("refined_mixed", mgp.FLAG_REFINE_F32)):
        e = mgp.Solver(DIMS, LEVELS, H, BC, mgp.FULLWEIGHTING, mgp.JACOBI, mgp.F64, 100, 1, tol, device=device,
                       flags=flag)
        stream = torch.cuda.ExternalStream(e.stream_handle, device=f"cuda:{device}")
        e.fill_problem(2)
        e.solve("Vcycle", NSMOOTH)  # warm-up: instantiates the graphs
        e.fill_problem(2)
        sec, stt = timed(torch, stream, lambda: e.solve("Vcycle", NSMOOTH))
        err_a, rel_a, _ = e.u_error(problem=2)
        out[name] = {"ms_to_tol": 1e3 * sec, "iterations": int(stt.iterations), "rel_res": stt.rel_res,
                     "reached": bool(stt.rel_res < tol), "max_abs_err_vs_analytic": err_a,
                     "rel_l2_err_vs_analytic": rel_a}
        e.close()
    out["workload"] = (f"513x257x129, 6 levels, x^3 y^2 z, BC {{N,N,N,N,D,D}}, FullWeighting + Trilinear + Jacobi "
                       f"(6/7), V-cycle: {cycles} plain cycles; refinement to {tol:g}")
    return out


def bench_mixed(mgp, torch, device=0, tols=(1e-8, 1e-9, 1e-10), maxiter=60):
    """1025x1025x513 (8 levels) u = cos(x z^2) sin(y^3) on [0,1]x[0,1]x[0,0.5], Dirichlet
    data from u, FullWeighting + red-black SOR, F-cycle corrections: iterative refinement with
    an FP32 correction hierarchy against the same with an FP64 one, each driven to every
    tolerance in `tols` from the zero guess.  A tolerance counts as reached when the relative
    residual is below it before `maxiter` iterations; the headline ratio is taken at the
    tightest tolerance both arms reach.  Errors: against the FP64 solution and against the
    analytic solution."""
    dims, levels, h = (1025, 1025, 513), 8, 1.0 / 1024
    out = {"by_tolerance": {}}
    solvers = {}
    for name, flag in (("fp64", mgp.FLAG_REFINE_F64), ("mixed", mgp.FLAG_REFINE_F32)):
        e = mgp.Solver(dims, levels, h, (0,) * 6, mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, mgp.F64, maxiter, 1, tols[0],
                       device=device, flags=flag)
        e.fill_problem(3)
        e.solve("Fcycle", 2)  # warm-up: instantiates the graphs
        solvers[name] = e
    for tol in tols:
        row = {}
        for name, e in solvers.items():
            stream = torch.cuda.ExternalStream(e.stream_handle, device=f"cuda:{device}")
            e.set_iteration_limits(maxiter, 1, tol)
            e.fill_problem(3)
            sec, st = timed(torch, stream, lambda: e.solve("Fcycle", 2))
            err_a, rel_a, _ = e.u_error(problem=3)
            row[name] = {"ms_per_solve": sec * 1e3, "iterations": int(st.iterations), "rel_res": st.rel_res,
                         "reached": bool(st.rel_res < tol and st.iterations < maxiter),
                         "dof_per_s": dims[0] * dims[1] * dims[2] / sec, "solves_per_s": 1.0 / sec,
                         "max_abs_err_vs_analytic": err_a, "rel_l2_err_vs_analytic": rel_a}
        err, rel, _ = solvers["mixed"].u_error(solvers["fp64"])
        row["mixed"]["max_abs_err_vs_fp64"] = err
        row["mixed"]["rel_l2_err_vs_fp64"] = rel
        row["speedup_mixed_over_fp64"] = row["fp64"]["ms_per_solve"] / row["mixed"]["ms_per_solve"]
        out["by_tolerance"][f"{tol:g}"] = row
    both = [t for t, r in out["by_tolerance"].items() if r["fp64"]["reached"] and r["mixed"]["reached"]]
    if both:
        t = min(both, key=float)
        out["headline_tolerance"] = t
        out["fp64"] = out["by_tolerance"][t]["fp64"]
        out["mixed"] = out["by_tolerance"][t]["mixed"]
        out["speedup_mixed_over_fp64"] = out["by_tolerance"][t]["speedup_mixed_over_fp64"]
    out["workload"] = ("1025x1025x513, 8 levels, cos(x z^2) sin(y^3), Dirichlet, FullWeighting + red-black SOR "
                       f"nu=2, F-cycle corrections, tolerances {', '.join(f'{t:g}' for t in tols)}, maxiter {maxiter}")
    for e in solvers.values():
        e.close()
    return out


def bench_batched(mgp, torch, device=0, count=256, tol=1e-8):
    """256 independent Dirichlet problems, cubes 2^k+1 with k uniform in {5,6,7,8}
    (k_i = 5 + splitmix64(i) % 4), levels k-1, right-hand side uniform in [-1,1] from the
    per-problem seed splitmix64(2^32 + i), zero boundary values; F-cycle corrections to 1e-8
    relative residual.  One batch: every level operation of every problem is one persistent
    work-list launch.  FP32 corrections (FP64 refinement) against an all-FP64 batch."""
    out = {}
    ks = [5 + splitmix64(i) % 4 for i in range(count)]
    dof = sum((2 ** k + 1) ** 3 for k in ks)
    for name, inner in (("fp64", mgp.F64), ("mixed", mgp.F32)):
        b = mgp.Batch(mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, inner, "Fcycle", 2, max_problems=count, device=device)
        ids = []
        for i, k in enumerate(ks):
            n = 2 ** k + 1
            pid = b.add((n, n, n), k - 1, 1.0 / (n - 1))
            ids.append(pid)

        def load():
            for i, pid in enumerate(ids):
                s = b.problem(pid)
                s.zero_u(0)
                s.fill_uniform(splitmix64((1 << 32) + i))
                b.restart(pid)

        load()
        b.solve(tol, 100)  # warm-up (schedules and graphs)
        load()
        stream = torch.cuda.ExternalStream(b.problem(ids[0]).stream_handle, device=f"cuda:{device}")
        t0 = time.perf_counter()
        steps = b.solve(tol, 100)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        its = [b.status(pid).iterations for pid in ids]
        rels = [b.status(pid).rel_res for pid in ids]
        out[name] = {"s_per_batch": sec, "solves_per_s": count / sec, "dof_per_s": dof / sec, "steps": steps,
                     "max_iterations": int(max(its)), "mean_iterations": float(np.mean(its)),
                     "max_rel_res": float(max(rels)), "launches_per_step": b.launches_per_step()}
        b.close()
        del stream
    # the plain FP64 form: each problem alone, FP64 F-cycles of the reference's solver to the
    # same tolerance (graphs captured by a first solve, then the right-hand side reloaded)
    solvers = []
    for i, k in enumerate(ks):
        n = 2 ** k + 1
        e = mgp.Solver((n, n, n), k - 1, 1.0 / (n - 1), (0,) * 6, mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, mgp.F64, 100,
                       1, tol, device=device)
        e.fill_uniform(splitmix64((1 << 32) + i))
        e.solve("Fcycle", 2)
        e.zero_u(0)
        e.fill_uniform(splitmix64((1 << 32) + i))
        solvers.append(e)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its, rels = [], []
    for e in solvers:
        st = e.solve("Fcycle", 2)
        its.append(st.iterations)
        rels.append(st.rel_res)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    for e in solvers:
        e.close()
    out["plain_fp64"] = {"s_total": sec, "solves_per_s": count / sec, "dof_per_s": dof / sec,
                         "max_iterations": int(max(its)), "mean_iterations": float(np.mean(its)),
                         "max_rel_res": float(max(rels)), "form": "one problem at a time, FP64 F-cycles"}
    out["speedup_mixed_over_fp64"] = out["fp64"]["s_per_batch"] / out["mixed"]["s_per_batch"]
    out["speedup_mixed_over_plain_fp64"] = sec / out["mixed"]["s_per_batch"]
    out["workload"] = f"{count} Dirichlet cubes 2^k+1, k in 5..8, {dof} DOF total, FW + red-black SOR, tol {tol}"
    return out


SERVED_ARMS = (("fp64", "F64", 32), ("mixed", "F32", 32), ("fp64_serial", "F64", 1))


def bench_served(mgp, device=0, count=120, rates=(50.0, 2000.0), seed=0, arms=SERVED_ARMS, warm_count=None):
    """Open-loop Poisson arrivals of `count` requests at each rate: boxes 2^k+1 per axis
    (k in 5..9 for x and y, 5..8 for z), Dirichlet / Neumann / mixed, 8 random sine modes,
    tolerance 1e-8; continuous batching with admission by free HBM.  By default a bounded
    sample of the 10,000-request stream; `--served-full` runs the whole stream at 50, 200, 1000
    and 2000 requests/s.  At 50/s the server keeps up with the arrivals (latency is the
    measure); at 2000/s the requests queue up (solves/s is the server's capacity).
    fp64_serial: one request on the device at a time (a queue in front of the FP64 solver)."""
    from mgp import serve

    out = {}
    for rate in rates:
        res = {}
        for name, inner, slots in arms:
            srv = serve.Server(inner=getattr(mgp, inner), max_batch=slots, device=device)
            # warm-up pass over (a prefix of) the same stream: the memory pool, the page-locked
            # landing buffer and the kernels' first-launch costs are paid before the measured pass
            srv.run(serve.make_stream(warm_count or count, rate, seed, kmax_z=8))
            reqs = serve.make_stream(count, rate, seed, kmax_z=8)  # largest box 513x513x257
            res[name] = srv.run(reqs)
            srv.close()
        if "fp64" in res and "mixed" in res:
            res["speedup_mixed_over_fp64"] = res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"]
        if "fp64_serial" in res and "mixed" in res:
            res["speedup_mixed_over_fp64_serial"] = res["mixed"]["solves_per_s"] / res["fp64_serial"]["solves_per_s"]
        out[f"rate_{int(rate)}"] = res
    out["workload"] = (f"{count} requests per rate, Poisson arrivals at {', '.join(str(int(r)) for r in rates)}/s, "
                       "sides 2^k+1, tol 1e-8" + (" (sample of the stream)" if count < 10000 else ""))
    return out


def run_served_full(args) -> int:
    """The whole served workload: 10,000 requests at each of 50, 200, 1000 and 2000 requests/s,
    FP64 and FP32-correction servers (warm-up on a 200-request prefix).  About a quarter of an
    hour on one B200; prints one JSON line."""
    import torch

    import mgp

    torch.cuda.set_device(0)
    res = bench_served(mgp, 0, count=10000, rates=(50.0, 200.0, 1000.0, 2000.0), arms=SERVED_ARMS[:2],
                       warm_count=200)
    print(json.dumps({"served_full": res}))
    return 0


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except (ValueError, KeyError):
            pass
    return 6650.0, "fallback"


def cycle_model_bytes() -> float:
    """Algorithmic bytes of one F-cycle + convergence check (FP64), composed from the
    per-operation compulsory traffic: sweep 3sN, residual 3sN, FullWeighting s(N+Nc),
    zero coarse u sNc, prolong+add s(2N+Nc), convergence check 2sN0."""
    s = 8.0
    dims = [tuple((d >> l) + 1 if l else d for d in DIMS) for l in range(LEVELS)]
    n = [a * b * c for a, b, c in dims]
    L = LEVELS
    total = 0.0

    def relax(l):
        return NSMOOTH * 3 * s * n[l]

    def setup(l):
        return 3 * s * n[l] + s * (n[l] + n[l + 1]) + s * n[l + 1]

    def padd(l):
        return s * (2 * n[l] + n[l + 1])

    def V(l):
        t = relax(l)
        if l >= L - 1:
            return t
        return t + setup(l) + V(l + 1) + padd(l) + relax(l)

    def F(l):
        t = relax(l) + setup(l)
        if l < L - 2:
            t += F(l + 1)
        t += V(l + 1) + padd(l)
        if l == 0:
            t += V(0)
        return t

    total = F(0) + 2 * s * n[0]
    return total


def cpu_reference(steps: int, warm: int, threads: int | None = None):
    """The reference's own OpenMP CPU build timed by its own solve_time()."""
    from oracle.oracle import REF_BIN, RefRun

    if not REF_BIN.exists():
        return None
    threads = threads or os.cpu_count() or 1
    st = RefRun().run(DIMS, LEVELS, bc=BC, restriction="fw", relaxation="jacobi", problem=2, mode="time",
                      cycle="Fcycle", nsmooth=NSMOOTH, maxiter=steps, tol=0.0, h=H, threads=threads,
                      extra={"warm": warm, "timed": steps, "miniter": steps}, timeout=1800)
    secs = st.stats["time"][-1]
    iters = st.stats["iters"][-1]
    return {"value": NDOF * iters / secs, "seconds": secs, "cycles": iters, "threads": threads}


def cpu_reference_best(cycles: int, warm: int):
    """The reference's CPU build at its fastest OpenMP thread count: one timed cycle after one
    warm-up cycle at each of 1, 2, 4, ..., nproc threads (its build can be slower with more
    threads; the first cycle after allocation also pays the arrays' first-touch page faults),
    then the bounded sample of `cycles` cycles after `warm` warm-up cycles at the fastest count."""
    nproc = os.cpu_count() or 1
    counts = []
    t = 1
    while t < nproc:
        counts.append(t)
        t *= 2
    counts.append(nproc)
    sweep = {}
    for t in counts:
        r = cpu_reference(1, 1, threads=t)
        if r is None:
            return None
        sweep[t] = r["value"]
    best_t = max(sweep, key=sweep.get)
    res = cpu_reference(cycles, warm, threads=best_t)
    sweep[best_t] = max(sweep[best_t], res["value"])
    res["sweep"] = {str(k): v for k, v in sorted(sweep.items())}
    res["warm"] = warm
    return res


def run_reference_arm(args):
    world, rank, local, pg = dist_setup(args.gpus)
    if rank != 0:
        return 0
    from oracle.oracle import REF_BIN

    if not REF_BIN.exists():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/ref_oracle not built"}))
        return 0
    # Bounded sample: the reference takes ~0.3-1 s per F-cycle of this grid, so at most
    # REF_ARM_CYCLES timed cycles (after at most 2 warm-up cycles) keep the run to a minute or
    # so whatever --steps says; the metric is per cycle, so the sample size does not change it.
    res = cpu_reference_best(min(args.steps, REF_ARM_CYCLES), min(args.warmup, 2))
    cores = res["threads"]
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / max(1, res["cycles"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic x^3 y^2 z problem)", "config": {"workload": WORKLOAD},
            "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{int(res['cycles'])} F-cycles on the full grid after {res['warm']} "
                                       f"warm-up cycles, OMP_NUM_THREADS={cores} (fastest of a thread sweep)"},
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "thread_sweep": res["sweep"]}
    print(json.dumps(line))
    return 0


def run_iterations_only(args) -> int:
    """The workload's solve iterations and nothing else (no timing, no other workloads): the
    command that ncu launch lists are taken from."""
    import torch

    import mgp

    torch.cuda.set_device(0)
    ps = build_solver(mgp, 0, maxiter=max(1, args.warmup + args.steps), pinned=False, flags=args.engine_flags)
    ps.to_device()
    eng = ps.engine
    eng.set_iteration_limits(args.warmup + args.steps, args.warmup + args.steps, 0.0)
    st = eng.solve("Fcycle", NSMOOTH)
    torch.cuda.synchronize()
    print(json.dumps({"iterations": st.cycles_run, "kernel_launches": st.kernel_launches, "rel_res": st.rel_res}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mgp", choices=["mgp", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernels", action="store_true", help="time each level-0 kernel alone")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the mixed-precision, batched and served workloads")
    ap.add_argument("--served-requests", type=int, default=120)
    ap.add_argument("--served-full", action="store_true",
                    help="run only the whole served workload (10,000 requests at 50/200/1000/2000 per second)")
    ap.add_argument("--iterations-only", action="store_true",
                    help="run --warmup + --steps solve iterations of the workload and exit (for ncu launch lists)")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the built-in launch shapes (no mgp_autotune search before timing)")
    ap.add_argument("--engine-flags", type=int, default=0,
                    help="extra MGP_FLAG_* bits for the benchmarked solver (e.g. 256: wavefront passes)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.kernels:
        return run_kernels(args)
    if args.iterations_only:
        return run_iterations_only(args)
    if args.served_full:
        return run_served_full(args)

    world, rank, local, pg = dist_setup(args.gpus)
    import torch

    import mgp

    torch.cuda.set_device(local)
    # Each rank: an independent replica of the whole solve on its own GPU.
    ps = build_solver(mgp, local, maxiter=args.steps, pinned=True, flags=args.engine_flags)
    ps.to_device()
    eng = ps.engine
    tuning = None
    if not args.no_tune:
        # launch shapes searched on this GPU (fields restored afterwards); bit-identical results
        t0 = time.time()
        tuning = eng.autotune("Fcycle", NSMOOTH, force=True)
        tuning["search_s"] = time.time() - t0
    stream = torch.cuda.ExternalStream(eng.stream_handle, device=f"cuda:{local}")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # warm-up (captures and instantiates the CUDA graph); the sampler's first readings
        # land here, under load, before the timed region
        eng.set_iteration_limits(args.warmup, args.warmup, 0.0)
        eng.solve("Fcycle", NSMOOTH)
        t_end = time.time() + 0.6
        while time.time() < t_end:
            eng.solve("Fcycle", NSMOOTH)
        eng.set_iteration_limits(args.steps, args.steps, 0.0)
        barrier(pg)
        torch.cuda.synchronize()
        ev0.record(stream)
        st = eng.solve("Fcycle", NSMOOTH)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    sec = ev0.elapsed_time(ev1) / 1e3
    assert st.cycles_run == args.steps, (st.cycles_run, args.steps)
    tmax = max_over_ranks(pg, sec, local)
    value = aggregate(NDOF * args.steps, world, tmax)

    # e2e through the reference-facing API: to_device + solve(4 F-cycles) + to_host per request
    eng.set_iteration_limits(E2E_CYCLES, E2E_CYCLES, 0.0)
    ps.to_device()
    ps.solve("Fcycle", NSMOOTH)
    ps.to_host()
    n_e2e = max(2, min(5, args.steps // 4))
    barrier(pg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n_e2e):
        ps.to_device()
        ps.solve("Fcycle", NSMOOTH)
        ps.to_host()
    e1.record(stream)
    e1.synchronize()
    barrier(pg)
    e2e_sec = max_over_ranks(pg, e0.elapsed_time(e1) / 1e3 / n_e2e, local)
    e2e_value = aggregate(NDOF * E2E_CYCLES, world, e2e_sec)
    esz = 8
    lv = ps.engine.level[0]
    face_elems = sum(a * b * c for a, b, c in lv.face_shape)
    h2d = (4 * lv.size + face_elems) * esz
    d2h = 3 * lv.size * esz

    # dominant kernel roofline
    ksec, kbytes = kernel_roofline(mgp, ps, torch, stream)
    peak, peak_kind = measured_peaks()
    achieved = kbytes / ksec / 1e9
    cyc_bytes = cycle_model_bytes()
    cyc_achieved = cyc_bytes / (sec / args.steps) / 1e9

    if rank != 0:
        return 0
    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_best(CPU_BASELINE_CYCLES, 1)
        except Exception as exc:  # noqa: BLE001 -- the baseline is informative only
            cpu = {"error": str(exc)}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tmax / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (analytic x^3 y^2 z problem on the host)",
        "config": {"workload": WORKLOAD, "l2": "inputs larger than L2 (4 x 143 MB fine arrays)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "step": f"to_device + {E2E_CYCLES}-cycle solve + to_host", "ms_per_request": 1e3 * e2e_sec},
        "roofline": {"bound": "hbm", "kernel": "k_stencil<double,OP_JACOBI> level 0", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": JACOBI_SWEEP_DRAM_BYTES, "traffic_source": "ncu dram__bytes_read+write, 1 launch",
                     "algorithmic_bytes_per_launch": kbytes, "launch_us": ksec * 1e6},
        "cycle_roofline": {"model_bytes_per_cycle": cyc_bytes, "achieved": cyc_achieved, "peak": peak,
                           "unit": "GB/s", "frac": cyc_achieved / peak, "ms_per_cycle": 1e3 * sec / args.steps},
        "gpu_launches": int(st.kernel_launches),
        "clocks": clocks,
        "rel_res_after": st.rel_res,
    }
    if tuning is not None:
        line["tuning"] = {"untuned_ms_per_iteration": tuning["untuned_ms"], "tuned_ms_per_iteration": tuning["tuned_ms"],
                          "search_s": tuning["search_s"],
                          "params_per_level": {"order": ["relax_planes", "resid_planes", "norm_planes", "setup_form",
                                                         "setup_planes", "wave_off", "tail_on", "prolong_sweep_off"],
                                               "values": tuning["params"]}}
    if not args.no_extra:
        for key, fn in (("c1_fcycle_65", lambda: bench_c1(mgp, torch, local)),
                        ("c2_vcycle_513x257x129", lambda: bench_c2(mgp, torch, local)),
                        ("mixed_precision", lambda: bench_mixed(mgp, torch, local)),
                        ("batched", lambda: bench_batched(mgp, torch, local)),
                        ("served", lambda: bench_served(mgp, local, count=args.served_requests))):
            try:
                line[key] = fn()
            except Exception as exc:  # noqa: BLE001 -- reported in the line, the main metric stands
                line[key] = {"error": repr(exc)}
    if cpu and "value" in cpu:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["threads"], "kind": "reference",
                                "sample": f"{int(cpu['cycles'])} F-cycles of the same workload after "
                                          f"{cpu['warm']} warm-up cycle, reference OpenMP build, "
                                          f"OMP_NUM_THREADS={cpu['threads']} (fastest of a thread sweep)",
                                "thread_sweep": cpu.get("sweep")}
    elif cpu:
        line["cpu_baseline"] = {"error": cpu.get("error")}
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
