#!/usr/bin/env python3
"""Pressure-solve benchmark: ms per pressure solve to relative residual 1e-6,
learned+mixed solve vs plain FP32 AMG-PCG on one B200.

Workload (default): the 5.3M-cell pressure-correction matrix: a 96^3 jittered
hex mesh of the unit cube (interior vertices +-0.15h, seed 1), each hex split
into six tetrahedra; face coefficients D_f |A_f| / |d_PN| with D per cell
log-uniform on [1e-3, 1] averaged over the face's two cells; Dirichlet p = 0 on
x = 1, Neumann elsewhere; b_i ~ N(0,1) V_i; reverse Cuthill-McKee order; float
values with the upward-rounded diagonal (a symmetric M-matrix).

A step is one outer-iteration pressure solve as the reference's SIMPLEC step
runs it: refresh(A), then solve from x = 0 to ||b - A x|| <= 1e-6 ||b||
(SolveControl{1e-6, 1e-12, 2000}).

* `value`: the learned+mixed solve: the mixed-precision solve (FP64 iterative
  refinement around an FP32 AMG-PCG with BF16 coarse levels and a dense FP64
  coarsest solve; the FP64 true residual of the returned FP64 solution meets
  the tolerance) with the trained learned stage as its warm start.
  `mixed_alone` times the same solver without the stage, `learned_cycle` with
  the stage after every AMG cycle instead.
* `plain`: the reference's own method (make_solver(AmgPcg, SymmetricMMatrix):
  V(5,5) L1-Jacobi, bit-exact aggregation and arithmetic) on the same GPU. In
  FP32 it cannot reach 1e-6 on this matrix: the float-rounded exact solution
  already has relative residual 2.79e-6; it stops where the reference stops.

Device times come from CUDA events with the inputs resident in HBM; `e2e`
repeats the mixed step through the public API with the matrix values and the
right-hand side copied from pinned host memory and the FP64 solution copied
back, every step. Inputs (26.4M nonzeros, > 300 MB per pass) exceed the 126 MB
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

At N = 1 rank 0 adds entries after the timed work: `cpu_baseline` (the
reference's CPU path on a bounded sample), `fp64_oracle` (the returned x's
error against an FP64 oracle solution) and `other_configs` (the graded
near-wall matrix to 1e-8 and an unseen seed of the learned stage's 128^3
evaluation configuration, each device-timed).

Under torchrun (N > 1) every rank runs an independent replica (the solve does
not shard); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ms per pressure solve to rel-res 1e-6: learned+mixed vs plain AMG-PCG, 1 B200"
UNIT = "ms/solve"
REL_TOL = 1e-6



def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _max_over_ranks(value: float, world: int, device) -> float:
    """The largest of the ranks' values (every rank gets it): a multi-GPU time
    is the slowest rank's. world == 1 returns the value unchanged."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _workload(args):
    from kutta_b200 import harness
    n = args.size
    return harness.box_system(n, n, n, tet=True, seed=args.seed)


def _config(args, s, world):
    return {
        "workload": f"pressure_tet{args.size}: {args.size}^3 jittered hex x 6 tets, "
                    f"{s.n} cells, {s.nnz} nonzeros, RCM, seed {args.seed}",
        "rows": s.n, "nnz": s.nnz, "rel_tol": REL_TOL, "abs_tol": 1e-12,
        "max_iter": args.max_iter, "l2_flush": "none: inputs exceed L2 (126 MB)",
        "parallelism": f"replicas{world}" if world > 1 else "single",
    }


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [[p.strip() for p in line.split(",")] for line in open(self.path)]
        rows = [r for r in rows if len(r) >= 9]
        os.unlink(self.path)
        if not rows:
            return None
        num = lambda v: v.replace(".", "", 1).isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        mx = [float(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    e = json.loads(p.read_text()).get(kernel, {})
    return e.get("dram_bytes_per_launch") if e.get("workload") == workload else None


def _timed(step, count, stream, sync):
    import torch
    sync()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    results = [step() for _ in range(count)]
    stop.record(stream)
    sync()
    return start.elapsed_time(stop) / count, results


def run_ours(args, rank, world, local):
    import numpy as np
    import scipy.sparse as sp
    import torch
    import torch.distributed as dist
    from kutta_b200 import linalg as L

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    s = _workload(args)
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    b64 = s.b.astype(np.float64)
    control = L.SolveControl(REL_TOL, 1e-12, args.max_iter)

    def sync():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(ms):
        return _max_over_ranks(ms, world, dev)

    a = L.upload(s, dev)
    b = torch.from_numpy(s.b).to(dev)
    from kutta_b200 import learn
    stage = learn.trained_stage()

    # ---- learned+mixed: the metric's method, the measured value ----
    # The mixed-precision solve with the trained learned stage as its warm
    # start (one safeguarded step along G(b - A x0) before the refinement
    # loop), the cheaper of the stage's two placements.
    t0 = time.perf_counter()
    mixed = L.make_mixed_solver(s)
    mixed_setup = time.perf_counter() - t0
    mixed.set_learned(stage, L.LEARNED_WARM_START)
    x64 = torch.zeros(s.n, dtype=torch.float64, device=dev)

    def mixed_step():
        mixed.refresh(a)
        x64.zero_()
        return mixed.solve(a, x64, b, control)

    for _ in range(args.warmup):
        mixed_step()
    clocks = Clocks(local)
    clocks.start()
    launches0 = L.kernel_launches()
    ms, stats = _timed(mixed_step, args.steps, stream, sync)
    launches = L.kernel_launches() - launches0
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    last = stats[-1]
    x_value = x64.cpu().numpy()  # the measured solve's FP64 solution
    true_rel = float(np.linalg.norm(b64 - A @ x_value) / last.initial_residual)
    # The same steps again with profiling on, for the fine-sweep kernel time
    # and the algorithmic bytes. Profiling brackets individual sweeps with
    # events, so this pass launches kernels one by one instead of replaying
    # captured graphs; the sweep kernel itself is the same.
    mixed.profile(True)
    prof_ms, _ = _timed(mixed_step, args.steps, stream, sync)
    prof = mixed.profile_read()
    mixed.profile(False)

    # ---- end to end through the public API with host buffers ----
    val_host = torch.from_numpy(s.val.astype(np.float32)).pin_memory()
    b_host = torch.from_numpy(s.b).pin_memory()
    x_host = torch.empty(s.n, dtype=torch.float64).pin_memory()
    a2 = L.upload(s, dev)
    b2 = torch.empty_like(b)

    def e2e_step():
        a2.val.copy_(val_host, non_blocking=True)
        b2.copy_(b_host, non_blocking=True)
        mixed.refresh(a2)
        x64.zero_()
        st = mixed.solve(a2, x64, b2, control)
        x_host.copy_(x64, non_blocking=True)
        return st

    e2e_step()
    e2e_ms, _ = _timed(e2e_step, args.steps, stream, sync)
    e2e_ms = max_over_ranks(e2e_ms)
    mixed.refresh(a)

    # ---- the same solver without the stage, and with it after each cycle ----
    mixed.set_learned(None)
    mixed_step()
    alone_ms, astats = _timed(mixed_step, args.steps, stream, sync)
    alone_ms = max_over_ranks(alone_ms)
    mixed.set_learned(stage, L.LEARNED_CYCLE)
    mixed_step()
    cycle_steps = max(1, min(args.steps, 5))
    cycle_ms, cstats = _timed(mixed_step, cycle_steps, stream, sync)
    cycle_ms = max_over_ranks(cycle_ms)
    mixed.set_learned(None)

    def summary(step_ms, st, steps, method):
        return {"method": method, "ms_per_solve": step_ms, "iterations": st.iterations,
                "refinements": st.refinements, "converged": st.converged,
                "relative_residual": st.final_residual / st.initial_residual, "steps": steps}

    # ---- plain FP32 AMG-PCG: the reference's method on the same GPU ----
    t0 = time.perf_counter()
    plain = L.make_solver(L.SolverKind.AmgPcg, s,
                          L.SolverOptions(structure=L.OperatorStructure.SymmetricMMatrix))
    plain_setup = time.perf_counter() - t0
    x = torch.zeros(s.n, dtype=torch.float32, device=dev)

    def plain_step():
        plain.refresh(a)
        x.zero_()
        return plain.solve(a, x, b, control)

    plain_step()
    plain.profile(True)
    plain_ms, pstats = _timed(plain_step, max(1, args.plain_steps), stream, sync)
    pprof = plain.profile_read()
    plain.profile(False)
    plain_ms = max_over_ranks(plain_ms)
    plast = pstats[-1]

    def roofline(p, step_ms, steps, kernel_key):
        sweep_ms = p["fine_sweep_ms"] / max(p["fine_sweeps"], 1)
        achieved = p["fine_sweep_bytes"] / (sweep_ms * 1e-3) / 1e9 if sweep_ms > 0 else None
        peak, kind = _peaks()
        return {
            "kernel": "fine-level damped L1-Jacobi post-sweep (one row per thread; in the mixed "
                      "solve k_packed_smooth_dot2 on the packed fine rows, with the flexible "
                      "PCG's r.z and z.q fused; in the plain solve k_smooth on CSR)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": kind,
            "bytes_per_launch": p["fine_sweep_bytes"], "launch_ms": sweep_ms,
            "launches_timed": p["fine_sweeps"],
            "traffic": _traffic(kernel_key, f"pressure_tet{args.size}"),
            "solve_level_gbs": p["algorithmic_bytes"] / (step_ms * steps * 1e-3) / 1e9,
        }

    line = {
        "metric": METRIC, "value": ms / world, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 operator, bf16 coarse levels, f64 refinement/reductions/coarsest; "
                 "learned stage bf16 weights, f32 accumulation",
        "data": "synthetic (seeded FV pressure matrix; no dataset)",
        "config": _config(args, s, world),
        "method": mixed.describe() + " + learned warm start (packaged trained weights, "
                                     "tensor-core forward)",
        "refinements": last.refinements, "iterations": last.iterations,
        "converged": last.converged,
        "relative_residual": last.final_residual / last.initial_residual,
        "true_relative_residual_fp64": true_rel, "setup_s": mixed_setup,
        "mixed_alone": summary(alone_ms, astats[-1], args.steps, mixed.describe()),
        "learned_cycle": summary(cycle_ms, cstats[-1], cycle_steps,
                                 "as method, with the learned stage after each cycle "
                                 "(z += alpha G(r - A z)) instead of the warm start"),
        "plain": {
            "method": plain.describe() + " (reference arithmetic, bit-exact aggregation)",
            "ms_per_solve": plain_ms, "iterations": plast.iterations,
            "converged": plast.converged,
            "relative_residual": plast.final_residual / plast.initial_residual,
            "setup_s": plain_setup, "steps": max(1, args.plain_steps),
            "roofline": roofline(pprof, plain_ms, max(1, args.plain_steps), "k_smooth"),
            "speedup_of_value": plain_ms / ms,
        },
        "roofline": dict(roofline(prof, prof_ms, args.steps, "k_packed_smooth_dot2"),
                         timed_in="profiled pass of the same steps (kernels launched one by one)",
                         profiled_ms_per_step=prof_ms),
        "e2e": {"value": e2e_ms / world, "unit": UNIT,
                "h2d_bytes_per_step": 4 * s.nnz + 4 * s.n, "d2h_bytes_per_step": 8 * s.n},
        "gpu_launches": int(launches),
        "gpu_launches_per_step": int(launches) / args.steps,
        "clocks": clk,
    }
    return line, s, x_value


def _device_ms(fn, steps):
    import torch
    best, out = None, None
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best, out


def other_configs(args):
    """One device-timed refresh + solve (best of two) of the other
    configurations, at N = 1 after the timed work: the graded near-wall
    matrix to 1e-8 (mixed with and without the learned warm start, against
    plain FP32 AMG-PCG, which stops at its FP32 floor), an unseen seed of
    the learned stage's evaluation configuration (128^3 jittered hex, smooth
    log-normal D_f, Fourier right-hand side) to 1e-6, and the Coupled
    4x4-block solve on a 128^3 hex box (10 solves after 3 warm-ups)."""
    import numpy as np
    import scipy.sparse as sp
    import torch
    from kutta_b200 import learn
    from kutta_b200 import linalg as L
    stage = learn.trained_stage()
    out = {}

    def arms(s, b, rel_tol, plain_steps):
        A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
        a = L.upload(s)
        control = L.SolveControl(rel_tol, 1e-30, args.max_iter)
        row = {"rows": s.n, "nnz": s.nnz, "rel_tol": rel_tol}
        mixed = L.make_mixed_solver(s)
        x64 = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        for name, mode in (("mixed", 0), ("learned+mixed", L.LEARNED_WARM_START),
                           ("learned_cycle+mixed", L.LEARNED_CYCLE)):
            mixed.set_learned(stage if mode else None, mode)

            def step():
                mixed.refresh(a)
                x64.zero_()
                return mixed.solve(a, x64, b, control)
            ms, st = _device_ms(step, 2)
            xr = x64.cpu().numpy()
            row[name] = {"ms_per_solve": ms, "iterations": st.iterations,
                         "refinements": st.refinements, "converged": st.converged,
                         "true_relative_residual_fp64": float(
                             np.linalg.norm(b.cpu().numpy().astype(np.float64) - A @ xr) /
                             st.initial_residual)}
        mixed.set_learned(None)
        plain = L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
            structure=L.OperatorStructure.SymmetricMMatrix))
        x = torch.zeros(s.n, dtype=torch.float32, device="cuda")

        def pstep():
            plain.refresh(a)
            x.zero_()
            return plain.solve(a, x, b, control)
        ms, st = _device_ms(pstep, plain_steps)
        row["plain"] = {"ms_per_solve": ms, "iterations": st.iterations,
                        "converged": st.converged,
                        "relative_residual": st.final_residual / st.initial_residual}
        return row

    s = _graded(args)
    out["graded_1e-8"] = dict(
        workload=f"graded_tet{args.size}: {args.size}^3 x 6 tets, 10-layer 1000:1 band at z = 0, "
                 "D_f log-uniform [1e-6, 1]",
        **arms(s, torch.from_numpy(s.b).cuda(), 1e-8, 1))
    s = learn.system(128, 90001)
    b = torch.from_numpy(learn.fourier_rhs(s, np.random.default_rng(90001))).cuda()
    out["learned_eval_hex128"] = dict(
        workload="hex128, unseen seed 90001: 128^3 jittered hex, smooth log-normal D_f "
                 "(sigma 1.5, correlation 0.1), 16 Fourier modes + 10 % noise",
        **arms(s, b, 1e-6, 1))
    # The Coupled 4x4-block solve (`--mode coupled` at its defaults, without
    # the reference's CPU solve, which that mode adds).
    import copy
    cargs = copy.copy(args)
    cargs.steps, cargs.warmup, cargs.no_cpu_baseline = 10, 3, True
    out["coupled_hex128"] = run_coupled(cargs)
    return out


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} threads on host)"
    except OSError:
        pass
    return None


def _reference_run(args, s, max_iter):
    """The reference's own CPU path (oracle/_ref; serial by design, 1 core):
    make_solver(AmgPcg, SymmetricMMatrix) setup, refresh, then PCG from x = 0
    for at most `max_iter` iterations, each phase timed."""
    from oracle import ref
    opts = ref.options(3, structure=1, use_make_solver=True)
    return ref.solve(s, opts=opts, rel_tol=REL_TOL, abs_tol=1e-12, max_iter=max_iter)


def fp64_oracle(s, x, max_iter=20000):
    """The returned solution's error against an FP64 oracle solution x64 on
    the host cores. x64 = x + e, where e solves A e = b - A x (residual in
    FP64) by the oracle's FP64 Jacobi-PCG until x64's relative residual is
    about 1e-12 (stated in the result): the x64 of a CG from zero to 1e-12, in
    fewer iterations when x is already close. The oracle is the checker here,
    never the measured path; a failure is reported in the line instead of
    failing the run."""
    import numpy as np
    import scipy.sparse as sp
    t0 = time.perf_counter()
    try:
        from oracle import kutta_oracle as O
        x = np.asarray(x, np.float64)
        A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
        b = s.b.astype(np.float64)
        r = b - A @ x
        r_norm = float(np.linalg.norm(r))
        e, iterations = np.zeros(s.n), 0
        if r_norm > 1e-12 * np.linalg.norm(b):
            e, iterations = O.cg64(s, b=r, rel_tol=min(0.1, 1e-12 * np.linalg.norm(b) / r_norm),
                                   max_iter=max_iter)
        x64 = x + e
        return {"relative_error": float(np.linalg.norm(e) / np.linalg.norm(x64)),
                "oracle": "FP64 Jacobi-PCG on the residual equation (OpenMP, host cores)",
                "oracle_relative_residual": float(np.linalg.norm(b - A @ x64) /
                                                  np.linalg.norm(b)),
                "oracle_iterations": int(iterations), "seconds": time.perf_counter() - t0}
    except Exception as e:  # noqa: BLE001 - reported, not raised
        return {"unavailable": f"{type(e).__name__}: {e}"}


def cpu_baseline(args, s, iterations):
    """The reference's CPU path on a bounded sample of the workload (setup,
    refresh and the first --cpu-sample-iters PCG iterations, about 20 s),
    scaled to one solve by `iterations`: the iteration count of this run's
    plain GPU solve, whose arithmetic and iterates are the reference's (the
    GPU parity tests check the counts are equal). The full, unscaled solve is
    what `--impl reference` times."""
    from oracle import ref
    if not ref.available():
        return None
    r = _reference_run(args, s, args.cpu_sample_iters)
    per_iter = r.solve_s / max(r.iterations, 1)
    return {"value": (r.refresh_s + per_iter * iterations) * 1e3, "unit": UNIT, "cores": 1,
            "kind": "reference",
            "sample": f"reference CPU path (oracle/_ref, built from the reference sources): setup "
                      f"{r.setup_s:.1f} s (not counted), refresh {r.refresh_s * 1e3:.0f} ms, first "
                      f"{r.iterations} PCG iterations in {r.solve_s:.1f} s; per solve = refresh + "
                      f"{per_iter:.2f} s/iteration x {iterations} iterations (the plain GPU "
                      "solve's count in this run, equal to the reference's); extrapolated, "
                      "the reference arm times the full solve", "cpu": _cpu_model()}


def _write_workload(args, path):
    """--mode workload: the benchmark matrix and right-hand side, written as
    .npz for the reference arm, which reads it without loading this
    repository's generator library."""
    import numpy as np
    s = _workload(args)
    np.savez(path, row_ptr=s.row_ptr, col=s.col, diag=s.diag, val=s.val, b=s.b)


def _read_workload(args):
    """The workload generated in a child process (`--mode workload`), so the
    reference arm's process maps only the reference's own library."""
    import types
    import numpy as np
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "workload.npz")
        subprocess.run([sys.executable, str(ROOT / "bench.py"), "--mode", "workload",
                        "--size", str(args.size), "--seed", str(args.seed), "--out", path],
                       check=True)
        d = np.load(path)
        s = types.SimpleNamespace(**{k: d[k] for k in d.files})
    s.n, s.nnz = len(s.diag), len(s.col)
    return s


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation on the host
    cores (serial by design: 1 thread). One complete solve is timed: the
    reference's make_solver setup (not counted, as the GPU arm's setup is not),
    then refresh and PCG from x = 0 until it stops (converged or not), the
    same step the GPU arm times. A solve takes about 9 minutes on the 5.3M-row
    matrix, so one timed solve is the whole run (no warm-up: a serial CPU
    solve has nothing to warm); `steps` and `warmup` say what ran."""
    if rank != 0:
        return None
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference CPU build) is missing"}
    s = _read_workload(args)
    r = _reference_run(args, s, args.max_iter)
    value = (r.refresh_s + r.solve_s) * 1e3
    sample = (f"one complete reference solve on the host, timed: setup {r.setup_s:.1f} s (not "
              f"counted), refresh {r.refresh_s * 1e3:.0f} ms, PCG {r.iterations} iterations in "
              f"{r.solve_s:.1f} s, relative residual {r.final_residual / r.initial_residual:.3e}, "
              f"converged {r.converged}")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1,
        "warmup": 0, "requested": {"steps": args.steps, "warmup": args.warmup},
        "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 reductions)",
        "data": "synthetic (seeded FV pressure matrix; no dataset)",
        "config": _config(args, s, world), "impl": "reference",
        "method": r.describe, "iterations": r.iterations, "converged": r.converged,
        "relative_residual": r.final_residual / r.initial_residual,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": sample, "cpu": _cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def profile_once(args):
    """One refresh and one solve of the workload (the command ncu captures)."""
    import torch
    from kutta_b200 import linalg as L
    s = _workload(args)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    if args.method == "mixed":
        solver = L.make_mixed_solver(s)
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    else:
        solver = L.make_solver(L.SolverKind.AmgPcg, s,
                               L.SolverOptions(structure=L.OperatorStructure.SymmetricMMatrix))
        x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
    solver.refresh(a)
    st = solver.solve(a, x, b, L.SolveControl(REL_TOL, 1e-12, args.max_iter))
    torch.cuda.synchronize()
    print(json.dumps({"describe": solver.describe(), "iterations": st.iterations,
                      "relative_residual": st.final_residual / st.initial_residual}))


def _graded(args, coeff_seed=0):
    from kutta_b200 import harness
    return harness.box_system(args.size, args.size, args.size, tet=True, seed=args.seed,
                              band_layers=10, aspect=1000.0, ratio=1.2, dmin=1e-6, dmax=1.0,
                              coeff_seed=coeff_seed)


def _blend(values, diag, boundary, row_ptr, fresh, keep):
    """keep * values + (1 - keep) * fresh for the off-diagonal entries (face
    coefficients are linear in D_f, so this blends the D fields), each
    diagonal recomputed as the upward-rounded float of its off-diagonal
    magnitudes plus the blended boundary term (the M-matrix construction)."""
    import numpy as np
    out = keep * values + (1.0 - keep) * fresh.val
    out = out.astype(np.float32).astype(np.float64)
    bnd = keep * boundary + (1.0 - keep) * fresh.boundary
    off = np.abs(out)
    off[diag] = 0.0
    total = np.add.reduceat(off, row_ptr[:-1]) + bnd
    d = total.astype(np.float32)
    d = np.where(d.astype(np.float64) < total, np.nextafter(d, np.float32(np.inf)), d)
    out[diag] = d.astype(np.float64)
    return out, bnd


def run_sequence(args):
    """Successive pressure solves as outer iterations produce them: the graded
    tet mesh, a right-hand side of 16 seeded Fourier modes over the cell
    centroids whose phases drift 0.01 rad per solve, and D_f blended toward a
    fresh seeded field with factor 0.7 every 50 solves, refreshing the
    solvers then. Each solve starts from the previous solution and runs to
    rel_tol relative to its own initial residual; the learned+mixed arm first
    corrects that start by the learned warm start (one safeguarded step along
    G(b - A x_prev), packaged trained weights). Reports total and per-solve
    p50/p99 device time for the mixed solve with and without the learned warm
    start and for the plain FP32 AMG-PCG."""
    import numpy as np
    import torch
    from kutta_b200 import linalg as L
    torch.cuda.set_device(0)
    s = _graded(args)
    values, boundary = s.val.copy(), s.boundary.copy()
    a = L.upload(s)
    centroid = torch.from_numpy(s.centroid).cuda()
    volume = torch.from_numpy(s.volume).cuda()
    rng = np.random.default_rng(args.seed)
    k = torch.from_numpy(rng.integers(1, 5, size=(16, 3)) * 2 * np.pi).cuda()
    amp = torch.from_numpy(rng.normal(size=16)).cuda()
    phase0 = torch.from_numpy(rng.uniform(0, 2 * np.pi, size=16)).cuda()

    def rhs(t):
        arg = centroid @ k.T + phase0 + 0.01 * t
        return ((torch.sin(arg) @ amp) * volume).to(torch.float32)

    control = L.SolveControl(args.rel_tol, 1e-30, args.max_iter)
    from kutta_b200 import learn
    stage = learn.trained_stage()
    arms = {"mixed": L.make_mixed_solver(s), "learned+mixed": L.make_mixed_solver(s),
            "plain": L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
                structure=L.OperatorStructure.SymmetricMMatrix))}
    x = {"mixed": torch.zeros(s.n, dtype=torch.float64, device="cuda"),
         "learned+mixed": torch.zeros(s.n, dtype=torch.float64, device="cuda"),
         "plain": torch.zeros(s.n, dtype=torch.float32, device="cuda")}
    times = {name: [] for name in arms}
    refresh_ms = {name: 0.0 for name in arms}
    iters = {name: [] for name in arms}
    conv = {name: 0 for name in arms}
    for name, solver in arms.items():
        solver.refresh(a)
    arms["learned+mixed"].set_learned(stage, L.LEARNED_WARM_START)
    for t in range(args.solves):
        if t > 0 and t % 50 == 0:
            fresh = _graded(args, coeff_seed=1000 + t)
            values, boundary = _blend(values, s.diag, boundary, s.row_ptr, fresh, 0.7)
            a.val.copy_(torch.from_numpy(values.astype(np.float32)))
            for name, solver in arms.items():
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                solver.refresh(a)
                e1.record()
                torch.cuda.synchronize()
                refresh_ms[name] += e0.elapsed_time(e1)
        b = rhs(t)
        for name, solver in arms.items():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            st = solver.solve(a, x[name], b, control)
            e1.record()
            torch.cuda.synchronize()
            times[name].append(e0.elapsed_time(e1))
            iters[name].append(st.iterations)
            conv[name] += int(st.converged)
    out = {"mode": "sequence", "solves": args.solves, "rel_tol": args.rel_tol,
           "workload": f"graded_tet{args.size}: {args.size}^3 x 6 tets, 10-layer 1000:1 band at "
                       f"z=0, D_f log-uniform [1e-6, 1], {s.n} cells, {s.nnz} nonzeros",
           "warm_start": "previous solution; learned+mixed: previous solution corrected by "
                         "the learned warm start"}
    for name, solver in arms.items():
        ts = sorted(times[name])
        out[name] = {"method": solver.describe(), "total_ms": sum(ts),
                     "p50_ms": ts[len(ts) // 2], "p99_ms": ts[min(len(ts) - 1, int(0.99 * len(ts)))],
                     "refresh_ms_total": refresh_ms[name],
                     "iterations_mean": float(np.mean(iters[name])),
                     "converged": f"{conv[name]}/{args.solves}"}
    return out


def run_graded(args):
    """One refresh + solve from zero to rel_tol on the graded tet matrix (the
    mixed-precision configuration), mixed against plain, device-timed."""
    import numpy as np
    import scipy.sparse as sp
    import torch
    from kutta_b200 import linalg as L
    torch.cuda.set_device(0)
    s = _graded(args)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    control = L.SolveControl(args.rel_tol, 1e-30, args.max_iter)
    out = {"mode": "graded", "rel_tol": args.rel_tol,
           "workload": f"graded_tet{args.size}: {s.n} cells, {s.nnz} nonzeros"}
    for name in ("mixed", "plain"):
        if name == "mixed":
            solver = L.make_mixed_solver(s)
            x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        else:
            solver = L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
                structure=L.OperatorStructure.SymmetricMMatrix))
            x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
        best = None
        for _ in range(max(1, args.steps)):
            x.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            solver.refresh(a)
            st = solver.solve(a, x, b, control)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        xr = x.cpu().numpy().astype(np.float64)
        true = float(np.linalg.norm(s.b.astype(np.float64) - A @ xr) / st.initial_residual)
        out[name] = {"method": solver.describe(), "ms_per_solve": best,
                     "iterations": st.iterations, "converged": st.converged,
                     "true_relative_residual_fp64": true}
    return out


def run_transport(args):
    """The non-symmetric twin of the pressure matrix (upwind convection by a
    divergence-free velocity plus nu = 1e-3 diffusion, diagonal under-relaxation
    0.7, on the same tet mesh): refresh + solve from zero to rel_tol with the
    reference's AMG-BiCGStab (make_solver defaults: V(5,5)) and BiCGStab-Jacobi,
    device-timed, with the FP64 true residual."""
    import numpy as np
    import scipy.sparse as sp
    import torch
    from kutta_b200 import harness
    from kutta_b200 import linalg as L
    torch.cuda.set_device(0)
    s = harness.convection_tet96(seed=args.seed, n=args.size)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    control = L.SolveControl(args.rel_tol, 1e-12, args.max_iter)
    out = {"mode": "transport", "rel_tol": args.rel_tol,
           "workload": f"convection_tet{args.size}: {s.n} cells, {s.nnz} nonzeros"}
    for name, kind in (("amg_bicgstab", L.SolverKind.AmgBicgstab),
                       ("bicgstab_jacobi", L.SolverKind.BicgstabJacobi)):
        t0 = time.perf_counter()
        solver = L.make_solver(kind, s, L.SolverOptions())
        setup = time.perf_counter() - t0
        x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
        best = None
        for _ in range(max(1, args.steps)):
            x.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            solver.refresh(a)
            st = solver.solve(a, x, b, control)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        xr = x.cpu().numpy().astype(np.float64)
        true = float(np.linalg.norm(s.b.astype(np.float64) - A @ xr) / st.initial_residual)
        out[name] = {"method": solver.describe(), "ms_per_solve": best, "setup_s": setup,
                     "iterations": st.iterations, "converged": st.converged,
                     "true_relative_residual_fp64": true}
    return out


def run_outer(args):
    """The steps on either side of the pressure solve in the steady solver's
    outer iteration (src/kutta/fv/steady_solver.cpp:1334-1366), on the
    headline mesh with synthetic face data (harness.fv_faces): the pressure
    assembly fused with the mixed solver's refresh against the assembly
    kernel followed by a separate refresh, and the flux and velocity
    corrections. Device-timed over --steps; algorithmic bytes per launch of
    the fused kernel for its HBM fraction."""
    import numpy as np
    import torch
    from kutta_b200 import harness
    from kutta_b200 import linalg as L
    torch.cuda.set_device(0)
    s = harness.pressure_tet96(seed=args.seed, n=args.size)
    c = harness.fv_faces(s.row_ptr, s.col, s.diag, seed=args.seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    fv = L.FvPressure(t(c.offsets), t(c.faces), t(c.sign), t(c.adjacent), t(c.entry),
                      t(c.coefficient), t(c.flux), -1)
    a = L.upload(s)
    rhs = torch.zeros(s.n, device="cuda")
    mixed = L.make_mixed_solver(s)
    rng = np.random.default_rng(args.seed)
    correction = t(rng.normal(size=s.n).astype(np.float32))
    flux = t(c.flux.copy())
    owner, neighbour, coefficient = t(c.owner), t(c.neighbour), t(c.coefficient)
    cells = [t(rng.uniform(0.5, 1.5, s.n).astype(np.float32)) for _ in range(3)]
    grads = [t(rng.normal(size=s.n).astype(np.float32)) for _ in range(3)]
    fields = [torch.zeros(s.n, device="cuda") for _ in range(4)]

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    fused_ms = timed(lambda: mixed.assemble_refresh(a, fv, rhs))
    separate_ms = timed(lambda: (L.fv_pressure_assemble(a, fv, rhs), mixed.refresh(a)))
    assemble_ms = timed(lambda: L.fv_pressure_assemble(a, fv, rhs))
    flux_ms = timed(lambda: L.fv_correct_flux(owner, neighbour, correction, coefficient, flux,
                                              c.internal))
    velocity_ms = timed(lambda: L.fv_correct_velocity(*cells, *grads, correction, *fields, 0.3))
    slots = len(c.faces)
    # offsets, four ints/floats per slot, gathered coefficient and flux per
    # slot, values written and re-read for the diagonal sum, rows and diag,
    # rhs; the L1 diagonal written by the fused form.
    assemble_bytes = 4 * (s.n + 1) + 16 * slots + 8 * slots + 8 * s.nnz + 8 * (s.n + 1) + 4 * s.n
    peak, kind = _peaks()
    return {"mode": "outer", "workload": f"pressure_tet{args.size}: {s.n} cells, {s.nnz} nonzeros, "
                                         f"{c.n_faces} faces ({c.internal} internal), {slots} "
                                         "cell-face slots",
            "assemble_refresh_fused_ms": fused_ms, "assemble_then_refresh_ms": separate_ms,
            "assemble_ms": assemble_ms, "correct_flux_ms": flux_ms,
            "correct_velocity_ms": velocity_ms,
            "assemble_algorithmic_bytes": assemble_bytes,
            "assemble_gbs": assemble_bytes / (assemble_ms * 1e-3) / 1e9,
            "assemble_frac_of_hbm": assemble_bytes / (assemble_ms * 1e-3) / 1e9 / peak,
            "peak_source": kind, "steps": args.steps}


def run_coupled(args):
    """The Coupled (4x4-block) pressure-velocity solve of the pseudo-transient
    Coupled scheme (src/kutta/fv/coupled_solver.cpp) on a structured hex box
    of --cells-per-side^3 cells (inlet, pressure outlet, walls, symmetry
    planes) with seeded flow fields (kutta_b200/coupled_harness.py): one step
    is the three momentum-diagonal captures plus CoupledSolver::solve
    (Jacobian assembly, Galerkin hierarchy refresh, block BiCGStab to the
    steady solver's control: relative 0.1, at most 20 iterations), device-
    timed over --steps after --warmup. The fine damped block-Jacobi sweep is
    timed on its own for its HBM fraction. With --coupled-mesh tet the box is
    split into six tets per hex (--cells-per-side^3 x 6 cells). The
    reference's own CPU solve (oracle/_ref) runs on a box of the same kind
    (--coupled-cpu-side, default the same box) as the CPU baseline."""
    import numpy as np
    import torch
    from kutta_b200 import coupled_harness as H
    from kutta_b200 import linalg as L
    torch.cuda.set_device(0)
    side = args.cells_per_side
    t0 = time.perf_counter()
    tet = args.coupled_mesh == "tet"
    mesh = (H.box_tet if tet else H.box_hex)(side, side, side)
    fields = H.flow_fields(mesh, args.seed)
    make_s = time.perf_counter() - t0
    n, nf, ni, entries, nnz = (int(v) for v in mesh["sizes"])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    dev = {k: (t(v) if isinstance(v, np.ndarray) else v) for k, v in fields.items()}
    rows, diag = t(mesh["pattern_row_ptr"]), t(mesh["pattern_diag"])
    t0 = time.perf_counter()
    solver = L.CoupledSolver(mesh, -1, L.CoupledOptions())
    setup_s = time.perf_counter() - t0
    control = L.SolveControl(args.coupled_rel_tol, 1e-12, args.coupled_max_iter)

    def step():
        for k, c in enumerate("uvw"):
            solver.capture_diagonal(k, rows, diag, dev["momentum_" + c], dev["physical_" + c])
        return solver.solve(dev, control)

    for _ in range(args.warmup):
        step()
    launches0 = L.kernel_launches()
    clocks = Clocks(0)
    clocks.start()
    ms, results = _timed(step, args.steps, torch.cuda.current_stream(), torch.cuda.synchronize)
    clk = clocks.stop()
    launches = (L.kernel_launches() - launches0) // args.steps
    st = results[-1]
    # The fine sweep alone: per cell x, b, next (float4 each) and the five
    # per-cell records (88 bytes); per internal cell-face slot the edge
    # (a, gx, gy, gz), h and (neighbour, face) (28 bytes); per face its
    # (sx, sy, sz, rc) record (16 bytes).
    width_slots = int(np.sum(mesh["adjacent"] >= 0))
    sweep_bytes = n * (48 + 88) + width_slots * 28 + nf * 16
    x4 = torch.randn(4 * n, device="cuda")
    b4 = torch.randn(4 * n, device="cuda")
    y4 = torch.empty(4 * n, device="cuda")
    for _ in range(3):
        solver.apply("smooth", x4, b4, y4)
    reps = 50
    sweep_ms, _ = _timed(lambda: solver.apply("smooth", x4, b4, y4), reps,
                         torch.cuda.current_stream(), torch.cuda.synchronize)
    spmv_ms, _ = _timed(lambda: solver.apply("spmv", x4, b4, y4), reps,
                        torch.cuda.current_stream(), torch.cuda.synchronize)
    peak, kind = _peaks()
    achieved = sweep_bytes / (sweep_ms * 1e-3) / 1e9
    out = {"mode": "coupled",
           "workload": f"coupled_{args.coupled_mesh}{side}: {side}^3 "
                       f"{'x 6 tet' if tet else 'hex'} box, {n} cells, {nf} faces, "
                       f"{width_slots} internal cell-face slots, 4 unknowns per cell",
           "method": solver.describe(), "control": [control.rel_tol, control.abs_tol,
                                                     control.max_iter],
           "ms_per_solve": ms, "iterations": st.iterations, "converged": st.converged,
           "initial_residual": st.initial_residual, "final_residual": st.final_residual,
           "gpu_launches_per_solve": launches, "setup_s": setup_s, "mesh_and_fields_s": make_s,
           "device_bytes": solver.bytes(), "steps": args.steps, "warmup": args.warmup,
           "fine_sweep": {"kernel": "k_cpl_fine_smooth", "ms": sweep_ms,
                          "bytes_per_launch": sweep_bytes, "achieved_gbs": achieved,
                          "peak_gbs": peak, "peak_source": kind, "frac": achieved / peak},
           "fine_spmv_ms": spmv_ms, "clocks": clk}
    if not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                cside = args.coupled_cpu_side or side
                case = ref.CoupledCase(tet, cside, cside, cside)
                f = H.flow_fields(case.arrays, args.seed)
                r = case.solve(f, ref.coupled_options(), rel_tol=control.rel_tol,
                               abs_tol=control.abs_tol, max_iter=control.max_iter, capture=False)
                cells = int(case.arrays["sizes"][0])
                out["cpu_baseline"] = {
                    "kind": "reference", "cores": 1,
                    "sample": f"the reference's CoupledSolver (oracle/_ref, serial CPU device) "
                              f"on a {cside}^3 {'x 6 tet' if tet else 'hex'} box of the same "
                              f"kind ({cells} cells)",
                    "ms_per_solve": r["solve_s"] * 1e3, "iterations": r["iterations"],
                    "construct_s": r["setup_s"], "describe": r["describe"],
                    "ns_per_cell_iteration": r["solve_s"] * 1e9 / cells / max(1, r["iterations"])}
                out["ns_per_cell_iteration"] = ms * 1e6 / n / max(1, st.iterations)
        except Exception as e:  # the baseline is informative only
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=96)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--max-iter", type=int, default=2000)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-iters", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the graded 1e-8 and learned-evaluation entries")
    ap.add_argument("--mode", default="bench",
                    choices=["bench", "profile", "sequence", "graded", "transport", "outer",
                             "workload", "coupled"],
                    help="profile: one refresh + one solve (with --max-iter), for ncu captures; "
                         "sequence: successive warm-started solves on the graded mesh; "
                         "graded: the graded matrix to --rel-tol (default 1e-8); "
                         "transport: the non-symmetric twin with AMG-BiCGStab and "
                         "BiCGStab-Jacobi (default 1e-6); outer: the pressure assembly fused "
                         "with the refresh, and the flux/velocity corrections; coupled: the "
                         "Coupled 4x4-block solve on a hex box")
    ap.add_argument("--method", default="mixed", choices=["mixed", "plain"])
    ap.add_argument("--solves", type=int, default=300, help="sequence mode: number of solves")
    ap.add_argument("--rel-tol", type=float, default=None,
                    help="sequence / graded modes (defaults 1e-6 / 1e-8)")
    ap.add_argument("--out", default=None, help="workload mode: the .npz to write")
    ap.add_argument("--cells-per-side", type=int, default=128, help="coupled mode: box side")
    ap.add_argument("--coupled-rel-tol", type=float, default=0.1)
    ap.add_argument("--coupled-max-iter", type=int, default=20)
    ap.add_argument("--coupled-mesh", default="hex", choices=["hex", "tet"],
                    help="coupled mode: hex box, or the box split into six tets per hex")
    ap.add_argument("--coupled-cpu-side", type=int, default=None,
                    help="coupled mode: box side of the reference CPU baseline "
                         "(default --cells-per-side)")
    args = ap.parse_args()
    rank, world, local = _dist()
    if args.mode == "workload":
        _write_workload(args, args.out)
        return
    if args.mode == "profile":
        profile_once(args)
        return
    if args.mode in ("sequence", "graded", "transport", "outer", "coupled"):
        if args.rel_tol is None:
            args.rel_tol = 1e-8 if args.mode == "graded" else 1e-6
        run = {"sequence": run_sequence, "graded": run_graded, "transport": run_transport,
               "outer": run_outer, "coupled": run_coupled}
        print(json.dumps(run[args.mode](args)))
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line))
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line, system, x = run_ours(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, system, line["plain"]["iterations"])
        line["fp64_oracle"] = fp64_oracle(system, x)
    if rank == 0 and world == 1 and not args.no_other_configs:
        line["other_configs"] = other_configs(args)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
