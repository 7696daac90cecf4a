#!/usr/bin/env python3
"""Pressure-solve benchmark: ms per pressure solve to relative residual 1e-6.

Workload (default): the 5.3M-cell pressure-correction matrix: a 96^3 jittered
hex mesh of the unit cube (interior vertices +-0.15h, seed 1), each hex split
into six tetrahedra; face coefficients D_f |A_f| / |d_PN| with D per cell
log-uniform on [1e-3, 1] averaged over the face's two cells; Dirichlet p = 0 on
x = 1, Neumann elsewhere; b_i ~ N(0,1) V_i; reverse Cuthill-McKee order; float
values with the upward-rounded diagonal (a symmetric M-matrix). Solved with
AMG-PCG exactly as the reference's pressure solver is built
(make_solver(AmgPcg, ..., {SymmetricMMatrix}): V(5,5) L1-Jacobi, 3 pairing
passes, threshold 0.25), SolveControl{1e-6, 1e-12, max_iter}.

A step is one outer-iteration pressure solve as the reference's SIMPLEC step
runs it: refresh(A) then solve(A, x = 0, b). `value` is device time per step
with the matrix and right-hand side resident in HBM; `e2e` is the same step
through the public API with the matrix values and right-hand side copied in
from pinned host memory and x copied back, every step. Inputs (26.4M nonzeros,
318 MB of matrix + vectors) exceed the 126 MB L2, so no flush is needed between
steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

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
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ms per pressure solve to rel-res 1e-6: learned+mixed vs plain AMG-PCG, 1 B200"
UNIT = "ms/solve"


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _workload(args):
    from kutta_b200 import harness
    n = args.size
    s = harness.box_system(n, n, n, tet=True, seed=args.seed)
    return s


def _config(args, s, world):
    return {
        "workload": f"pressure_tet{args.size}: {args.size}^3 jittered hex x 6 tets, "
                    f"{s.n} cells, {s.nnz} nonzeros, RCM, seed {args.seed}",
        "solver": "AMG-PCG V(5,5) L1-Jacobi, SymmetricMMatrix (reference pressure defaults)",
        "rel_tol": 1e-6, "abs_tol": 1e-12, "max_iter": args.max_iter,
        "rows": s.n, "nnz": s.nnz, "l2_flush": "none: inputs exceed L2 (126 MB)",
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
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    e = d.get(kernel, {})
    if e.get("workload") != workload:
        return None
    return e.get("dram_bytes_per_launch")


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import numpy as np
    from kutta_b200 import linalg as L

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    s = _workload(args)
    opts = L.SolverOptions(structure=L.OperatorStructure.SymmetricMMatrix)
    t0 = time.perf_counter()
    solver = L.make_solver(L.SolverKind.AmgPcg, s, opts)
    setup_s = time.perf_counter() - t0
    a = L.upload(s, dev)
    b = torch.from_numpy(s.b).to(dev)
    x = torch.zeros(s.n, dtype=torch.float32, device=dev)
    control = L.SolveControl(1e-6, 1e-12, args.max_iter)
    stream = torch.cuda.current_stream()

    def step():
        solver.refresh(a)
        x.zero_()
        return solver.solve(a, x, b, control)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        st = step()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    solver.profile(True)
    launches0 = L.kernel_launches()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    start.record(stream)
    stats = [step() for _ in range(args.steps)]
    stop.record(stream)
    barrier()
    launches = L.kernel_launches() - launches0
    prof = solver.profile_read()
    solver.profile(False)
    clk = clocks.stop()
    ms = start.elapsed_time(stop) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # End to end through the public API with host buffers, every step.
    val_host = torch.from_numpy(s.val.astype(np.float32)).pin_memory()
    b_host = torch.from_numpy(s.b).pin_memory()
    x_host = torch.empty(s.n, dtype=torch.float32).pin_memory()
    a2 = L.upload(s, dev)
    b2 = torch.empty_like(b)

    def e2e_step():
        a2.val.copy_(val_host, non_blocking=True)
        b2.copy_(b_host, non_blocking=True)
        solver.refresh(a2)
        x.zero_()
        st = solver.solve(a2, x, b2, control)
        x_host.copy_(x, non_blocking=True)
        return st

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    barrier()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    e2e_steps = max(1, args.steps)
    for _ in range(e2e_steps):
        e2e_step()
    e_stop.record(stream)
    barrier()
    e2e_ms = e_start.elapsed_time(e_stop) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    last = stats[-1]
    # Accuracy of the returned x against the FP64 oracle is reported by
    # tests; here the true residual of the returned iterate in FP64.
    xr = x.double().cpu().numpy()
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    true_rel = float(np.linalg.norm(s.b.astype(np.float64) - A @ xr) / last.initial_residual)

    sweep_ms = prof["fine_sweep_ms"] / max(prof["fine_sweeps"], 1)
    achieved = prof["fine_sweep_bytes"] / (sweep_ms * 1e-3) / 1e9 if sweep_ms > 0 else None
    peak, peak_kind = _peaks()
    solve_gbs = prof["algorithmic_bytes"] / (ms * args.steps * 1e-3) / 1e9
    workload = f"pressure_tet{args.size}"
    line = {
        "metric": METRIC, "value": ms / world, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 reductions)",
        "data": "synthetic (seeded FV pressure matrix; no dataset)",
        "config": _config(args, s, world),
        "method": "plain FP32 AMG-PCG (reference arithmetic, bit-exact aggregation)",
        "iterations": last.iterations, "converged": last.converged,
        "relative_residual": last.final_residual / last.initial_residual,
        "true_relative_residual_fp64": true_rel,
        "setup_s": setup_s, "describe": solver.describe(),
        "solve_level_gbs": solve_gbs,
        "roofline": {
            "kernel": "k_smooth<false> (fine-level damped L1-Jacobi sweep, CSR row per thread)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
            "bytes_per_launch": prof["fine_sweep_bytes"], "launch_ms": sweep_ms,
            "launches_timed": prof["fine_sweeps"],
            "traffic": _traffic("k_smooth", workload),
        },
        "e2e": {"value": e2e_ms / world, "unit": UNIT,
                "h2d_bytes_per_step": 4 * s.nnz + 4 * s.n, "d2h_bytes_per_step": 4 * s.n},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    return line, s


def cpu_baseline(args, s, gpu_iterations):
    """The reference's own CPU path (serial by design: 1 core) on a bounded
    sample of the same workload: setup, one refresh, and the first
    `sample_iters` PCG iterations; per-solve time = refresh + per-iteration time
    x the iteration count the solve needs."""
    from oracle import ref
    if not ref.available():
        return None
    opts = ref.options(3, structure=1, use_make_solver=True)
    r = ref.solve(s, opts=opts, rel_tol=1e-6, abs_tol=1e-12, max_iter=args.cpu_sample_iters)
    per_iter = r.solve_s / max(r.iterations, 1)
    value_ms = (r.refresh_s + per_iter * gpu_iterations) * 1e3
    return {"value": value_ms, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"reference CPU path (oracle/_ref) on this workload: setup {r.setup_s:.1f} s, "
                      f"refresh {r.refresh_s * 1e3:.0f} ms, first {r.iterations} PCG iterations in "
                      f"{r.solve_s:.1f} s; per solve = refresh + {per_iter:.2f} s/iteration x "
                      f"{gpu_iterations} iterations", "cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} threads on host)"
    except OSError:
        pass
    return None


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation, timed on the
    host cores (serial by design, 1 thread), each step a bounded sample."""
    if rank != 0:
        return None
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) missing"}
    s = _workload(args)
    opts = ref.options(3, structure=1, use_make_solver=True)
    iters = args.reference_iterations
    times = []
    r = None
    for k in range(args.warmup + args.steps):
        r = ref.solve(s, opts=opts, rel_tol=1e-6, abs_tol=1e-12, max_iter=args.cpu_sample_iters)
        if k >= args.warmup:
            per_iter = r.solve_s / max(r.iterations, 1)
            times.append((r.refresh_s + per_iter * iters) * 1e3)
    value = statistics.median(times)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 reductions)", "data": "synthetic",
        "config": _config(args, s, world), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"per step: reference setup+refresh and the first "
                                   f"{r.iterations} PCG iterations; per solve = refresh + "
                                   f"per-iteration time x {iters} iterations", "cpu": _cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def profile_once(args):
    """One refresh and one solve of the workload (the command ncu captures)."""
    import torch
    from kutta_b200 import linalg as L
    s = _workload(args)
    solver = L.make_solver(L.SolverKind.AmgPcg, s,
                           L.SolverOptions(structure=L.OperatorStructure.SymmetricMMatrix))
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
    solver.refresh(a)
    st = solver.solve(a, x, b, L.SolveControl(1e-6, 1e-12, args.max_iter))
    torch.cuda.synchronize()
    print(json.dumps({"describe": solver.describe(), "iterations": st.iterations,
                      "relative_residual": st.final_residual / st.initial_residual}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=96)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--max-iter", type=int, default=2000)
    ap.add_argument("--cpu-sample-iters", type=int, default=2)
    ap.add_argument("--reference-iterations", type=int, default=0,
                    help="iterations the reference needs on this workload (per-solve scaling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="bench", choices=["bench", "profile"],
                    help="profile: one refresh + one solve (with --max-iter), for ncu captures")
    args = ap.parse_args()
    rank, world, local = _dist()
    if args.mode == "profile":
        profile_once(args)
        return
    if args.impl == "reference":
        if not args.reference_iterations:
            args.reference_iterations = REFERENCE_ITERATIONS.get((args.size, args.seed), 0)
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line))
        return
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    line, system = run_ours(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, system, line["iterations"])
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# Iterations the reference's CPU path takes on the default workloads (measured
# with oracle/_ref in full runs; used only to scale the reference arm's bounded
# per-iteration sample to a per-solve time).
REFERENCE_ITERATIONS = {}

if __name__ == "__main__":
    main()
