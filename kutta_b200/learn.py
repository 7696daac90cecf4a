"""Training and evaluation of the learned preconditioner stage.

Training data: seeded 64^3 jittered hex meshes of the unit cube with smooth
log-normal D_f (sigma 1.5, correlation length 0.1), right-hand sides of 16
seeded Fourier modes over the cell centroids plus 10 % white noise (scaled by
cell volume), and their solutions computed by the mixed solve itself to
relative 1e-8 (FP64, rounded to float): (matrix, right-hand side, solution)
triples. Training runs the CUDA forward, backward and Adam kernels
(b2_gnn_train_step) over the triples, cycling through them in a seeded random
order.

Evaluation: unseen 128^3 seeds of the same family, the mixed solve to
relative 1e-6 with and without the stage attached, and the plain FP32
AMG-PCG, device-timed.

    python -m kutta_b200.learn --out weights.npy [--systems 48] [--steps 4000]
"""
from __future__ import annotations

import argparse
import json
import pathlib
import time

import numpy as np

from kutta_b200 import harness
from kutta_b200 import linalg as L

FIELD_SIGMA = 1.5
FIELD_CORR = 0.1


def fourier_rhs(s: harness.HostSystem, rng: np.random.Generator, modes: int = 16,
                noise: float = 0.1) -> np.ndarray:
    """sum_q a_q sin(2 pi k_q . x + p_q) + noise * N(0, 1) (relative to the
    modes' RMS), times the cell volume; k_q integer vectors in [1, 4]^3."""
    k = rng.integers(1, 5, size=(modes, 3)) * 2.0 * np.pi
    amp = rng.normal(size=modes)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    field = np.sin(s.centroid @ k.T + phase) @ amp
    field += noise * np.sqrt(np.mean(field ** 2)) * rng.normal(size=s.n)
    return (field * s.volume).astype(np.float32)


def system(n_side: int, seed: int) -> harness.HostSystem:
    return harness.box_system(n_side, n_side, n_side, tet=False, seed=seed,
                              field_sigma=FIELD_SIGMA, field_corr=FIELD_CORR)


def training_set(count: int, n_side: int, rhs_per_system: int, seed0: int):
    """[(device matrix, b, x)] with x the mixed solve's solution of A x = b."""
    import torch
    rng = np.random.default_rng(seed0)
    data = []
    for k in range(count):
        s = system(n_side, seed0 + k)
        a = L.upload(s)
        solver = L.make_mixed_solver(s)
        solver.refresh(a)
        for _ in range(rhs_per_system):
            b = torch.from_numpy(fourier_rhs(s, rng)).cuda()
            x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
            if st.converged:
                data.append((a, b, x.float()))
        del solver
    return data


def train(stage: L.LearnedStage, data, steps: int, learning_rate: float, seed: int = 0):
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(data))
    bound = None
    losses = []
    for step in range(steps):
        a, b, x = data[order[step % len(order)]]
        if bound is not a:
            stage.bind(a)
            bound = a
        # Cosine decay to a tenth of the rate.
        lr = learning_rate * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * step / steps)))
        losses.append(stage.train_step(b, x, learning_rate=float(lr)))
    return losses


def evaluate(stage: L.LearnedStage | None, n_side: int, seeds, rel_tol: float = 1e-6) -> dict:
    """Mixed solve with and without the stage, and the plain FP32 AMG-PCG."""
    import torch
    rng = np.random.default_rng(12345)
    results = []
    for seed in seeds:
        s = system(n_side, seed)
        a = L.upload(s)
        b = torch.from_numpy(fourier_rhs(s, rng)).cuda()
        row = {"seed": seed, "n": s.n}
        arms = [("mixed", None), ("plain", None)]
        if stage is not None:
            arms.insert(1, ("learned+mixed", stage))
        for name, g in arms:
            if name == "plain":
                solver = L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
                    structure=L.OperatorStructure.SymmetricMMatrix))
                x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
            else:
                solver = L.make_mixed_solver(s)
                if g is not None:
                    solver.set_learned(g)
                x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            solver.refresh(a)
            best, st = None, None
            for _ in range(3):
                x.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                st = solver.solve(a, x, b, L.SolveControl(rel_tol, 1e-30, 3000))
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            row[name] = {"ms": best, "iterations": st.iterations, "converged": bool(st.converged),
                         "relative_residual": st.final_residual / st.initial_residual}
            if g is not None:
                solver.set_learned(None)
            del solver
        results.append(row)
    return {"rel_tol": rel_tol, "mesh": f"{n_side}^3 jittered hex, smooth log-normal D_f "
                                         f"(sigma {FIELD_SIGMA}, corr {FIELD_CORR})",
            "results": results}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="weights file (.npy) to write")
    ap.add_argument("--systems", type=int, default=48)
    ap.add_argument("--rhs", type=int, default=4)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--eval-n", type=int, default=128)
    ap.add_argument("--eval-seeds", type=int, default=2)
    args = ap.parse_args()
    t0 = time.time()
    data = training_set(args.systems, args.n, args.rhs, args.seed)
    t1 = time.time()
    stage = L.LearnedStage(seed=args.seed)
    losses = train(stage, data, args.steps, args.lr)
    t2 = time.time()
    np.save(args.out, stage.weights())
    report = {"triples": len(data), "data_s": t1 - t0, "train_s": t2 - t1,
              "loss_first": float(np.mean(losses[:50])), "loss_last": float(np.mean(losses[-50:])),
              "evaluation": evaluate(stage, args.eval_n,
                                     [args.seed + 10_000 + k for k in range(args.eval_seeds)])}
    print(json.dumps(report))
    pathlib.Path(args.out).with_suffix(".json").write_text(json.dumps(report, indent=1))


if __name__ == "__main__":
    main()
