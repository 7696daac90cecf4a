"""Training and evaluation of the learned preconditioner stage.

Training data: seeded 64^3 jittered hex meshes of the unit cube with smooth
log-normal D_f (sigma 1.5, correlation length 0.1), right-hand sides of 16
seeded Fourier modes over the cell centroids plus 10 % white noise (scaled by
cell volume), and their solutions x computed by the plain FP32 AMG-PCG (the
reference's method) to relative 1e-6 or its FP32 floor. Each (matrix, b, x)
triple yields the pairs the stage sees inside the mixed solve: for an iterate
x_k (x_k = 0, and the mixed solve's iterate at relative 1e-3), z = M(r) is
one application of the mixed solve's AMG preconditioner to r = b - A x_k,
e = (x - x_k) - z the error it leaves and t = A e (FP64), so A e = t holds
exactly. Training runs the CUDA forward, the backward (its 32-wide layers on
the tensor cores) and the Adam step (b2_gnn_train_step) over the pairs in a
seeded random order, on the energy loss 1 - (c.t)^2 / ((c.Ac)(t.e)) for
c = G(t): the fraction of the error's A-energy that the best step along c
leaves.

Evaluation: unseen 128^3 seeds of the same family, the mixed solve to
relative 1e-6 with and without the stage attached, and the plain FP32
AMG-PCG, device-timed; the held-out energy loss on the same kind of pairs.

    python -m kutta_b200.learn --out weights.npy [--systems 250] [--rhs 8] [--steps 20000]
    python -m kutta_b200.learn --time-forward 128
"""
from __future__ import annotations

import argparse
import json
import pathlib
import sys
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


def _csr64(s: harness.HostSystem):
    import torch
    return torch.sparse_csr_tensor(torch.from_numpy(s.row_ptr.astype(np.int64)),
                                   torch.from_numpy(s.col.astype(np.int64)),
                                   torch.from_numpy(s.val.astype(np.float64)),
                                   (s.n, s.n)).cuda()


def pairs(s: harness.HostSystem, a: L.CsrMatrix, mixed: L.MixedSolver, b, x):
    """(t, e) pairs with A e = t exactly, from the plain solver's solution x of
    A x = b, for the iterates the stage meets inside the mixed solve: x_k = 0,
    and the mixed solve's own iterate at relative 1e-3. z is one application
    of the mixed solve's preconditioner to r = b - A x_k, e = (x - x_k) - z the
    error that remains, and t = A e in FP64 (the residual the stage sees, up
    to the plain solution's own small error)."""
    import torch
    A = _csr64(s)
    out = []
    xk = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    for tol in (None, 1e-3):
        if tol is not None:
            mixed.solve(a, xk, b, L.SolveControl(tol, 1e-30, 3000))
        r = (b.double() - A @ xk).float()
        z = torch.zeros(s.n, dtype=torch.float32, device="cuda")
        mixed.precondition(a, r, z)
        e = (x - xk) - z.double()
        t = A @ e
        out.append((t.float(), e.float()))
    return out


def geometry(s: harness.HostSystem):
    """The system's per-entry geometric face coefficients as a CUDA float32
    tensor (the learned stage's geometry gate input), or None."""
    import torch
    if s.geometry is None:
        return None
    return torch.from_numpy(s.geometry.astype(np.float32)).cuda()


def training_set(count: int, n_side: int, rhs_per_system: int, seed0: int,
                 with_geometry: bool = True):
    """[(device matrix, geometry, t, e)] from `count` systems x
    `rhs_per_system` solves of the plain FP32 AMG-PCG (the reference's method;
    to relative 1e-6 or its FP32 floor, whichever it reaches); geometry is
    None unless with_geometry."""
    import torch
    rng = np.random.default_rng(seed0)
    data = []
    for k in range(count):
        s = system(n_side, seed0 + k)
        a = L.upload(s)
        geo = geometry(s) if with_geometry else None
        plain = L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
            structure=L.OperatorStructure.SymmetricMMatrix))
        plain.refresh(a)
        mixed = L.make_mixed_solver(s)
        mixed.refresh(a)
        for _ in range(rhs_per_system):
            b = torch.from_numpy(fourier_rhs(s, rng)).cuda()
            x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
            plain.solve(a, x, b, L.SolveControl(1e-6, 1e-30, 3000))
            data.extend((a, geo, t, e) for t, e in pairs(s, a, mixed, b, x.double()))
        del plain, mixed
    return data


def train(stage: L.LearnedStage, data, steps: int, learning_rate: float, seed: int = 0):
    rng = np.random.default_rng(seed)
    order = np.concatenate([rng.permutation(len(data))
                            for _ in range(steps // max(1, len(data)) + 1)])
    bound = None
    losses = []
    for step in range(steps):
        a, geo, t, e = data[order[step]]
        if bound is not a:
            stage.set_geometry(geo)
            stage.bind(a)
            bound = a
        # Cosine decay to a tenth of the rate.
        lr = learning_rate * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * step / steps)))
        losses.append(stage.train_step(t, e, learning_rate=float(lr)))
        if (step + 1) % 1000 == 0:
            print(f"step {step + 1}: energy loss {np.mean(losses[-1000:]):.4f}", file=sys.stderr,
                  flush=True)
    return losses


def held_out_loss(stage: L.LearnedStage, data) -> float:
    """Mean energy loss over pairs, measured as a training step with a
    negligible rate on a copy of the weights (the weights are restored)."""
    w = stage.weights()
    bound, losses = None, []
    for a, geo, t, e in data:
        if bound is not a:
            stage.set_geometry(geo)
            stage.bind(a)
            bound = a
        losses.append(stage.train_step(t, e, learning_rate=1e-30))
        stage.set_weights(w)
    return float(np.mean(losses))


def evaluate(stage: L.LearnedStage | None, n_side: int, seeds, rel_tol: float = 1e-6,
             with_geometry: bool = True) -> dict:
    """Mixed solve with and without the stage, and the plain FP32 AMG-PCG."""
    import torch
    rng = np.random.default_rng(12345)
    results = []
    for seed in seeds:
        s = system(n_side, seed)
        a = L.upload(s)
        geo = geometry(s) if with_geometry else None
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
                x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            solver.refresh(a)
            if g is not None:
                g.set_geometry(geo)
                solver.set_learned(g, L.LEARNED_CYCLE)
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
                plain = L.make_solver(L.SolverKind.AmgPcg, s, L.SolverOptions(
                    structure=L.OperatorStructure.SymmetricMMatrix))
                plain.refresh(a)
                x_plain = torch.zeros(s.n, dtype=torch.float32, device="cuda")
                plain.solve(a, x_plain, b, L.SolveControl(1e-6, 1e-30, 3000))
                held_out = [(a, geo, t, e) for t, e in pairs(s, a, solver, b, x_plain.double())]
                row["held_out_energy_loss"] = held_out_loss(g, held_out)
                if geo is not None:
                    # The same weights with the gate off (theta = 0).
                    w = g.weights()
                    off = w.copy()
                    off[-2:] = 0.0
                    g.set_weights(off)
                    row["held_out_energy_loss_gate_off"] = held_out_loss(g, held_out)
                    g.set_weights(w)
            del solver
        results.append(row)
    return {"rel_tol": rel_tol, "mesh": f"{n_side}^3 jittered hex, smooth log-normal D_f "
                                         f"(sigma {FIELD_SIGMA}, corr {FIELD_CORR})",
            "results": results}


WEIGHTS = pathlib.Path(__file__).resolve().parent / "data" / "learned_stage.npy"


def trained_stage() -> L.LearnedStage:
    """The stage with the packaged weights (data/learned_stage.npy, written by
    this module's training run; data/learned_stage.json records the command
    and its report)."""
    g = L.LearnedStage(seed=1)
    g.set_weights(np.load(WEIGHTS))
    return g


def time_forward(n_side: int, repeats: int = 10) -> dict:
    """Device time of one tensor-core forward of an (untrained) stage on the
    n^3 evaluation mesh, averaged over `repeats` applications."""
    import torch
    s = system(n_side, 5)
    a = L.upload(s)
    g = L.LearnedStage(seed=1)
    g.bind(a)
    r = torch.from_numpy(fourier_rhs(s, np.random.default_rng(5))).cuda()
    z = torch.zeros(s.n, device="cuda")
    for _ in range(3):
        g.apply(r, z)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(repeats):
        g.apply(r, z)
    e1.record()
    torch.cuda.synchronize()
    return {"n": s.n, "nnz": int(s.row_ptr[-1]), "forward_ms": e0.elapsed_time(e1) / repeats}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", help="weights file (.npy) to write")
    ap.add_argument("--time-forward", type=int, metavar="N",
                    help="only time the forward on the N^3 mesh and exit")
    ap.add_argument("--systems", type=int, default=250)
    ap.add_argument("--rhs", type=int, default=8)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--eval-n", type=int, default=128)
    ap.add_argument("--eval-seeds", type=int, default=2)
    ap.add_argument("--no-geometry", action="store_true",
                    help="train without the geometry gate (theta stays 0)")
    ap.add_argument("--init", help="start from these weights (.npy) instead of random ones")
    args = ap.parse_args()
    if args.time_forward:
        print(json.dumps(time_forward(args.time_forward)))
        return
    if not args.out:
        ap.error("--out is required for training")
    t0 = time.time()
    data = training_set(args.systems, args.n, args.rhs, args.seed,
                        with_geometry=not args.no_geometry)
    t1 = time.time()
    stage = L.LearnedStage(seed=args.seed)
    if args.init:
        stage.set_weights(np.load(args.init))
    losses = train(stage, data, args.steps, args.lr)
    t2 = time.time()
    np.save(args.out, stage.weights())
    report = {"pairs": len(data), "solutions": len(data) // 2, "data_s": t1 - t0, "train_s": t2 - t1,
              "loss_first": float(np.mean(losses[:50])), "loss_last": float(np.mean(losses[-50:])),
              "evaluation": evaluate(stage, args.eval_n,
                                     [args.seed + 10_000 + k for k in range(args.eval_seeds)],
                                     with_geometry=not args.no_geometry)}
    print(json.dumps(report))
    pathlib.Path(args.out).with_suffix(".json").write_text(json.dumps(report, indent=1))


if __name__ == "__main__":
    main()
