"""Real assembled pressure matrices as fixtures, with the reference's results.

Reads the two float pressure matrices the reference captured from its own FV
flow path on the NASA TMR bump case (validation/results/pressure_float/
bump_current_iteration15.coo.gz and bump_iteration18_reassembled.coo.gz in the
reference project; format: "n completed_steps" then "row col value" lines,
written by bench/bench_pressure.cpp:56-62), converts each to CSR, builds two
seeded right-hand sides, and runs the reference library built from its sources
(oracle/_ref) on it with the steady solver's pressure options
(make_amg_solver, SymmetricMMatrix; src/kutta/fv/steady_solver.cpp:578-580)
at the relative tolerance the solver uses per outer iteration (1e-3) and at
1e-6. Each fixture stores the matrix, the right-hand side, the reference's
iterations, residuals and solution, and digests of its AMG hierarchy.

Needs the reference sources on this machine; the fixtures are committed and the
tests read them without the reference.

    python tests/golden/make_real.py
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from kutta_b200 import harness  # noqa: E402
from oracle import ref  # noqa: E402

# The reference checkout (read-only), as for oracle/build.py.
REFERENCE = pathlib.Path(os.environ.get("KUTTA_REFERENCE", "/root/reference"))
SOURCE = REFERENCE / "validation" / "results" / "pressure_float"
CASES = {
    "tmr_bump_pressure_it15": "bump_current_iteration15.coo.gz",
    "tmr_bump_pressure_it18": "bump_iteration18_reassembled.coo.gz",
}
TOLERANCES = (1e-3, 1e-6)
RHS = ("random", "smooth")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def read_coo(path: pathlib.Path) -> harness.HostSystem:
    with gzip.open(path, "rt") as f:
        n, _steps = map(int, f.readline().split())
        data = np.loadtxt(f, dtype=np.float64, ndmin=2)
    rows, cols, vals = data[:, 0].astype(np.int64), data[:, 1].astype(np.int64), data[:, 2]
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = np.zeros(n + 1, np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    diag = np.array([row_ptr[i] + np.searchsorted(cols[row_ptr[i]:row_ptr[i + 1]], i)
                     for i in range(n)], np.int32)
    assert np.all(cols[diag] == np.arange(n)), "a diagonal entry is missing"
    assert np.all(vals.astype(np.float32).astype(np.float64) == vals), "not float values"
    return harness.HostSystem(row_ptr, cols.astype(np.int32), diag, vals,
                              np.zeros(n, np.float32))


def right_hand_side(s: harness.HostSystem, kind: str) -> np.ndarray:
    """b = A x for a known, bounded x, rounded to float, as the reference's
    solver tests build theirs (tests/linalg/matrices.hpp:71-86). The matrices
    are nearly singular (smallest eigenvalue ~1e-13, diagonals from 1e-14 to
    0.1), so white-noise forcing gives solutions of 1e12 and more.
    random: the tests' seeded random solution (mostly high-frequency content,
    which the smoother removes). smooth: that solution after 20 damped
    L1-Jacobi sweeps towards A x = 0, which leaves the smooth content the
    coarse levels must correct."""
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    x = harness.random_solution(s.n).astype(np.float64)
    if kind == "smooth":
        d = np.abs(A).sum(axis=1).A1
        for _ in range(20):
            x -= (2.0 / 3.0) * (A @ x) / d
        x /= np.max(np.abs(x))
    return (A @ x).astype(np.float32)


def make_case(name: str, source: str) -> dict:
    s = read_coo(SOURCE / source)
    opts = ref.options(ref.AMG_PCG, structure=1)
    data = {"row_ptr": s.row_ptr, "col": s.col, "diag": s.diag, "val": s.val}
    meta = {"name": name, "source": source, "n": s.n, "nnz": int(s.row_ptr[-1]), "results": []}
    for rhs in RHS:
        s.b = right_hand_side(s, rhs)
        data[f"b_{rhs}"] = s.b
        for tol in TOLERANCES:
            r = ref.solve(s, opts=opts, rel_tol=tol, abs_tol=1e-30, max_iter=2000)
            meta["results"].append(dict(rhs=rhs, rel_tol=tol, iterations=r.iterations,
                                        converged=r.converged,
                                        initial_residual=r.initial_residual,
                                        final_residual=r.final_residual, describe=r.describe))
            data[f"x_{rhs}_{tol:g}"] = r.x
    levels = ref.hierarchy(s, opts)
    meta["levels"] = [lv.n for lv in levels]
    meta["level_sha"] = [dict(row_ptr=digest(lv.row_ptr), col=digest(lv.col), val=digest(lv.val),
                              l1=digest(lv.l1),
                              aggregate=digest(lv.aggregate) if lv.aggregate is not None else None)
                         for lv in levels]
    data["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / f"{name}.npz", **data)
    return meta


def main():
    for name, source in CASES.items():
        m = make_case(name, source)
        for r in m["results"]:
            print(f"{name}: {r['rhs']} rhs, rel_tol {r['rel_tol']:g}: {r['iterations']} it, "
                  f"converged={r['converged']}, rel={r['final_residual'] / r['initial_residual']:.3e}")
        print(f"  levels {m['levels']}")


if __name__ == "__main__":
    main()
