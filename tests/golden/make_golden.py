"""Generates tests/golden/*.npz from the reference's own CPU path.

Runs the reference library built from its sources (oracle/_ref/libkutta_ref.so,
see oracle/build_ref.sh) on seeded systems and stores, per case: iteration
count, convergence flag, initial/final residuals, the solution x, and the AMG
hierarchy the reference's V-cycle actually used (aggregates, coarse CSR
patterns, coarse values, L1 inverse diagonals). Large cases store SHA-256
digests of the arrays instead of the arrays; "x" stores the solution but only
digests of the hierarchy. HIERARCHIES holds cases too large for a reference
solve in a fixture run (the 5.3M-row tet matrix: about 9 minutes of serial
reference solve): only the hierarchy the reference sets up and refreshes is
captured, as level sizes and array digests.

Needs the reference sources on this machine; the fixtures it writes are
committed and read by the tests without them.

    python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from kutta_b200 import harness  # noqa: E402
from oracle import ref  # noqa: E402


def _rhs_from_solution(s):
    """b = A x_exact with the reference tests' random_solution (matrices.hpp:71-79)."""
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    s.b = (A @ harness.random_solution(s.n).astype(np.float64)).astype(np.float32)
    return s


def _forced(s):
    s.b = harness.random_forcing(s.n)
    return s


# name -> (system factory, kind, m_matrix, rel_tol, max_iter, store arrays? (True, False or
# "x": the solution only)[, AmgOptions overrides])
CASES = {
    "poisson_aniso1000_amgpcg": (lambda: _rhs_from_solution(harness.poisson(12, 9, 5, 1000)), 3, 0, 1e-6, 2000, True),
    "poisson_random2d_amgpcg": (lambda: _rhs_from_solution(harness.poisson(8, 7, 1, 1, True)), 3, 0, 1e-6, 2000, True),
    "poisson_wind3_amgbicgstab": (lambda: _rhs_from_solution(harness.poisson(20, 18, 1, 1, False, False, 3)), 4, 0, 1e-6, 2000, True),
    "poisson_jacobi": (lambda: _rhs_from_solution(harness.poisson(16, 12, 8)), 0, 0, 1e-5, 500, True),
    "poisson_pcgjacobi": (lambda: _rhs_from_solution(harness.poisson(16, 12, 8)), 1, 0, 1e-5, 500, True),
    "poisson_wind5_bicgstabjacobi": (lambda: _rhs_from_solution(harness.poisson(16, 12, 8, 1, False, False, 5)), 2, 0, 1e-5, 500, True),
    "hex8_pressure_amgpcg": (lambda: harness.box_system(8, 8, 8, tet=False, seed=21), 3, 1, 1e-6, 2000, True),
    "tet8_pressure_amgpcg": (lambda: harness.box_system(8, 8, 8, tet=True, seed=22), 3, 1, 1e-6, 2000, True),
    "tet6_convection_amgbicgstab": (lambda: harness.box_system(6, 6, 6, tet=True, seed=23, convection=1e-3), 4, 0, 1e-6, 2000, True),
    # The 32^3 jittered-hex pressure configuration: aggregates bit-exact and x
    # against the reference. With the caller's defaults (V(5,5)), and with the
    # SST caller's V(2,2) (src/kutta/fv/steady_solver.cpp:575-578).
    "hex32_pressure_amgpcg": (lambda: harness.pressure_hex32(1), 3, 1, 1e-6, 2000, "x"),
    "hex32_pressure_amgpcg_v22": (lambda: harness.pressure_hex32(1), 3, 1, 1e-6, 2000, "x",
                                  dict(pre_sweeps=2, post_sweeps=2)),
    "tet8_pressure_amgpcg_v22": (lambda: harness.box_system(8, 8, 8, tet=True, seed=22), 3, 1, 1e-6,
                                 2000, True, dict(pre_sweeps=2, post_sweeps=2)),
    "poisson32_forced_amgpcg": (lambda: _forced(harness.poisson(32, 32, 32)), 3, 0, 1e-6, 300, False),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# name -> (system factory, kind, m_matrix, AmgOptions overrides): hierarchy only.
HIERARCHIES = {
    # The 5.3M-row scale configuration: 96^3 jittered hex split into 6 tets,
    # with the pressure caller's options (steady_solver.cpp:579-580).
    "tet96_pressure_hierarchy": (lambda: harness.pressure_tet96(1), 3, 1, {}),
}


def _level_digests(levels):
    return [dict(row_ptr=digest(lv.row_ptr), col=digest(lv.col), val=digest(lv.val),
                 l1=digest(lv.l1),
                 aggregate=digest(lv.aggregate) if lv.aggregate is not None else None)
            for lv in levels]


def make_hierarchy_case(name):
    factory, kind, m_matrix, overrides = HIERARCHIES[name]
    s = factory()
    levels = ref.hierarchy(s, ref.options(kind, structure=m_matrix, **overrides))
    meta = dict(name=name, kind=kind, m_matrix=m_matrix, options=overrides, n=s.n, nnz=s.nnz,
                matrix_sha=digest(s.val) + digest(s.col), levels=[lv.n for lv in levels],
                level_nnz=[int(lv.row_ptr[-1]) for lv in levels],
                level_sha=_level_digests(levels))
    np.savez_compressed(HERE / f"{name}.npz",
                        meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8))
    return meta


def make_case(name):
    if name in HIERARCHIES:
        return make_hierarchy_case(name)
    factory, kind, m_matrix, rel_tol, max_iter, arrays, *rest = CASES[name]
    overrides = rest[0] if rest else {}
    s = factory()
    opts = ref.options(kind, structure=m_matrix, **overrides)
    r = ref.solve(s, opts=opts, rel_tol=rel_tol, abs_tol=1e-12, max_iter=max_iter)
    meta = dict(name=name, kind=kind, m_matrix=m_matrix, rel_tol=rel_tol, abs_tol=1e-12,
                max_iter=max_iter, iterations=r.iterations, converged=r.converged,
                initial_residual=r.initial_residual, final_residual=r.final_residual,
                describe=r.describe, n=s.n, nnz=s.nnz, matrix_sha=digest(s.val) + digest(s.col),
                rhs_sha=digest(s.b), x_sha=digest(r.x))
    if overrides:
        meta["options"] = overrides
    data = {}
    if kind >= 3:
        levels = ref.hierarchy(s, opts)
        meta["levels"] = [lv.n for lv in levels]
        meta["level_sha"] = _level_digests(levels)
        if arrays is True:
            for i, lv in enumerate(levels):
                data[f"l{i}_row_ptr"] = lv.row_ptr
                data[f"l{i}_col"] = lv.col
                data[f"l{i}_val"] = lv.val
                data[f"l{i}_l1"] = lv.l1
                if lv.aggregate is not None:
                    data[f"l{i}_aggregate"] = lv.aggregate
    if arrays:
        data["x"] = r.x
    data["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / f"{name}.npz", **data)
    return meta


def main(names=None):
    for name in names or [*CASES, *HIERARCHIES]:
        m = make_case(name)
        if name in HIERARCHIES:
            print(f"{name}: levels {m['levels']}")
            continue
        print(f"{name}: {m['iterations']} it, converged={m['converged']}, "
              f"rel={m['final_residual'] / max(m['initial_residual'], 1e-300):.6e}")


if __name__ == "__main__":
    main(sys.argv[1:])
