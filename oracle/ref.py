"""Test infrastructure only: ctypes front end for ``oracle/_ref/libkutta_ref.so``,
the reference's own CPU solve path compiled from its sources by
``oracle/build_ref.sh`` (see ``oracle/ref_shim.cpp``).

Used by the tests, the golden-fixture generator and ``bench.py``'s reference /
CPU-baseline arm. The product never imports this module.
"""
from __future__ import annotations

import ctypes
import dataclasses
import pathlib

import numpy as np

LIB = pathlib.Path(__file__).resolve().parent / "_ref" / "libkutta_ref.so"

# SolverKind order of src/kutta/linalg/solver.hpp:32-38.
JACOBI, PCG_JACOBI, BICGSTAB_JACOBI, AMG_PCG, AMG_BICGSTAB = range(5)


class Options(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("cycle", ctypes.c_int),
                ("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarse_sweeps", ctypes.c_int), ("coarse_rows", ctypes.c_int),
                ("max_levels", ctypes.c_int), ("passes", ctypes.c_int),
                ("threshold", ctypes.c_double), ("nullspace", ctypes.c_int),
                ("structure", ctypes.c_int), ("use_make_solver", ctypes.c_int)]


class Control(ctypes.Structure):
    _fields_ = [("rel_tol", ctypes.c_double), ("abs_tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("interval", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("levels", ctypes.c_int), ("pad", ctypes.c_int),
                ("initial_residual", ctypes.c_double), ("final_residual", ctypes.c_double),
                ("setup_s", ctypes.c_double), ("refresh_s", ctypes.c_double),
                ("solve_s", ctypes.c_double)]


def available() -> bool:
    return LIB.exists()


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} missing: build it with oracle/build_ref.sh")
        lib = ctypes.CDLL(str(LIB))
        I = ctypes.POINTER(ctypes.c_int)
        F = ctypes.POINTER(ctypes.c_float)
        D = ctypes.POINTER(ctypes.c_double)
        lib.kref_solve.restype = ctypes.c_int
        lib.kref_solve.argtypes = [ctypes.c_int, ctypes.c_int, I, I, I, D, F, F,
                                   ctypes.POINTER(Options), ctypes.POINTER(Control),
                                   ctypes.POINTER(Stats), ctypes.c_char_p, ctypes.c_int]
        lib.kref_last_error.restype = ctypes.c_char_p
        lib.kref_hierarchy.restype = ctypes.c_void_p
        lib.kref_hierarchy.argtypes = [ctypes.c_int, ctypes.c_int, I, I, I, D,
                                       ctypes.POINTER(Options)]
        lib.kref_hierarchy_levels.restype = ctypes.c_int
        lib.kref_hierarchy_levels.argtypes = [ctypes.c_void_p]
        lib.kref_hierarchy_shape.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I, I]
        lib.kref_hierarchy_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I, F, F, I]
        lib.kref_hierarchy_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def options(kind=AMG_PCG, *, cycle=0, pre_sweeps=5, post_sweeps=5, coarse_sweeps=32,
            coarse_rows=24, max_levels=24, passes=3, threshold=0.25, nullspace=0,
            structure=0, use_make_solver=False) -> Options:
    return Options(kind, cycle, pre_sweeps, post_sweeps, coarse_sweeps, coarse_rows,
                   max_levels, passes, threshold, nullspace, structure, int(use_make_solver))


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


@dataclasses.dataclass
class RefResult:
    x: np.ndarray
    iterations: int
    converged: bool
    initial_residual: float
    final_residual: float
    setup_s: float
    refresh_s: float
    solve_s: float
    describe: str


def solve(system, b=None, x0=None, opts: Options | None = None, rel_tol=1e-6, abs_tol=1e-12,
          max_iter=2000, interval=8) -> RefResult:
    lib = _load()
    opts = opts or options()
    row_ptr = np.ascontiguousarray(system.row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(system.col, dtype=np.int32)
    diag = np.ascontiguousarray(system.diag, dtype=np.int32)
    val = np.ascontiguousarray(system.val, dtype=np.float64)
    b = np.ascontiguousarray(system.b if b is None else b, dtype=np.float32)
    x = np.zeros(system.n, np.float32) if x0 is None else np.array(x0, np.float32, copy=True)
    st = Stats()
    desc = ctypes.create_string_buffer(256)
    rc = lib.kref_solve(system.n, system.nnz, _ptr(row_ptr, ctypes.c_int), _ptr(col, ctypes.c_int),
                        _ptr(diag, ctypes.c_int), _ptr(val, ctypes.c_double),
                        _ptr(b, ctypes.c_float), _ptr(x, ctypes.c_float), ctypes.byref(opts),
                        ctypes.byref(Control(rel_tol, abs_tol, max_iter, interval)),
                        ctypes.byref(st), desc, 256)
    if rc != 0:
        raise RuntimeError(lib.kref_last_error().decode())
    return RefResult(x, st.iterations, bool(st.converged), st.initial_residual,
                     st.final_residual, st.setup_s, st.refresh_s, st.solve_s,
                     desc.value.decode())


@dataclasses.dataclass
class RefLevel:
    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    l1: np.ndarray
    aggregate: np.ndarray | None


def hierarchy(system, opts: Options | None = None) -> list[RefLevel]:
    """The AMG hierarchy the reference's V-cycle actually uses, after refresh."""
    lib = _load()
    opts = opts or options()
    row_ptr = np.ascontiguousarray(system.row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(system.col, dtype=np.int32)
    diag = np.ascontiguousarray(system.diag, dtype=np.int32)
    val = np.ascontiguousarray(system.val, dtype=np.float64)
    h = lib.kref_hierarchy(system.n, system.nnz, _ptr(row_ptr, ctypes.c_int),
                           _ptr(col, ctypes.c_int), _ptr(diag, ctypes.c_int),
                           _ptr(val, ctypes.c_double), ctypes.byref(opts))
    if not h:
        raise RuntimeError(lib.kref_last_error().decode())
    out = []
    try:
        for lv in range(lib.kref_hierarchy_levels(h)):
            n, nnz, has = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            lib.kref_hierarchy_shape(h, lv, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(has))
            rp = np.zeros(n.value + 1, np.int32)
            cl = np.zeros(nnz.value, np.int32)
            vl = np.zeros(nnz.value, np.float32)
            l1 = np.zeros(n.value, np.float32)
            ag = np.zeros(n.value, np.int32) if has.value else None
            lib.kref_hierarchy_copy(h, lv, _ptr(rp, ctypes.c_int), _ptr(cl, ctypes.c_int),
                                    _ptr(vl, ctypes.c_float), _ptr(l1, ctypes.c_float),
                                    _ptr(ag, ctypes.c_int) if ag is not None else None)
            out.append(RefLevel(n.value, rp, cl, vl, l1, ag))
    finally:
        lib.kref_hierarchy_free(h)
    return out
