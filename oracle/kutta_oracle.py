"""Test infrastructure: ctypes front end of the oracle's C restatement
(``oracle/kutta_oracle.c`` -> ``oracle/_lib/libkutta_oracle.so``).

``solve`` runs the reference's solve path on the CPU exactly as restated;
``hierarchy`` returns the AMG levels after refresh; ``cg64`` is the FP64 CG
oracle every reported solution states its error against.
"""
from __future__ import annotations

import ctypes
import dataclasses
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_lib" / "libkutta_oracle.so"

JACOBI, PCG_JACOBI, BICGSTAB_JACOBI, AMG_PCG, AMG_BICGSTAB = range(5)


class Options(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("cycle", ctypes.c_int),
                ("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarse_sweeps", ctypes.c_int), ("coarse_rows", ctypes.c_int),
                ("max_levels", ctypes.c_int), ("passes", ctypes.c_int),
                ("threshold", ctypes.c_double), ("nullspace", ctypes.c_int),
                ("m_matrix", ctypes.c_int), ("absorb", ctypes.c_int)]


class Control(ctypes.Structure):
    _fields_ = [("rel_tol", ctypes.c_double), ("abs_tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("interval", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("initial_residual", ctypes.c_double), ("final_residual", ctypes.c_double)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from oracle import build
            build.build_restatement()
        lib = ctypes.CDLL(str(LIB))
        P = ctypes.c_void_p
        I = ctypes.c_int
        lib.ko_create.restype = P
        lib.ko_create.argtypes = [I, I, P, P, P, P, ctypes.POINTER(Options), ctypes.c_char_p, I]
        lib.ko_refresh.restype = I
        lib.ko_refresh.argtypes = [P, P, ctypes.c_char_p, I]
        lib.ko_solve.restype = I
        lib.ko_solve.argtypes = [P, P, P, P, ctypes.POINTER(Control), ctypes.POINTER(Stats),
                                 ctypes.c_char_p, I]
        lib.ko_describe.argtypes = [P, ctypes.c_char_p, I]
        lib.ko_levels.argtypes = [P]
        lib.ko_level_shape.argtypes = [P, I, P, P]
        lib.ko_level_copy.argtypes = [P, I, P, P, P, P, P]
        lib.ko_destroy.argtypes = [P]
        for name, n in [("ko_spmv", 6), ("ko_residual", 7)]:
            getattr(lib, name).argtypes = [I] + [P] * (n - 1)
        lib.ko_smooth.argtypes = [I, P, P, P, P, P, P, P, P, I]
        lib.ko_coarse_solve.argtypes = [P, P, P, P, P, P, P, I, I]
        lib.ko_diagonal.argtypes = [I, P, P, P, P, P, I]
        lib.ko_restrict.argtypes = [I, P, P, P, P]
        lib.ko_prolong.argtypes = [I, P, P, P]
        lib.ko_galerkin.argtypes = [I, P, P, P, P]
        lib.ko_scalar.argtypes = [I, P, P, I]
        lib.ko_solver_step.argtypes = [I, P, P, P, P, P, P]
        lib.ko_cg64.restype = I
        lib.ko_cg64.argtypes = [I, P, P, P, P, P, ctypes.c_double, I, I]
        lib.ko_true_residual.restype = ctypes.c_double
        lib.ko_true_residual.argtypes = [I, P, P, P, P, P]
        _lib = lib
    return _lib


def lib():
    return _load()


def p(a):
    """Pointer to a contiguous numpy array (None when empty)."""
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


def _arrays(system):
    return (np.ascontiguousarray(system.row_ptr, np.int32), np.ascontiguousarray(system.col, np.int32),
            np.ascontiguousarray(system.diag, np.int32), np.ascontiguousarray(system.val, np.float64))


class OracleError(RuntimeError):
    pass


class OracleNonfinite(OracleError):
    pass


def options(kind=AMG_PCG, *, pre_sweeps=5, post_sweeps=5, coarse_sweeps=32, coarse_rows=24,
            max_levels=24, passes=3, threshold=0.25, nullspace=False, m_matrix=False,
            absorb=False) -> Options:
    return Options(kind, 0, pre_sweeps, post_sweeps, coarse_sweeps, coarse_rows, max_levels,
                   passes, threshold, int(nullspace), int(m_matrix), int(absorb))


class Solver:
    """make_solver / make_amg_solver + refresh + solve, restated on the CPU."""

    def __init__(self, system, opts: Options):
        L = _load()
        self._keep = _arrays(system)
        rp, cl, dg, vl = self._keep
        err = ctypes.create_string_buffer(512)
        h = L.ko_create(system.n, system.nnz, p(rp), p(cl), p(dg), p(vl), ctypes.byref(opts), err, 512)
        if not h:
            raise OracleError(err.value.decode())
        self._h = ctypes.c_void_p(h)
        self.n = system.n

    def refresh(self, val32: np.ndarray):
        err = ctypes.create_string_buffer(512)
        self._val = np.ascontiguousarray(val32, np.float32)
        if _load().ko_refresh(self._h, p(self._val), err, 512) != 0:
            raise OracleError(err.value.decode())

    def solve(self, val32, x, b, rel_tol=1e-2, abs_tol=1e-12, max_iter=200, interval=8):
        err = ctypes.create_string_buffer(512)
        self._val = np.ascontiguousarray(val32, np.float32)
        st = Stats()
        b = np.ascontiguousarray(b, np.float32)
        rc = _load().ko_solve(self._h, p(self._val), p(x), p(b),
                              ctypes.byref(Control(rel_tol, abs_tol, max_iter, interval)),
                              ctypes.byref(st), err, 512)
        if rc == -2:
            raise OracleNonfinite(err.value.decode())
        if rc != 0:
            raise OracleError(err.value.decode())
        return st

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(256)
        _load().ko_describe(self._h, buf, 256)
        return buf.value.decode()

    def levels(self):
        L = _load()
        out = []
        count = L.ko_levels(self._h)
        for lv in range(count):
            n, nnz = ctypes.c_int(), ctypes.c_int()
            L.ko_level_shape(self._h, lv, ctypes.byref(n), ctypes.byref(nnz))
            rp = np.zeros(n.value + 1, np.int32)
            cl = np.zeros(nnz.value, np.int32)
            vl = np.zeros(nnz.value, np.float32) if lv else None
            l1 = np.zeros(n.value, np.float32)
            ag = np.zeros(n.value, np.int32) if lv + 1 < count else None
            L.ko_level_copy(self._h, lv, p(rp), p(cl), p(vl), p(l1), p(ag))
            out.append(dict(n=n.value, row_ptr=rp, col=cl, val=vl, l1=l1, aggregate=ag))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ko_destroy(self._h)
            self._h = None


@dataclasses.dataclass
class Result:
    x: np.ndarray
    iterations: int
    converged: bool
    initial_residual: float
    final_residual: float
    describe: str


def solve(system, kind=AMG_PCG, *, m_matrix=False, nullspace=False, b=None, x0=None,
          rel_tol=1e-6, abs_tol=1e-12, max_iter=2000, interval=8, opts: Options | None = None,
          refresh=True) -> Result:
    opts = opts or options(kind, m_matrix=m_matrix, nullspace=nullspace)
    s = Solver(system, opts)
    val32 = system.val.astype(np.float32)
    if refresh:
        s.refresh(val32)
    x = np.zeros(system.n, np.float32) if x0 is None else np.array(x0, np.float32, copy=True)
    st = s.solve(val32, x, system.b if b is None else b, rel_tol, abs_tol, max_iter, interval)
    return Result(x, st.iterations, bool(st.converged), st.initial_residual, st.final_residual,
                  s.describe())


def cg64(system, b=None, rel_tol=1e-12, max_iter=100000, threads=0) -> tuple[np.ndarray, int]:
    """FP64 CG solution of A x = b (double values, double arithmetic)."""
    rp, cl, _, vl = _arrays(system)
    bb = np.ascontiguousarray(system.b if b is None else b, np.float64)
    x = np.zeros(system.n, np.float64)
    it = _load().ko_cg64(system.n, p(rp), p(cl), p(vl), p(bb), p(x), rel_tol, max_iter, threads)
    return x, it


def true_residual(system, x, b=None) -> float:
    """||b - A x||_2 in double for a float32 x."""
    rp, cl, _, vl = _arrays(system)
    bb = np.ascontiguousarray(system.b if b is None else b, np.float64)
    xx = np.ascontiguousarray(x, np.float32)
    return float(_load().ko_true_residual(system.n, p(rp), p(cl), p(vl), p(bb), p(xx)))
