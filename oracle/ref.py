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


# ---- the reference's Coupled block solve (oracle/ref_coupled.cpp) ---------------

class CoupledOptions(ctypes.Structure):
    _fields_ = [("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarsest_sweeps", ctypes.c_int), ("coarsest_rows", ctypes.c_int),
                ("aggregation_passes", ctypes.c_int), ("recompute", ctypes.c_int),
                ("smoother_damping", ctypes.c_double), ("courant", ctypes.c_double)]


def coupled_options(*, pre_sweeps=1, post_sweeps=2, coarsest_sweeps=8, coarsest_rows=48,
                    aggregation_passes=3, recompute=False, smoother_damping=0.7,
                    courant=200.0) -> CoupledOptions:
    """CoupledOptions defaults of src/kutta/fv/coupled_solver.hpp:26-38."""
    return CoupledOptions(pre_sweeps, post_sweeps, coarsest_sweeps, coarsest_rows,
                          aggregation_passes, int(recompute), smoother_damping, courant)


_DTYPES = {b"i": np.int32, b"f": np.float32, b"d": np.float64}


def _coupled_lib():
    lib = _load()
    if not getattr(lib, "_coupled_typed", False):
        P = ctypes.c_void_p
        F = ctypes.POINTER(ctypes.c_float)
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        lib.kref_coupled_last_error.restype = ctypes.c_char_p
        lib.kref_coupled_mesh.restype = P
        lib.kref_coupled_mesh.argtypes = [ctypes.c_int] * 4 + [D, D, I]
        lib.kref_coupled_solve.restype = ctypes.c_int
        lib.kref_coupled_solve.argtypes = (
            [P, ctypes.POINTER(CoupledOptions)] + [F] * 14 +
            [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
             ctypes.c_int, ctypes.c_int, I, F, F, ctypes.c_double, ctypes.c_double,
             ctypes.c_float, ctypes.c_float, I, I, D, ctypes.c_char_p, ctypes.c_int])
        lib.kref_coupled_array.restype = ctypes.c_longlong
        lib.kref_coupled_array.argtypes = [P, ctypes.c_char_p, P, ctypes.c_char_p]
        lib.kref_coupled_names.restype = ctypes.c_int
        lib.kref_coupled_names.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
        lib.kref_coupled_free.argtypes = [P]
        lib._coupled_typed = True
    return lib


class CoupledCase:
    """A box mesh built by the reference (make_box_hex / make_box_tet) with its
    geometry, device mesh, stencil and pressure least-squares fit; `arrays`
    holds every array a Coupled solver reads, by name."""

    def __init__(self, tet: bool, nx: int, ny: int, nz: int, lo=(0, 0, 0), hi=(1, 1, 1),
                 patch_kinds=(1, 2, 0, 0, 3, 3)):
        self._lib = _coupled_lib()
        lo = np.array(lo, np.float64)
        hi = np.array(hi, np.float64)
        kinds = np.array(patch_kinds, np.int32)
        self._h = self._lib.kref_coupled_mesh(int(tet), nx, ny, nz, _ptr(lo, ctypes.c_double),
                                              _ptr(hi, ctypes.c_double), _ptr(kinds, ctypes.c_int))
        if not self._h:
            raise RuntimeError(self._lib.kref_coupled_last_error().decode())
        self.arrays = self._read_all()

    def _read_all(self) -> dict:
        size = self._lib.kref_coupled_names(self._h, None, 0)
        buf = ctypes.create_string_buffer(size)
        self._lib.kref_coupled_names(self._h, buf, size)
        out = {}
        for name in buf.value.decode().split():
            t = ctypes.create_string_buffer(1)
            nbytes = self._lib.kref_coupled_array(self._h, name.encode(), None, t)
            a = np.zeros(nbytes // np.dtype(_DTYPES[t.raw]).itemsize, _DTYPES[t.raw])
            self._lib.kref_coupled_array(self._h, name.encode(), a.ctypes.data, t)
            out[name] = a
        return out

    def solve(self, fields: dict, opts: CoupledOptions | None = None, *, rel_tol=0.1,
              abs_tol=1e-12, max_iter=20, capture=True, low_order=None, pairs=None) -> dict:
        """One CoupledSolver construction + solve + update on this mesh. `fields`
        holds momentum_u/v/w (over the stencil pattern), physical_u/v/w,
        ru/rv/rw, mass, viscosity, physical_diagonal, face_weights,
        net_outflow (or None), density, velocity_scale and reference.
        low_order: n int flags or None. pairs: (hi, lo, alpha_u, alpha_p,
        velocity_slack, pressure_slack) with hi, lo float32 planes of 4n, or
        None. Returns the captured arrays plus iterations, converged,
        residuals, seconds and describe."""
        lib = self._lib
        opts = opts or coupled_options()
        f32 = {k: np.ascontiguousarray(fields[k], np.float32) for k in (
            "momentum_u", "momentum_v", "momentum_w", "physical_u", "physical_v", "physical_w",
            "ru", "rv", "rw", "mass", "viscosity", "physical_diagonal", "face_weights")}
        net = fields.get("net_outflow")
        net = None if net is None else np.ascontiguousarray(net, np.float32)
        it, conv = ctypes.c_int(), ctypes.c_int()
        res = np.zeros(4, np.float64)
        desc = ctypes.create_string_buffer(512)
        F = ctypes.c_float
        low = None if low_order is None else np.ascontiguousarray(low_order, np.int32)
        if pairs is not None:
            hi, lo, au, ap, vs, ps = pairs
            hi = np.ascontiguousarray(hi, np.float32)
            lo = np.ascontiguousarray(lo, np.float32)
        else:
            hi = lo = None
            au = ap = vs = ps = 0.0
        rc = lib.kref_coupled_solve(
            self._h, ctypes.byref(opts), *(_ptr(f32[k], F) for k in (
                "momentum_u", "momentum_v", "momentum_w", "physical_u", "physical_v",
                "physical_w", "ru", "rv", "rw", "mass", "viscosity", "physical_diagonal",
                "face_weights")),
            _ptr(net, F) if net is not None else None, float(fields["density"]),
            float(fields["velocity_scale"]), int(fields["reference"]), rel_tol, abs_tol,
            max_iter, int(capture), _ptr(low, ctypes.c_int) if low is not None else None,
            _ptr(hi, F) if hi is not None else None, _ptr(lo, F) if lo is not None else None,
            float(au), float(ap), float(vs), float(ps), ctypes.byref(it), ctypes.byref(conv),
            _ptr(res, ctypes.c_double), desc, 512)
        if rc != 0:
            raise RuntimeError(lib.kref_coupled_last_error().decode())
        out = self._read_all() if capture else {}
        out.update(iterations=it.value, converged=bool(conv.value), initial_residual=res[0],
                   final_residual=res[1], setup_s=res[2], solve_s=res[3],
                   describe=desc.value.decode())
        return out

    def close(self):
        if self._h:
            self._lib.kref_coupled_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
