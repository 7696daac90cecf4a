"""Python mirror of the reference's linear-solver boundary over the C ABI.

Same names, argument meaning and error behaviour as ``src/kutta/linalg``
(solver.hpp, amg.hpp, csr.hpp): ``make_solver`` / ``make_amg_solver`` build a
solver from a host CSR (setup on the host, hierarchy uploaded to the GPU);
``LinearSolver.refresh`` recomputes value-dependent data on the device;
``LinearSolver.solve`` runs the Krylov iteration on the device and returns
``SolveStats``. Usage errors raise :class:`KuttaError` (kutta::Error),
nonfinite input vectors :class:`NonfiniteError` (kutta::NonfiniteError).

Device vectors are CUDA ``torch.Tensor`` s (float32 values, int32 indices); the
work is enqueued on torch's current stream. Every compute call goes through
``libkutta_b200.so``; there is no other implementation behind these names.
"""
from __future__ import annotations

import ctypes
import dataclasses
import enum
import pathlib

import numpy as np

_LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libkutta_b200.so"


class KuttaError(RuntimeError):
    """kutta::Error: invalid CSR, options, controls or matrix values."""


class NonfiniteError(KuttaError):
    """kutta::NonfiniteError: a nonfinite input vector."""


class DeviceError(KuttaError):
    """A CUDA runtime failure (or out of device memory)."""


class DeviceTimeout(DeviceError):
    """A bounded host wait on the device ran out."""


class SolverKind(enum.IntEnum):  # solver.hpp:32-38
    Jacobi = 0
    PcgJacobi = 1
    BicgstabJacobi = 2
    AmgPcg = 3
    AmgBicgstab = 4


class NullSpace(enum.IntEnum):  # solver.hpp:40
    None_ = 0
    Constant = 1


class OperatorStructure(enum.IntEnum):  # solver.hpp:41
    General = 0
    SymmetricMMatrix = 1


class AmgCycle(enum.IntEnum):  # amg.hpp:9
    V = 0
    K = 1


@dataclasses.dataclass
class SolveControl:  # solver.hpp:18-23
    rel_tol: float = 1e-2
    abs_tol: float = 1e-12
    max_iter: int = 200
    residual_check_interval: int = 8


@dataclasses.dataclass
class SolveStats:  # solver.hpp:25-30
    iterations: int = 0
    initial_residual: float = 0.0
    final_residual: float = 0.0
    converged: bool = False


class KrylovWorkspace:  # solver.hpp:47-64
    def __init__(self, rows: int):
        lib = _load()
        handle = ctypes.c_void_p()
        _check(lib.b2_workspace_create(int(rows), ctypes.byref(handle)))
        self._handle = handle
        self._rows = int(rows)

    def rows(self) -> int:
        return self._rows

    def __del__(self):
        if getattr(self, "_handle", None) and _lib is not None:
            _lib.b2_workspace_destroy(self._handle)
            self._handle = None


class Setup(enum.IntEnum):
    """b2_setup: where the AMG hierarchy is built (the same results either way)."""
    Host = 0
    Device = 1


@dataclasses.dataclass
class SolverOptions:  # solver.hpp:66-72
    nullspace: NullSpace = NullSpace.None_
    structure: OperatorStructure = OperatorStructure.General
    workspace: KrylovWorkspace | None = None
    setup: Setup = Setup.Device


@dataclasses.dataclass
class AmgOptions:  # amg.hpp:8-20
    cycle: AmgCycle = AmgCycle.V
    pre_sweeps: int = 5
    post_sweeps: int = 5
    coarse_sweeps: int = 32
    coarse_rows: int = 24
    max_levels: int = 24
    aggregation_passes: int = 3
    strength_threshold: float = 0.25
    nullspace: NullSpace = NullSpace.None_
    structure: OperatorStructure = OperatorStructure.General
    workspace: KrylovWorkspace | None = None
    setup: Setup = Setup.Device


class _Options(ctypes.Structure):
    _fields_ = [("cycle", ctypes.c_int), ("pre_sweeps", ctypes.c_int),
                ("post_sweeps", ctypes.c_int), ("coarse_sweeps", ctypes.c_int),
                ("coarse_rows", ctypes.c_int), ("max_levels", ctypes.c_int),
                ("aggregation_passes", ctypes.c_int), ("strength_threshold", ctypes.c_double),
                ("nullspace", ctypes.c_int), ("structure", ctypes.c_int),
                ("workspace", ctypes.c_void_p), ("setup", ctypes.c_int)]


class _Control(ctypes.Structure):
    _fields_ = [("rel_tol", ctypes.c_double), ("abs_tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("residual_check_interval", ctypes.c_int)]


class _Profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_longlong), ("fine_sweeps", ctypes.c_longlong),
                ("fine_sweep_ms", ctypes.c_double), ("fine_sweep_bytes", ctypes.c_double),
                ("algorithmic_bytes", ctypes.c_double), ("solves", ctypes.c_longlong)]


class _Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("initial_residual", ctypes.c_double), ("final_residual", ctypes.c_double)]


# Every symbol include/kutta_b200.h declares, with its ctypes signature.
_I = ctypes.c_int
_P = ctypes.c_void_p
_SIGNATURES = {
    "b2_options_default": (None, [_P]),
    "b2_control_default": (None, [_P]),
    "b2_last_error": (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
    "b2_workspace_create": (_I, [_I, _P]),
    "b2_workspace_destroy": (None, [_P]),
    "b2_solver_create": (_I, [_I, _I, _I, _P, _P, _P, _P, _P, _I, _P]),
    "b2_solver_refresh": (_I, [_P, _P, _P]),
    "b2_solver_solve": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "b2_solver_describe": (ctypes.c_size_t, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "b2_solver_destroy": (None, [_P]),
    "b2_csr_spmv": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "b2_csr_residual": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "b2_solver_profile": (_I, [_P, _I]),
    "b2_solver_profile_read": (_I, [_P, _P]),
    "b2_kernel_launches": (ctypes.c_longlong, []),
    "b2_amg_smooth": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "b2_solver_levels": (_I, [_P]),
    "b2_solver_level_shape": (_I, [_P, _I, _P, _P]),
    "b2_solver_level_copy": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "b2_solver_level_transfer": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "b2_fv_pressure_assemble": (_I, [_I] + [_P] * 11 + [_I, _P]),
    "b2_fv_correct_flux": (_I, [_I, _P, _P, _P, _P, _P, _I, _P]),
    "b2_fv_correct_velocity": (_I, [_I] + [_P] * 11 + [ctypes.c_float, _P]),
    "b2_solver_assemble_refresh": (_I, [_P] + [_P] * 9 + [_I, _P]),
    "b2_mixed_assemble_refresh": (_I, [_P] + [_P] * 9 + [_I, _P]),
    "b2_hierarchy_build": (_I, [_I, _I, _P, _P, _P, _P, _P, _I, _P]),
    "b2_hierarchy_levels": (_I, [_P]),
    "b2_hierarchy_level_shape": (_I, [_P, _I, _P, _P]),
    "b2_hierarchy_level_copy": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "b2_hierarchy_free": (None, [_P]),
    "b2_mixed_options_default": (None, [_P]),
    "b2_mixed_create": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "b2_mixed_refresh": (_I, [_P, _P, _P]),
    "b2_mixed_solve": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "b2_mixed_solve_f32": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "b2_mixed_describe": (ctypes.c_size_t, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "b2_mixed_destroy": (None, [_P]),
    "b2_mixed_hierarchy_build": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "b2_dense_inverse": (_I, [_I, _P, _P, _P, _P, _P, _P]),
    "b2_dense_inverse_noalloc": (_I, [_I, _P, _P, _P, _P, _P, _P]),
    "b2_gnn_create": (_I, [ctypes.c_uint64, _P]),
    "b2_gnn_destroy": (None, [_P]),
    "b2_gnn_parameter_count": (_I, []),
    "b2_gnn_bind": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "b2_gnn_apply": (_I, [_P, _P, _P, ctypes.c_float, _P]),
    "b2_gnn_train_step": (_I, [_P, _P, _P, ctypes.c_float, _P, _P]),
    "b2_gnn_set_wait_limit": (_I, [_P, ctypes.c_longlong]),
    "b2_gnn_gradient": (_I, [_P, _P, _P, _I, _P, ctypes.c_size_t, _P, _P]),
    "b2_gnn_set_geometry": (_I, [_P, _P]),
    "b2_gnn_get_weights": (_I, [_P, _P, ctypes.c_size_t]),
    "b2_gnn_set_weights": (_I, [_P, _P, ctypes.c_size_t]),
    "b2_mixed_set_learned": (_I, [_P, _P, _I]),
    "b2_mixed_precondition": (_I, [_P, _P, _P, _P, _P]),
    "b2_mixed_profile": (_I, [_P, _I]),
    "b2_mixed_profile_read": (_I, [_P, _P]),
    "b2_coupled_options_default": (None, [_P]),
    "b2_coupled_create": (_I, [_P, _I, _P, _P, _P]),
    "b2_coupled_capture_diagonal": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "b2_coupled_solve": (_I, [_P, _P, _P, _P, _P]),
    "b2_coupled_update": (_I, [_P, _P, _P, _P, _P, ctypes.c_double, ctypes.c_double, _P]),
    "b2_coupled_paired_update": (_I, [_P] + [_P] * 8 + [ctypes.c_double, ctypes.c_double,
                                                         ctypes.c_float, ctypes.c_float, _P]),
    "b2_coupled_bytes": (ctypes.c_size_t, [_P]),
    "b2_coupled_describe": (ctypes.c_size_t, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "b2_coupled_destroy": (None, [_P]),
    "b2_coupled_copy": (ctypes.c_longlong, [_P, _I, _P, _P]),
    "b2_coupled_levels": (_I, [_P]),
    "b2_coupled_level_shape": (_I, [_P, _I, _P, _P]),
    "b2_coupled_level_copy": (_I, [_P, _I] + [_P] * 10),
    "b2_coupled_apply": (_I, [_P, _I, _P, _P, _P, _P]),
    "b2_coupled_level_apply": (_I, [_P, _I, _I, _P, _P, _P, _P]),
    "b2_coupled_setup_build": (_I, [_P, _P, _P]),
    "b2_coupled_setup_levels": (_I, [_P]),
    "b2_coupled_setup_level_shape": (_I, [_P, _I, _P, _P]),
    "b2_coupled_setup_level_copy": (_I, [_P, _I] + [_P] * 6),
    "b2_coupled_setup_cell": (_I, [_P, _P]),
    "b2_coupled_setup_width": (_I, [_P]),
    "b2_coupled_setup_free": (None, [_P]),
}

_lib = None


def library_path() -> pathlib.Path:
    return _LIB_PATH


def _load():
    """Loads libkutta_b200.so; fails loudly when the native build is missing."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(
                f"kutta_b200 native library missing ({_LIB_PATH}); build it with "
                "`python -m kutta_b200.build` (there is no fallback implementation)")
        lib = ctypes.CDLL(str(_LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def last_error() -> str:
    lib = _load()
    buf = ctypes.create_string_buffer(4096)
    lib.b2_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def _check(code: int):
    if code == 0:
        return
    msg = last_error()
    if code == 2:
        raise NonfiniteError(msg)
    if code == 4:
        raise DeviceTimeout(msg)
    if code in (3, 5):
        raise DeviceError(msg)
    raise KuttaError(msg)


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


def _tptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclasses.dataclass
class CsrMatrixHost:
    """csr.hpp:16-28 (pattern + double values)."""
    n_rows: int
    row_ptr: np.ndarray
    col: np.ndarray
    diag: np.ndarray
    val: np.ndarray

    @classmethod
    def of(cls, system) -> "CsrMatrixHost":
        return cls(int(system.row_ptr.shape[0] - 1), system.row_ptr, system.col, system.diag,
                   system.val)

    def arrays(self):
        return (np.ascontiguousarray(self.row_ptr, np.int32), np.ascontiguousarray(self.col, np.int32),
                np.ascontiguousarray(self.diag, np.int32), np.ascontiguousarray(self.val, np.float64))

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])


def _host(a) -> CsrMatrixHost:
    return a if isinstance(a, CsrMatrixHost) else CsrMatrixHost.of(a)


@dataclasses.dataclass
class CsrMatrix:
    """Device CSR (csr.hpp:31-38); ``val`` is the only part expected to change."""
    n_rows: int
    nnz: int
    row_ptr: "torch.Tensor"
    col: "torch.Tensor"
    diag: "torch.Tensor"
    val: "torch.Tensor"


def upload(a, device="cuda") -> CsrMatrix:
    """upload(dev, CsrMatrixHost), csr.cpp:61-73: values stored as float32."""
    import torch
    h = _host(a)
    row_ptr, col, diag, val = h.arrays()
    if not np.all(np.isfinite(val)) or np.any(np.abs(val) > np.finfo(np.float32).max):
        raise KuttaError("CSR: nonfinite or out-of-range value")
    return CsrMatrix(h.n_rows, h.nnz, torch.from_numpy(row_ptr).to(device),
                     torch.from_numpy(col).to(device), torch.from_numpy(diag).to(device),
                     torch.from_numpy(val.astype(np.float32)).to(device))


def _options_struct(o, use_amg: bool) -> _Options:
    s = _Options()
    _load().b2_options_default(ctypes.byref(s))
    if isinstance(o, AmgOptions):
        s.cycle, s.pre_sweeps, s.post_sweeps = int(o.cycle), o.pre_sweeps, o.post_sweeps
        s.coarse_sweeps, s.coarse_rows, s.max_levels = o.coarse_sweeps, o.coarse_rows, o.max_levels
        s.aggregation_passes, s.strength_threshold = o.aggregation_passes, o.strength_threshold
    if o is not None:
        s.nullspace, s.structure = int(o.nullspace), int(o.structure)
        s.workspace = o.workspace._handle if o.workspace is not None else None
        s.setup = int(o.setup)
    return s


class LinearSolver:
    """solver.hpp:74-81."""

    def __init__(self, kind: SolverKind, a, options, use_amg: bool):
        lib = _load()
        h = _host(a)
        row_ptr, col, diag, val = h.arrays()
        opts = _options_struct(options, use_amg)
        handle = ctypes.c_void_p()
        _check(lib.b2_solver_create(int(kind), h.n_rows, h.nnz, _ptr(row_ptr), _ptr(col),
                                    _ptr(diag), _ptr(val), ctypes.byref(opts), int(use_amg),
                                    ctypes.byref(handle)))
        self._handle = handle
        self._workspace = getattr(options, "workspace", None)  # keep alive
        self.kind = SolverKind(kind)
        self.n_rows = h.n_rows
        self.nnz = h.nnz

    def _check_matrix(self, a: CsrMatrix):
        if a.n_rows != self.n_rows or a.nnz != self.nnz or a.val.numel() != self.nnz:
            raise KuttaError("solver: device or matrix mismatch")

    def refresh(self, a: CsrMatrix) -> None:
        self._check_matrix(a)
        _check(_load().b2_solver_refresh(self._handle, _tptr(a.val), _stream()))

    def assemble_refresh(self, a: CsrMatrix, fv: "FvPressure", rhs) -> None:
        """b2_solver_assemble_refresh: assembles the pressure matrix into a.val
        and rhs from the face data, refreshing the solver in the same pass."""
        self._check_matrix(a)
        _check(_load().b2_solver_assemble_refresh(self._handle, *fv.pointers(), _tptr(a.val),
                                                  _tptr(rhs), fv.reference, _stream()))

    def solve(self, a: CsrMatrix, x, b, control: SolveControl | None = None) -> SolveStats:
        self._check_matrix(a)
        if x.numel() != self.n_rows or b.numel() != self.n_rows or (
                x.numel() and x.data_ptr() == b.data_ptr()):
            raise KuttaError("solve: vector size or alias mismatch")
        control = control or SolveControl()
        c = _Control(control.rel_tol, control.abs_tol, control.max_iter,
                     control.residual_check_interval)
        st = _Stats()
        _check(_load().b2_solver_solve(self._handle, _tptr(a.val), _tptr(x), _tptr(b),
                                       ctypes.byref(c), ctypes.byref(st), _stream()))
        return SolveStats(st.iterations, st.initial_residual, st.final_residual, bool(st.converged))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        _load().b2_solver_describe(self._handle, buf, 512)
        return buf.value.decode()

    def profile(self, enable: bool) -> None:
        """Turns solve-time measurement on (resetting it) or off."""
        _check(_load().b2_solver_profile(self._handle, int(enable)))

    def profile_read(self) -> dict:
        p = _Profile()
        _check(_load().b2_solver_profile_read(self._handle, ctypes.byref(p)))
        return {f: getattr(p, f) for f, _ in _Profile._fields_}

    def levels(self):
        """The device hierarchy read back: [(n, row_ptr, col, val, inverse_l1, aggregate)]."""
        lib = _load()
        out = []
        for lv in range(lib.b2_solver_levels(self._handle)):
            n, nnz = ctypes.c_int(), ctypes.c_int()
            _check(lib.b2_solver_level_shape(self._handle, lv, ctypes.byref(n), ctypes.byref(nnz)))
            rp = np.zeros(n.value + 1, np.int32)
            cl = np.zeros(nnz.value, np.int32)
            vl = np.zeros(nnz.value, np.float32)
            l1 = np.zeros(n.value, np.float32)
            ag = np.full(n.value, -2, np.int32)
            _check(lib.b2_solver_level_copy(self._handle, lv, _ptr(rp), _ptr(cl), _ptr(vl),
                                            _ptr(l1), _ptr(ag), _stream()))
            out.append((n.value, rp, cl, vl, l1, ag))
        return out

    def level_transfer(self, level: int) -> dict:
        """Level `level`'s diagonal positions and its transfer to level + 1
        (member_offsets, members, entry_offsets, entries; empty on the coarsest)."""
        lib = _load()
        count = lib.b2_solver_levels(self._handle)
        n, nnz = ctypes.c_int(), ctypes.c_int()
        _check(lib.b2_solver_level_shape(self._handle, level, ctypes.byref(n), ctypes.byref(nnz)))
        nc, nnz_c = ctypes.c_int(0), ctypes.c_int(0)
        if level + 1 < count:
            _check(lib.b2_solver_level_shape(self._handle, level + 1, ctypes.byref(nc),
                                             ctypes.byref(nnz_c)))
        diag = np.zeros(n.value, np.int32)
        offsets = np.zeros(nc.value + 1, np.int32)
        members = np.full(n.value, -1, np.int32)
        entry_offsets = np.zeros(nnz_c.value + 1, np.int32)
        entries = np.full(nnz.value, -1, np.int32)
        _check(lib.b2_solver_level_transfer(self._handle, level, _ptr(diag), _ptr(offsets),
                                            _ptr(members), _ptr(entry_offsets), _ptr(entries),
                                            _stream()))
        if level + 1 >= count:
            return {"diag": diag}
        return {"diag": diag, "member_offsets": offsets, "members": members[:offsets[-1]],
                "entry_offsets": entry_offsets, "entries": entries[:entry_offsets[-1]]}

    def __del__(self):
        if getattr(self, "_handle", None) and _lib is not None:
            _lib.b2_solver_destroy(self._handle)
            self._handle = None


def make_solver(kind: SolverKind, a, options: SolverOptions | None = None) -> LinearSolver:
    """solver.hpp:85-88 / amg.cpp:384-406."""
    return LinearSolver(kind, a, options or SolverOptions(), use_amg=False)


def make_amg_solver(kind: SolverKind, a, options: AmgOptions) -> LinearSolver:
    """amg.hpp:26-27 / amg.cpp:345-382."""
    return LinearSolver(kind, a, options, use_amg=True)


def spmv(a: CsrMatrix, x, y) -> None:
    """csr.hpp:40-41: y = A x (Kahan-compensated float)."""
    if x.numel() != a.n_rows or y.numel() != a.n_rows:
        raise KuttaError("CSR: vector size mismatch")
    if a.n_rows and x.data_ptr() == y.data_ptr():
        raise KuttaError("CSR: input/output aliasing is unsupported")
    _check(_load().b2_csr_spmv(a.n_rows, a.nnz, _tptr(a.row_ptr), _tptr(a.col), _tptr(a.val),
                               _tptr(x), _tptr(y), _stream()))


def kernel_launches() -> int:
    """Kernels this library has launched in this process."""
    return int(_load().b2_kernel_launches())


def amg_smooth(a: CsrMatrix, x, b, inverse, out, zero_start=False) -> None:
    """One damped L1-Jacobi sweep (amg_smooth / amg_smooth_zero)."""
    _check(_load().b2_amg_smooth(a.n_rows, _tptr(a.row_ptr), _tptr(a.col), _tptr(a.val), _tptr(x),
                                 _tptr(b), _tptr(inverse), _tptr(out), int(zero_start), _stream()))


def residual(a: CsrMatrix, x, b, r) -> None:
    """csr.hpp:43-46: r = b - A x (Neumaier + Dekker compensated float)."""
    if x.numel() != a.n_rows or r.numel() != a.n_rows or b.numel() != a.n_rows:
        raise KuttaError("CSR: vector size mismatch")
    if a.n_rows and (x.data_ptr() == r.data_ptr() or b.data_ptr() == r.data_ptr()):
        raise KuttaError("CSR: residual RHS size or alias mismatch")
    _check(_load().b2_csr_residual(a.n_rows, a.nnz, _tptr(a.row_ptr), _tptr(a.col), _tptr(a.val),
                                   _tptr(x), _tptr(b), _tptr(r), _stream()))


@dataclasses.dataclass
class MixedOptions:
    """b2_mixed_options: the mixed-precision solve (no reference counterpart)."""
    amg: AmgOptions = dataclasses.field(default_factory=lambda: AmgOptions(
        cycle=AmgCycle.K, pre_sweeps=1, post_sweeps=1,
        structure=OperatorStructure.SymmetricMMatrix))
    absorb_singletons: bool = True
    dense_rows: int = 112
    coarse_bf16: bool = True
    inner_rel_tol: float = 1e-3
    inner_max_iter: int = 300
    max_refinements: int = 30
    fused_coarse: bool = False
    k_cycle_levels: int = 1
    cuda_graphs: bool = True
    packed_rows: bool = True


@dataclasses.dataclass
class MixedStats:
    refinements: int = 0
    iterations: int = 0
    converged: bool = False
    initial_residual: float = 0.0
    final_residual: float = 0.0
    learned_fallback: bool = False


class _MixedOptions(ctypes.Structure):
    _fields_ = [("amg", _Options), ("absorb_singletons", ctypes.c_int),
                ("dense_rows", ctypes.c_int), ("coarse_bf16", ctypes.c_int),
                ("inner_rel_tol", ctypes.c_double), ("inner_max_iter", ctypes.c_int),
                ("max_refinements", ctypes.c_int), ("fused_coarse", ctypes.c_int),
                ("k_cycle_levels", ctypes.c_int), ("cuda_graphs", ctypes.c_int),
                ("packed_rows", ctypes.c_int)]


class _MixedStats(ctypes.Structure):
    _fields_ = [("refinements", ctypes.c_int), ("iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("initial_residual", ctypes.c_double),
                ("final_residual", ctypes.c_double), ("learned_fallback", ctypes.c_int)]


def _mixed_struct(o: MixedOptions) -> _MixedOptions:
    s = _MixedOptions()
    _load().b2_mixed_options_default(ctypes.byref(s))
    s.amg = _options_struct(o.amg, True)
    s.absorb_singletons, s.dense_rows, s.coarse_bf16 = int(o.absorb_singletons), o.dense_rows, int(o.coarse_bf16)
    s.inner_rel_tol, s.inner_max_iter, s.max_refinements = o.inner_rel_tol, o.inner_max_iter, o.max_refinements
    s.fused_coarse = int(o.fused_coarse)
    s.k_cycle_levels = int(o.k_cycle_levels)
    s.cuda_graphs = int(o.cuda_graphs)
    s.packed_rows = int(o.packed_rows)
    return s


# b2_mixed_set_learned mode bits.
LEARNED_CYCLE = 1
LEARNED_WARM_START = 2


class MixedSolver:
    """FP64 iterative refinement around the FP32 AMG-PCG with BF16 coarse
    levels and a dense FP64 coarsest solve; the solution is FP64."""

    def __init__(self, a, options: MixedOptions | None = None):
        lib = _load()
        h = _host(a)
        row_ptr, col, diag, val = h.arrays()
        opts = _mixed_struct(options or MixedOptions())
        handle = ctypes.c_void_p()
        _check(lib.b2_mixed_create(h.n_rows, h.nnz, _ptr(row_ptr), _ptr(col), _ptr(diag), _ptr(val),
                                   ctypes.byref(opts), ctypes.byref(handle)))
        self._handle = handle
        self.n_rows, self.nnz = h.n_rows, h.nnz

    def refresh(self, a: CsrMatrix) -> None:
        _check(_load().b2_mixed_refresh(self._handle, _tptr(a.val), _stream()))

    def assemble_refresh(self, a: CsrMatrix, fv: "FvPressure", rhs) -> None:
        """b2_mixed_assemble_refresh (see LinearSolver.assemble_refresh)."""
        _check(_load().b2_mixed_assemble_refresh(self._handle, *fv.pointers(), _tptr(a.val),
                                                 _tptr(rhs), fv.reference, _stream()))

    def solve(self, a: CsrMatrix, x, b, control: SolveControl | None = None) -> MixedStats:
        """x: float64 CUDA tensor (initial guess in, FP64 solution out), or
        float32 (b2_mixed_solve_f32: the solution rounded to FP32, as
        LinearSolver.solve returns it); b: float32."""
        import torch
        if x.dtype not in (torch.float64, torch.float32) or x.numel() != self.n_rows \
                or b.numel() != self.n_rows:
            raise KuttaError("solve: vector size or alias mismatch")
        control = control or SolveControl()
        c = _Control(control.rel_tol, control.abs_tol, control.max_iter,
                     control.residual_check_interval)
        st = _MixedStats()
        entry = _load().b2_mixed_solve if x.dtype == torch.float64 else _load().b2_mixed_solve_f32
        _check(entry(self._handle, _tptr(a.val), _tptr(x), _tptr(b), ctypes.byref(c),
                     ctypes.byref(st), _stream()))
        return MixedStats(st.refinements, st.iterations, bool(st.converged), st.initial_residual,
                          st.final_residual, bool(st.learned_fallback))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        _load().b2_mixed_describe(self._handle, buf, 512)
        return buf.value.decode()

    def profile(self, enable: bool) -> None:
        _check(_load().b2_mixed_profile(self._handle, int(enable)))

    def profile_read(self) -> dict:
        p = _Profile()
        _check(_load().b2_mixed_profile_read(self._handle, ctypes.byref(p)))
        return {f: getattr(p, f) for f, _ in _Profile._fields_}

    def set_learned(self, stage: "LearnedStage | None", mode: int = LEARNED_CYCLE) -> None:
        """Attaches a learned stage (None detaches): after each AMG cycle
        (LEARNED_CYCLE, the energy-optimal step) and/or as a warm-start step
        (LEARNED_WARM_START, the residual-optimal step); the stage must stay
        alive while attached."""
        self._learned = stage
        _check(_load().b2_mixed_set_learned(self._handle, stage._handle if stage else None,
                                            int(mode) if stage else 0))

    def precondition(self, a: CsrMatrix, r, z) -> None:
        """z = M(r): one application of the preconditioner (float32 tensors)."""
        _check(_load().b2_mixed_precondition(self._handle, _tptr(a.val), _tptr(r), _tptr(z),
                                             _stream()))

    def __del__(self):
        if getattr(self, "_handle", None) and _lib is not None:
            _lib.b2_mixed_destroy(self._handle)
            self._handle = None


class LearnedStage:
    """b2_gnn: the learned preconditioner stage (no reference counterpart), a
    3-layer message-passing network of width 32 over the matrix graph, mapping
    a residual r to a correction direction G(r) (G(lambda r) = lambda G(r));
    trained with hand-written CUDA forward, backward and Adam kernels on the
    energy loss of (residual, error) pairs."""

    def __init__(self, seed: int = 1):
        handle = ctypes.c_void_p()
        _check(_load().b2_gnn_create(seed, ctypes.byref(handle)))
        self._handle = handle

    @staticmethod
    def parameter_count() -> int:
        return int(_load().b2_gnn_parameter_count())

    def bind(self, a: CsrMatrix) -> None:
        self._bound = a
        _check(_load().b2_gnn_bind(self._handle, a.n_rows, _tptr(a.row_ptr), _tptr(a.col),
                                   _tptr(a.diag), _tptr(a.val), _stream()))

    def set_geometry(self, geometry) -> None:
        """b2_gnn_set_geometry: per-entry geometric face coefficients (a CUDA
        float32 tensor over the bound pattern, 0 on the diagonal) for the
        matrices bound from now on, or None. The tensor is kept alive here."""
        self._geometry = geometry
        _check(_load().b2_gnn_set_geometry(self._handle, _tptr(geometry)))

    def apply(self, r, z, beta: float = 0.0) -> None:
        _check(_load().b2_gnn_apply(self._handle, _tptr(r), _tptr(z), beta, _stream()))

    def set_wait_limit(self, polls: int) -> None:
        """Testing hook: each tensor-core tile's first wait for its MMA polls at
        most `polls` times (< 0: the built-in bound) before the forward gives
        up and raises DeviceTimeout."""
        _check(_load().b2_gnn_set_wait_limit(self._handle, int(polls)))

    def train_step(self, t, e, learning_rate: float = 1e-3) -> float:
        """One Adam step on the energy loss 1 - (c.t)^2 / ((c.Ac)(t.e)), c = G(t),
        for A e = t with the bound matrix; returns the loss before the step."""
        loss = ctypes.c_float()
        _check(_load().b2_gnn_train_step(self._handle, _tptr(t), _tptr(e), learning_rate,
                                         ctypes.byref(loss), _stream()))
        return float(loss.value)

    def gradient(self, t, e, tensor_cores: bool = True) -> tuple[np.ndarray, float]:
        """(gradient of the energy loss at the current weights, loss), no step;
        tensor_cores: the 32-wide layers' backward on the tensor cores (as
        train_step) or in FP32 on CUDA cores."""
        g = np.empty(self.parameter_count(), np.float32)
        loss = ctypes.c_float()
        _check(_load().b2_gnn_gradient(self._handle, _tptr(t), _tptr(e), int(tensor_cores),
                                       _ptr(g), g.size, ctypes.byref(loss), _stream()))
        return g, float(loss.value)

    def weights(self) -> np.ndarray:
        w = np.empty(self.parameter_count(), np.float32)
        _check(_load().b2_gnn_get_weights(self._handle, _ptr(w), w.size))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        _check(_load().b2_gnn_set_weights(self._handle, _ptr(w), w.size))

    def __del__(self):
        if getattr(self, "_handle", None) and _lib is not None:
            _lib.b2_gnn_destroy(self._handle)
            self._handle = None


@dataclasses.dataclass
class FvPressure:
    """Face data of the pressure assembly (fv_pressure_assemble's inputs,
    src/kutta/kernels/fv_flow.kern.h:164-167) as CUDA tensors: cell-face slot
    offsets (int32, n_cells + 1), the face, side sign (+1 owner, -1
    neighbour), adjacent cell (-1 boundary) and CSR entry of each slot, and
    per-face coefficients and mass fluxes (float32); reference: an eliminated
    cell or -1."""
    offsets: object
    faces: object
    sign: object
    adjacent: object
    entry: object
    coefficient: object
    flux: object
    reference: int = -1

    def pointers(self):
        return (_tptr(self.offsets), _tptr(self.faces), _tptr(self.sign), _tptr(self.adjacent),
                _tptr(self.entry), _tptr(self.coefficient), _tptr(self.flux))


def fv_pressure_assemble(a: CsrMatrix, fv: FvPressure, rhs) -> None:
    """b2_fv_pressure_assemble: the pressure matrix into a.val and rhs."""
    o, f, sg, adj, e, c, fl = fv.pointers()
    _check(_load().b2_fv_pressure_assemble(a.n_rows, o, f, sg, adj, e, _tptr(a.row_ptr),
                                           _tptr(a.diag), c, fl, _tptr(a.val), _tptr(rhs),
                                           fv.reference, _stream()))


def fv_correct_flux(owner, neighbour, correction, coefficient, flux, internal: int) -> None:
    """b2_fv_correct_flux over owner.numel() faces."""
    _check(_load().b2_fv_correct_flux(owner.numel(), _tptr(owner), _tptr(neighbour),
                                      _tptr(correction), _tptr(coefficient), _tptr(flux),
                                      internal, _stream()))


def fv_correct_velocity(volume, inverse, diagonal, gx, gy, gz, correction, u, v, w, p,
                        alpha: float) -> None:
    """b2_fv_correct_velocity over volume.numel() cells."""
    _check(_load().b2_fv_correct_velocity(volume.numel(), *(_tptr(t) for t in (
        volume, inverse, diagonal, gx, gy, gz, correction, u, v, w, p)), alpha, _stream()))


def dense_inverse(a: CsrMatrix, inverse, not_spd) -> None:
    """Dense FP64 Cholesky inverse of a small SPD CSR operator (n <= 1024):
    inverse (n*n float64 CUDA tensor, row-major) and not_spd (1 float64 flag)."""
    _check(_load().b2_dense_inverse(a.n_rows, _tptr(a.row_ptr), _tptr(a.col), _tptr(a.val),
                                    _tptr(inverse), _tptr(not_spd), _stream()))


def dense_inverse_noalloc(a: CsrMatrix, inverse, not_spd) -> None:
    """dense_inverse for callers that cannot allocate device memory (n <= 512):
    the factor scratch is a 2 MiB array built into the library, shared by every
    call on the device, so calls that overlap on the GPU race. The first call on
    a device looks that array up; make it before any stream capture."""
    _check(_load().b2_dense_inverse_noalloc(a.n_rows, _tptr(a.row_ptr), _tptr(a.col),
                                            _tptr(a.val), _tptr(inverse), _tptr(not_spd),
                                            _stream()))


def make_mixed_solver(a, options: MixedOptions | None = None) -> MixedSolver:
    return MixedSolver(a, options)


def build_mixed_hierarchy(a, options: MixedOptions | None = None) -> list:
    """The mixed solve's host hierarchy (no GPU)."""
    lib = _load()
    h = _host(a)
    row_ptr, col, diag, val = h.arrays()
    opts = _mixed_struct(options or MixedOptions())
    handle = ctypes.c_void_p()
    _check(lib.b2_mixed_hierarchy_build(h.n_rows, h.nnz, _ptr(row_ptr), _ptr(col), _ptr(diag),
                                        _ptr(val), ctypes.byref(opts), ctypes.byref(handle)))
    return _read_hierarchy(lib, handle)


def _read_hierarchy(lib, handle) -> list:
    out = []
    try:
        count = lib.b2_hierarchy_levels(handle)
        for lv in range(count):
            n, nnz = ctypes.c_int(), ctypes.c_int()
            _check(lib.b2_hierarchy_level_shape(handle, lv, ctypes.byref(n), ctypes.byref(nnz)))
            rp = np.zeros(n.value + 1, np.int32)
            cl = np.zeros(nnz.value, np.int32)
            vl = np.zeros(nnz.value, np.float32)
            l1 = np.zeros(n.value, np.float32)
            ag = np.zeros(n.value, np.int32) if lv + 1 < count else None
            _check(lib.b2_hierarchy_level_copy(handle, lv, _ptr(rp), _ptr(cl), _ptr(vl), _ptr(l1),
                                               _ptr(ag) if ag is not None else None))
            out.append(HostLevel(n.value, rp, cl, vl, l1, ag))
    finally:
        lib.b2_hierarchy_free(handle)
    return out


@dataclasses.dataclass
class HostLevel:
    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    inverse_l1: np.ndarray
    aggregate: np.ndarray | None


def build_hierarchy(a, options: AmgOptions | None = None, spd: bool = True) -> list[HostLevel]:
    """The host AMG setup alone (no GPU): aggregates, coarse operators, L1 diagonals."""
    lib = _load()
    h = _host(a)
    row_ptr, col, diag, val = h.arrays()
    opts = _options_struct(options or AmgOptions(), True)
    handle = ctypes.c_void_p()
    _check(lib.b2_hierarchy_build(h.n_rows, h.nnz, _ptr(row_ptr), _ptr(col), _ptr(diag),
                                  _ptr(val), ctypes.byref(opts), int(spd), ctypes.byref(handle)))
    out = []
    try:
        count = lib.b2_hierarchy_levels(handle)
        for lv in range(count):
            n, nnz = ctypes.c_int(), ctypes.c_int()
            _check(lib.b2_hierarchy_level_shape(handle, lv, ctypes.byref(n), ctypes.byref(nnz)))
            rp = np.zeros(n.value + 1, np.int32)
            cl = np.zeros(nnz.value, np.int32)
            vl = np.zeros(nnz.value, np.float32)
            l1 = np.zeros(n.value, np.float32)
            ag = np.zeros(n.value, np.int32) if lv + 1 < count else None
            _check(lib.b2_hierarchy_level_copy(handle, lv, _ptr(rp), _ptr(cl), _ptr(vl), _ptr(l1),
                                               _ptr(ag) if ag is not None else None))
            out.append(HostLevel(n.value, rp, cl, vl, l1, ag))
    finally:
        lib.b2_hierarchy_free(handle)
    return out


# ---- Coupled (4x4-block) pressure-velocity solve -----------------------------------
# kutta::fv::CoupledSolver (src/kutta/fv/coupled_solver.hpp:61-101).

@dataclasses.dataclass
class CoupledOptions:  # coupled_solver.hpp:26-38
    pre_sweeps: int = 1
    post_sweeps: int = 2
    coarsest_sweeps: int = 8
    smoother_damping: float = 0.7
    courant: float = 200.0
    coarsest_rows: int = 48
    aggregation_passes: int = 3
    recompute: bool = False


class _CoupledOptions(ctypes.Structure):
    _fields_ = [("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarsest_sweeps", ctypes.c_int), ("smoother_damping", ctypes.c_float),
                ("courant", ctypes.c_double), ("coarsest_rows", ctypes.c_int),
                ("aggregation_passes", ctypes.c_int), ("recompute", ctypes.c_int)]


def _coupled_options(o: CoupledOptions | None) -> _CoupledOptions:
    o = o or CoupledOptions()
    return _CoupledOptions(o.pre_sweeps, o.post_sweeps, o.coarsest_sweeps, o.smoother_damping,
                           o.courant, o.coarsest_rows, o.aggregation_passes, int(o.recompute))


# b2_coupled_mesh field order: (name, dtype) of each host array.
_COUPLED_MESH = [
    ("owner", np.int32), ("neighbour", np.int32), ("cell_face_offsets", np.int32),
    ("cell_faces", np.int32), ("cell_face_sign", np.float32), ("adjacent", np.int32),
    ("area_x", np.float32), ("area_y", np.float32), ("area_z", np.float32),
    ("face_area", np.float64), ("cell_centroid", np.float64),
    ("owner_to_face_x", np.float32), ("owner_to_face_y", np.float32),
    ("owner_to_face_z", np.float32), ("neighbour_to_face_x", np.float32),
    ("neighbour_to_face_y", np.float32), ("neighbour_to_face_z", np.float32),
    ("lsq_x", np.float32), ("lsq_y", np.float32), ("lsq_z", np.float32),
    ("boundary_delta_x", np.float32), ("boundary_delta_y", np.float32),
    ("boundary_delta_z", np.float32), ("lsq_inverse", np.float32), ("diffusion", np.float32),
    ("volume", np.float32), ("boundary_kind", np.int32), ("pattern_row_ptr", np.int32),
    ("pattern_col", np.int32), ("pattern_diag", np.int32), ("low_order", np.int32),
]


class _CoupledMesh(ctypes.Structure):
    _fields_ = [("n_cells", ctypes.c_int), ("n_faces", ctypes.c_int),
                ("n_internal", ctypes.c_int)] + [(name, _P) for name, _ in _COUPLED_MESH]


class _CoupledResiduals(ctypes.Structure):
    _fields_ = [(name, _P) for name in ("ru", "rv", "rw", "mass", "viscosity",
                                        "physical_diagonal", "face_weights", "net_outflow")] + \
               [("density", ctypes.c_double), ("velocity_scale", ctypes.c_double)]


class CoupledMesh:
    """The host arrays of b2_coupled_mesh, by name (the keys a reference box
    case or coupled_harness.box_hex / box_tet give; `lsq_x` are the pressure fit's rows,
    `low_order` is optional). The arrays are kept alive with the struct."""

    def __init__(self, arrays: dict):
        sizes = np.asarray(arrays["sizes"])
        self.n_cells, self.n_faces, self.n_internal = (int(v) for v in sizes[:3])
        self._keep = {}
        fields = {}
        for name, dtype in _COUPLED_MESH:
            src = name if name not in ("lsq_x", "lsq_y", "lsq_z") else name
            a = arrays.get(src)
            if a is None:
                fields[name] = None
                continue
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep[name] = a
            fields[name] = _ptr(a)
        self.struct = _CoupledMesh(self.n_cells, self.n_faces, self.n_internal,
                                   *(fields[name] for name, _ in _COUPLED_MESH))


class CoupledSolver:
    """b2_coupled: the Coupled block solve. Vectors are CUDA tensors on torch's
    current stream: per-cell and per-face float32 fields, momentum CSR
    arrays over the stencil pattern."""

    def __init__(self, mesh, reference: int = -1, options: CoupledOptions | None = None):
        lib = _load()
        self.mesh = mesh if isinstance(mesh, CoupledMesh) else CoupledMesh(mesh)
        opts = _coupled_options(options)
        handle = ctypes.c_void_p()
        _check(lib.b2_coupled_create(ctypes.byref(self.mesh.struct), int(reference),
                                     ctypes.byref(opts), _stream(), ctypes.byref(handle)))
        self._handle = handle
        self.n_cells = self.mesh.n_cells
        self.n_faces = self.mesh.n_faces

    def capture_diagonal(self, component: int, row_ptr, diag, values, physical) -> None:
        _check(_load().b2_coupled_capture_diagonal(self._handle, int(component), _tptr(row_ptr),
                                                   _tptr(diag), _tptr(values), _tptr(physical),
                                                   _stream()))

    def solve(self, fields: dict, control: SolveControl | None = None) -> SolveStats:
        """fields: ru, rv, rw, mass, viscosity, physical_diagonal, face_weights
        (CUDA float32 tensors), net_outflow (tensor or None), density and
        velocity_scale (floats)."""
        r = _CoupledResiduals(*(_tptr(fields.get(k)) for k in (
            "ru", "rv", "rw", "mass", "viscosity", "physical_diagonal", "face_weights",
            "net_outflow")), float(fields["density"]), float(fields["velocity_scale"]))
        control = control or SolveControl(0.1, 1e-12, 20)
        c = _Control(control.rel_tol, control.abs_tol, control.max_iter,
                     control.residual_check_interval)
        st = _Stats()
        _check(_load().b2_coupled_solve(self._handle, ctypes.byref(r), ctypes.byref(c),
                                        ctypes.byref(st), _stream()))
        return SolveStats(st.iterations, st.initial_residual, st.final_residual,
                          bool(st.converged))

    def update(self, u, v, w, p, alpha_u: float, alpha_p: float) -> None:
        _check(_load().b2_coupled_update(self._handle, _tptr(u), _tptr(v), _tptr(w), _tptr(p),
                                         float(alpha_u), float(alpha_p), _stream()))

    def paired_update(self, u, v, w, p, u_lo, v_lo, w_lo, p_lo, alpha_u: float,
                      alpha_p: float, velocity_slack: float, pressure_slack: float) -> None:
        _check(_load().b2_coupled_paired_update(
            self._handle, *(_tptr(t) for t in (u, v, w, p, u_lo, v_lo, w_lo, p_lo)),
            float(alpha_u), float(alpha_p), float(velocity_slack), float(pressure_slack),
            _stream()))

    def bytes(self) -> int:
        return int(_load().b2_coupled_bytes(self._handle))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        _load().b2_coupled_describe(self._handle, buf, 512)
        return buf.value.decode()

    def copy(self, what: str) -> np.ndarray:
        """'x' / 'rhs' (4n, planes [u|v|w|p~]), 'cell' (27n), 'coefficient' (n_faces)."""
        code = {"x": 0, "rhs": 1, "cell": 2, "coefficient": 3}[what]
        lib = _load()
        count = lib.b2_coupled_copy(self._handle, code, None, _stream())
        if count < 0:
            _check(1)
        out = np.zeros(count, np.float32)
        if lib.b2_coupled_copy(self._handle, code, _ptr(out), _stream()) < 0:
            _check(1)
        return out

    def levels(self) -> int:
        return int(_load().b2_coupled_levels(self._handle))

    def level(self, k: int) -> dict:
        """Coarse level k >= 1: rows, cols, diag, a, c, g, h, d and the aggregate
        of level k - 1."""
        lib = _load()
        n, nnz = ctypes.c_int(), ctypes.c_int()
        _check(lib.b2_coupled_level_shape(self._handle, k, ctypes.byref(n), ctypes.byref(nnz)))
        prev = ctypes.c_int()
        _check(lib.b2_coupled_level_shape(self._handle, k - 1, ctypes.byref(prev), None))
        n, nnz = n.value, nnz.value
        out = {"rows": np.zeros(n + 1, np.int32), "cols": np.zeros(nnz, np.int32),
               "diag": np.zeros(n, np.int32), "a": np.zeros(nnz, np.float32),
               "c": np.zeros(nnz, np.float32), "g": np.zeros(3 * nnz, np.float32),
               "h": np.zeros(3 * nnz, np.float32), "d": np.zeros(11 * n, np.float32),
               "aggregate": np.zeros(prev.value, np.int32)}
        _check(lib.b2_coupled_level_copy(self._handle, k, *(_ptr(out[key]) for key in (
            "rows", "cols", "diag", "a", "c", "g", "h", "d", "aggregate")), _stream()))
        return out

    def apply(self, op: str, x, b, y) -> None:
        """op 'spmv' (y = J x), 'residual' (y = b - J x), 'smooth' (one sweep
        from x), 'smooth_zero' (from x = 0); float4-per-cell CUDA tensors."""
        code = {"spmv": 0, "residual": 1, "smooth": 2, "smooth_zero": 3}[op]
        _check(_load().b2_coupled_apply(self._handle, code, _tptr(x), _tptr(b), _tptr(y),
                                        _stream()))

    def level_apply(self, level: int, op: str, x, b, y) -> None:
        """On coarse level `level` >= 1: 'residual', 'smooth', 'smooth_zero';
        'restrict' (x on level - 1, y on level), 'prolong' (y on level - 1 +=
        x on level)."""
        code = {"residual": 1, "smooth": 2, "smooth_zero": 3, "restrict": 4, "prolong": 5}[op]
        _check(_load().b2_coupled_level_apply(self._handle, int(level), code, _tptr(x), _tptr(b),
                                              _tptr(y), _stream()))

    def __del__(self):
        if getattr(self, "_handle", None) and _lib is not None:
            _lib.b2_coupled_destroy(self._handle)
            self._handle = None


def build_coupled_setup(mesh, options: CoupledOptions | None = None) -> dict:
    """Host-only Coupled setup (b2_coupled_setup_build): 'cell' (27n with the
    sensitivities), 'width', and per level its n, rows/cols/diag (coarse
    levels) and aggregate/member_offsets/members (all but the coarsest)."""
    lib = _load()
    mesh = mesh if isinstance(mesh, CoupledMesh) else CoupledMesh(mesh)
    opts = _coupled_options(options)
    h = ctypes.c_void_p()
    _check(lib.b2_coupled_setup_build(ctypes.byref(mesh.struct), ctypes.byref(opts),
                                      ctypes.byref(h)))
    try:
        cell = np.zeros(27 * mesh.n_cells, np.float32)
        _check(lib.b2_coupled_setup_cell(h, _ptr(cell)))
        count = lib.b2_coupled_setup_levels(h)
        sizes = []
        for k in range(count):
            n, nnz = ctypes.c_int(), ctypes.c_int()
            _check(lib.b2_coupled_setup_level_shape(h, k, ctypes.byref(n), ctypes.byref(nnz)))
            sizes.append((n.value, nnz.value))
        levels = []
        for k, (n, nnz) in enumerate(sizes):
            lv = {"n": n}
            if k > 0:
                lv.update(rows=np.zeros(n + 1, np.int32), cols=np.zeros(nnz, np.int32),
                          diag=np.zeros(n, np.int32))
            if k + 1 < count:
                lv.update(aggregate=np.zeros(n, np.int32),
                          member_offsets=np.zeros(sizes[k + 1][0] + 1, np.int32),
                          members=np.zeros(n, np.int32))
            _check(lib.b2_coupled_setup_level_copy(h, k, *(_ptr(lv.get(key)) for key in (
                "rows", "cols", "diag", "aggregate", "member_offsets", "members"))))
            levels.append(lv)
        return {"cell": cell, "width": int(lib.b2_coupled_setup_width(h)), "levels": levels}
    finally:
        lib.b2_coupled_setup_free(h)
