"""The C ABI's argument contract, without a GPU: every entry point rejects a
null handle, a null output or a null array of a non-empty input with
B2_INVALID_ARGUMENT and a message, treats empty inputs (n = 0) as a no-op,
and does either before any device work. On this CPU-only machine a device
call fails with B2_DEVICE_ERROR, so that status showing up means a check
came too late. The destroy functions accept NULL, as free() does."""
import ctypes

import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L

B2_OK, B2_INVALID_ARGUMENT, B2_DEVICE_ERROR = 0, 1, 3
# The int-returning entry points that return a status (the others return counts).
COUNTS = {"b2_gnn_parameter_count", "b2_solver_levels", "b2_hierarchy_levels",
          "b2_coupled_levels", "b2_coupled_setup_levels", "b2_coupled_setup_width"}
STATUS_FUNCTIONS = [n for n, (res, _) in L._SIGNATURES.items() if res is ctypes.c_int
                    and n not in COUNTS]
# Entry points whose all-zero call is a valid empty operation.
EMPTY_OK = {"b2_csr_spmv", "b2_csr_residual", "b2_amg_smooth", "b2_fv_correct_flux",
            "b2_fv_correct_velocity"}


def _args(name, size):
    out = []
    for a in L._SIGNATURES[name][1]:
        if a in (ctypes.c_float, ctypes.c_double):
            out.append(0.5)
        elif a in (ctypes.c_int, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_longlong):
            out.append(size)
        else:
            out.append(None)
    return out


def _call(name, args):
    lib = L._load()
    status = getattr(lib, name)(*args)
    return status, L.last_error()


@pytest.fixture(scope="module", autouse=True)
def no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks that no device work happens need a machine without a GPU")


@pytest.mark.parametrize("name", STATUS_FUNCTIONS)
def test_zero_arguments_are_rejected_or_empty_before_device_work(name):
    status, message = _call(name, _args(name, 0))
    if name in EMPTY_OK:
        assert status == B2_OK, message
    else:
        assert status == B2_INVALID_ARGUMENT, (status, message)
        assert message


@pytest.mark.parametrize("name", STATUS_FUNCTIONS)
def test_null_arrays_of_non_empty_inputs_are_rejected(name):
    """Sizes of 4 with every pointer NULL: a handle, an output or an array is
    missing, whichever the entry point checks first."""
    status, message = _call(name, _args(name, 4))
    if name == "b2_workspace_create":  # no pointer inputs besides the output handle
        assert status == B2_INVALID_ARGUMENT and "invalid arguments" in message
        return
    assert status == B2_INVALID_ARGUMENT, (status, message)
    assert any(w in message for w in ("null", "out of range", "alias", "outside")), message


def test_kernel_entry_points_name_the_missing_array():
    lib = L._load()
    x, y = ctypes.c_void_p(16), ctypes.c_void_p(32)  # never dereferenced: the checks fail first
    assert lib.b2_csr_spmv(4, 8, None, None, None, x, y, None) == B2_INVALID_ARGUMENT
    assert L.last_error() == "CSR: null argument"
    assert lib.b2_csr_residual(4, 8, None, None, None, x, x, y, None) == B2_INVALID_ARGUMENT
    assert L.last_error() == "CSR: null argument"
    assert lib.b2_amg_smooth(4, None, None, None, None, x, x, y, 1, None) == B2_INVALID_ARGUMENT
    assert L.last_error() == "smooth: null argument"


def test_destroy_functions_accept_null():
    lib = L._load()
    for name in ("b2_workspace_destroy", "b2_solver_destroy", "b2_hierarchy_free",
                 "b2_mixed_destroy", "b2_gnn_destroy"):
        getattr(lib, name)(None)


def test_describe_and_level_counts_of_null_handles_are_zero():
    lib = L._load()
    buf = ctypes.create_string_buffer(16)
    assert lib.b2_solver_describe(None, buf, 16) == 0
    assert lib.b2_mixed_describe(None, buf, 16) == 0
    assert lib.b2_solver_levels(None) == 0
    assert lib.b2_hierarchy_levels(None) == 0


def test_last_error_reports_its_full_length_and_truncates():
    lib = L._load()
    assert lib.b2_solver_refresh(None, None, None) == B2_INVALID_ARGUMENT
    full = lib.b2_last_error(None, 0)
    assert full == len("solver: null handle")
    small = ctypes.create_string_buffer(7)
    assert lib.b2_last_error(small, 7) == full
    assert small.value == b"solver"


def test_header_is_c99_and_a_c_caller_links_and_runs():
    """tests/c_abi_check.c: the header compiles as C99 with -pedantic, a C
    program links against the library, and its calls that fail before device
    work return the declared statuses and the reference's messages."""
    import pathlib
    import subprocess
    root = pathlib.Path(__file__).resolve().parent.parent
    lib_dir = L.library_path().parent
    out = lib_dir / "checks"
    out.mkdir(exist_ok=True)
    exe = out / "c_abi_check"
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
           f"-I{root / 'include'}", str(root / "tests" / "c_abi_check.c"), "-o", str(exe),
           f"-L{lib_dir}", "-lkutta_b200", f"-Wl,-rpath,{lib_dir}", "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_python_mirror_maps_statuses_and_checks_before_device_work():
    """linalg.py raises the reference's exception types for the ABI's statuses,
    and its factories reject what the reference rejects before device work;
    an accepted input then meets the missing device as a DeviceError."""
    s = harness.poisson(6, 5, 4)
    m = L.AmgOptions(structure=L.OperatorStructure.SymmetricMMatrix)
    with pytest.raises(L.KuttaError, match="AMG: expected an AMG solver kind"):
        L.make_amg_solver(L.SolverKind.PcgJacobi, s, L.AmgOptions())
    with pytest.raises(L.KuttaError, match="AMG-PCG requires equal pre/post sweeps"):
        L.make_amg_solver(L.SolverKind.AmgPcg, s, L.AmgOptions(pre_sweeps=1, post_sweeps=2))
    with pytest.raises(L.KuttaError, match="Krylov workspace size mismatch"):
        L.make_solver(L.SolverKind.BicgstabJacobi, s,
                      L.SolverOptions(workspace=L.KrylovWorkspace(s.n + 1)))
    bad = harness.HostSystem(s.row_ptr, s.col, s.diag, s.val.copy(), s.b)
    bad.val[bad.diag[7]] = 0.0
    with pytest.raises(L.KuttaError, match="zero diagonal"):
        L.make_solver(L.SolverKind.PcgJacobi, bad)
    for make in (lambda: L.make_amg_solver(L.SolverKind.AmgPcg, s, m),
                 lambda: L.make_solver(L.SolverKind.PcgJacobi, s),
                 lambda: L.make_mixed_solver(s)):
        with pytest.raises(L.DeviceError) as e:
            make()
        assert not isinstance(e.value, L.DeviceTimeout)
    for code, kind in ((1, L.KuttaError), (2, L.NonfiniteError), (3, L.DeviceError),
                       (4, L.DeviceTimeout), (5, L.DeviceError), (6, L.KuttaError)):
        with pytest.raises(kind):
            L._check(code)
    L._check(0)
