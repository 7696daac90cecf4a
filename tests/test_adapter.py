"""The reference-side adapter (kutta_b200/csrc/adapter/b200_solver.cpp), which
implements kutta::LinearSolver (src/kutta/linalg/solver.hpp:74-81) over the C
ABI. Compiled here against the reference's own headers, with warnings as
errors, and linked with the reference's CPU library and libkutta_b200.so.
tests/adapter_check.cpp then runs the reference's factories
(make_amg_solver, make_solver on the CPU Device) and the adapter's on the same
inputs; the adapter's mixed-precision factory is compared with the pressure
solver it stands in for, make_solver(AmgPcg). Every input the reference rejects before device work is rejected by
the adapter with the same exception type and message, and the inputs it
accepts pass every host check of the adapter (whose solver then needs a
GPU). The AMG diagonal checks (solver.cpp:37-53) run on the device during
the device setup, so without a GPU that case only shows the host checks
passing.

Runs only where the reference sources and oracle/_ref are present and no GPU
is visible."""
import os
import pathlib
import subprocess

import pytest

from kutta_b200 import linalg as L
from oracle import build as oracle_build

ROOT = pathlib.Path(__file__).resolve().parent.parent
ADAPTER = ROOT / "kutta_b200" / "csrc" / "adapter" / "b200_solver.cpp"
CHECK = ROOT / "tests" / "adapter_check.cpp"
REF_LIB = ROOT / "oracle" / "_ref" / "libkutta_ref.so"
OUT = ROOT / "oracle" / "_ref" / "adapter"
# Checked on the device by the device setup (same message there).
DEVICE_CHECKED = {"negative_diagonal"}


def _cuda_include():
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return pathlib.Path(home) / "include"


def _headers():
    return oracle_build.REFERENCE / "src"


needs_reference = pytest.mark.skipif(
    not (_headers() / "kutta" / "linalg" / "solver.hpp").exists() or not REF_LIB.exists()
    or not (_cuda_include() / "cuda_runtime.h").exists(),
    reason="reference sources, oracle/_ref or the CUDA headers not present")


def _compile(src, obj, includes):
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-fPIC",
           *(f"-I{i}" for i in includes), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.fixture(scope="module")
def adapter_check():
    OUT.mkdir(parents=True, exist_ok=True)
    lib_dir = L.library_path().parent
    _compile(ADAPTER, OUT / "b200_solver.o", [_headers(), _cuda_include(), ROOT / "include"])
    _compile(CHECK, OUT / "adapter_check.o", [_headers()])
    exe = OUT / "adapter_check"
    cmd = ["g++", str(OUT / "b200_solver.o"), str(OUT / "adapter_check.o"), "-o", str(exe),
           f"-L{REF_LIB.parent}", "-lkutta_ref", f"-L{lib_dir}", "-lkutta_b200",
           f"-Wl,-rpath,{REF_LIB.parent}", f"-Wl,-rpath,{lib_dir}",
           "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _strip_location(message):
    """'csr.cpp:28: CSR: ...' -> 'CSR: ...' (KUTTA_REQUIRE, core/types.hpp:42-46)."""
    head, sep, rest = message.partition(": ")
    return rest if sep and ".cpp:" in head else message


@needs_reference
def test_adapter_rejects_what_the_reference_rejects(adapter_check):
    import torch
    if torch.cuda.is_available():
        pytest.skip("the expectations for accepted inputs are those without a GPU")
    r = subprocess.run([str(adapter_check)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = [line.split("|") for line in r.stdout.splitlines()]
    assert len(rows) >= 32
    for name, ref_type, ref_message, b2_type, b2_message in rows:
        if ref_type == "none" or name in DEVICE_CHECKED:
            # Every host check passed; the adapter then stops at the missing GPU.
            assert b2_type == "Error" and b2_message.startswith("CUDA error"), (name, b2_message)
            assert (ref_type == "none") == name.startswith(("valid", "mixed_valid",
                                                             "nullspace_row")), name
        else:
            assert (b2_type, b2_message) == (ref_type, _strip_location(ref_message)), name
