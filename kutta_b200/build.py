"""Build recipe for the native parts of kutta_b200.

Compiles, in-tree, into ``kutta_b200/_lib/``:

* ``libkutta_b200.so``: the product: sm_100a CUDA kernels (nvcc,
  ``-gencode arch=compute_100a,code=sm_100a``), host setup and Krylov drivers
  (g++), and the C ABI of ``include/kutta_b200.h``;
* ``libkutta_harness.so``: synthetic system generators (C).

Rebuilds only when a source's content changed (a hash stamp per output).
Run ``python -m kutta_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "_lib"
OBJ = PKG / "_lib" / "obj"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# Reference-parity kernels: no FMA contraction, IEEE division and square root,
# no flush-to-zero, so float results round exactly like the reference CPU path.
EXACT = ["--fmad=false", "--prec-div=true", "--prec-sqrt=true", "--ftz=false"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             f"-I{CUDA_HOME}/include", f"-I{ROOT / 'include'}"]

PRODUCT_CU = {
    "exact_kernels.cu": EXACT,
    "mixed_kernels.cu": [],
    "tail_cycle.cu": [],
    "learned.cu": [],
    "learned_tc.cu": [],
    "setup_kernels.cu": EXACT,
    "fv_kernels.cu": EXACT,
    "noalloc.cu": [],
    "coupled_kernels.cu": EXACT,
}
PRODUCT_CPP = ["host/setup.cpp", "host/solver.cpp", "host/device_setup.cpp", "host/mixed.cpp",
               "host/learned.cpp", "host/coupled_setup.cpp", "host/coupled.cpp", "capi.cpp"]


def _hash(paths, extra=""):
    h = hashlib.sha256(extra.encode())
    for p in sorted(paths):
        h.update(str(p).encode())
        h.update(pathlib.Path(p).read_bytes())
    return h.hexdigest()


def _deps():
    """Every header that a product source may include."""
    return list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + [ROOT / "include" / "kutta_b200.h"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _up_to_date(out: pathlib.Path, digest: str) -> bool:
    stamp = out.with_suffix(out.suffix + ".stamp")
    return out.exists() and stamp.exists() and stamp.read_text() == digest


def _stamp(out: pathlib.Path, digest: str):
    out.with_suffix(out.suffix + ".stamp").write_text(digest)


def build_product(verbose=False) -> pathlib.Path:
    LIB.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    out = LIB / "libkutta_b200.so"
    sources = [CSRC / "cuda" / f for f in PRODUCT_CU] + [CSRC / f for f in PRODUCT_CPP]
    flags = repr((NVCC_FLAGS, CXX_FLAGS, PRODUCT_CU))
    digest = _hash(sources + _deps(), flags)
    if _up_to_date(out, digest):
        return out
    jobs = []
    objs = []
    for name, extra in PRODUCT_CU.items():
        src = CSRC / "cuda" / name
        obj = OBJ / (name + ".o")
        objs.append(obj)
        jobs.append([NVCC, *NVCC_FLAGS, *extra, f"-I{ROOT / 'include'}", "-c", str(src), "-o", str(obj)])
    for name in PRODUCT_CPP:
        src = CSRC / name
        obj = OBJ / (name.replace("/", "_") + ".o")
        objs.append(obj)
        jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        logs = list(ex.map(_run, jobs))
    if verbose:
        for log in logs:
            if log.strip():
                print(log)
    _run([NVCC, "-shared", *ARCH, "-o", str(out), *map(str, objs),
          f"-L{CUDA_HOME}/lib64", "-lcudart"])
    _stamp(out, digest)
    return out


def build_harness() -> pathlib.Path:
    LIB.mkdir(parents=True, exist_ok=True)
    out = LIB / "libkutta_harness.so"
    src = CSRC / "harness" / "systems.c"
    digest = _hash([src])
    if not _up_to_date(out, digest):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-Wall", str(src), "-o", str(out), "-lm"])
        _stamp(out, digest)
    return out


def build_oracle() -> None:
    """The oracle (test infrastructure): the C restatement, and the reference's
    own CPU path when its sources are present on this machine."""
    sys.path.insert(0, str(ROOT))
    try:
        from oracle import build as oracle_build  # noqa: WPS433
    finally:
        sys.path.pop(0)
    oracle_build.build()


def ptxas_report(name="exact_kernels.cu") -> str:
    """Registers / spills / shared memory per kernel (nvcc -Xptxas -v)."""
    src = CSRC / "cuda" / name
    extra = PRODUCT_CU.get(name, [])
    r = subprocess.run([NVCC, *NVCC_FLAGS, *extra, "-Xptxas", "-v", f"-I{ROOT / 'include'}", "-c",
                        str(src), "-o", os.devnull], capture_output=True, text=True)
    return r.stdout + r.stderr


def build_all(verbose=False):
    build_harness()
    build_product(verbose)
    build_oracle()


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print("built", LIB)
