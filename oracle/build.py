"""Builds the oracle (test infrastructure): the C restatement into
oracle/_lib/libkutta_oracle.so and, when the reference sources are present on
this machine, the reference's own CPU path into oracle/_ref/ (build_ref.sh)."""
from __future__ import annotations

import hashlib
import os
import pathlib
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_lib"
REFERENCE = pathlib.Path(os.environ.get("KUTTA_REFERENCE", "/root/reference"))


def build_restatement() -> pathlib.Path | None:
    src = HERE / "kutta_oracle.c"
    if not src.exists():
        return None
    LIB.mkdir(exist_ok=True)
    out = LIB / "libkutta_oracle.so"
    stamp = LIB / "libkutta_oracle.so.stamp"
    digest = hashlib.sha256(src.read_bytes() + (HERE / "kutta_oracle.h").read_bytes()).hexdigest()
    if out.exists() and stamp.exists() and stamp.read_text() == digest:
        return out
    # -ffp-contract=off: no FMA contraction, as the reference's CPU build.
    cmd = ["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
           "-Wall", "-Wextra", str(src), "-o", str(out), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    stamp.write_text(digest)
    return out


def build_reference() -> None:
    if (REFERENCE / "src" / "kutta" / "linalg").is_dir():
        subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True)


def build() -> None:
    build_restatement()
    build_reference()


if __name__ == "__main__":
    build()
