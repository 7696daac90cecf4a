#!/usr/bin/env bash
# Test infrastructure: builds the reference's own CPU solve path from the
# reference sources where they lie (read-only) into oracle/_ref/ (git-ignored),
# together with the shim oracle/ref_shim.cpp, as oracle/_ref/libkutta_ref.so.
#
# Steps (the reference's own generator, then its linalg + serial CPU runtime,
# and for the Coupled block solve its mesh, box generator, device mesh,
# stencil / least-squares operators and fv/coupled_solver.cpp):
#   python3 tools/kernelgen.py  -> oracle/_ref/gen/kernels*.{hpp,cpp}
#   g++ -std=c++20 -O3 -DNDEBUG  src/kutta/linalg/*.cpp runtime/device.cpp
#       runtime/cpu/cpu_device.cpp core/memory.cpp mesh/{mesh,topology,
#       polyhedral}.cpp io/generators.cpp fv/{device_mesh,operators,
#       coupled_solver}.cpp + generated host/cpu tables
# No cmake, no external libraries, nothing written under the reference tree.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${KUTTA_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src/kutta/linalg" ]; then
  echo "build_ref: reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/gen"
K="$REF/src/kutta/kernels"
python3 "$REF/tools/kernelgen.py" --src-root "$REF/src" --out "$OUT/gen" \
  "$K/amg.kern.h" "$K/blas.kern.h" "$K/linalg.kern.h" "$K/scalars.kern.h" "$K/fv_flow.kern.h" \
  "$K/fv_coupled.kern.h" "$K/fv_gradient.kern.h"
SRC=(
  "$REF/src/kutta/linalg/amg.cpp"
  "$REF/src/kutta/linalg/csr.cpp"
  "$REF/src/kutta/linalg/solver.cpp"
  "$REF/src/kutta/runtime/device.cpp"
  "$REF/src/kutta/runtime/cpu/cpu_device.cpp"
  "$REF/src/kutta/core/memory.cpp"
  "$REF/src/kutta/mesh/mesh.cpp"
  "$REF/src/kutta/mesh/topology.cpp"
  "$REF/src/kutta/mesh/polyhedral.cpp"
  "$REF/src/kutta/io/generators.cpp"
  "$REF/src/kutta/fv/device_mesh.cpp"
  "$REF/src/kutta/fv/operators.cpp"
  "$REF/src/kutta/fv/coupled_solver.cpp"
  "$OUT/gen/kernels_host.cpp"
  "$OUT/gen/kernels_cpu.cpp"
  "$HERE/ref_shim.cpp"
  "$HERE/ref_coupled.cpp"
)
STAMP="$OUT/.stamp"
NEWEST=$(stat -c %Y "${SRC[@]}" "$0" "$HERE/ref_watch.hpp" | sort -n | tail -1)
if [ -f "$OUT/libkutta_ref.so" ] && [ -f "$STAMP" ] && [ "$(cat "$STAMP")" = "$NEWEST" ]; then
  exit 0
fi
mkdir -p "$OUT/obj"
pids=()
objs=()
for s in "${SRC[@]}"; do
  o="$OUT/obj/$(basename "$s").o"
  objs+=("$o")
  g++ -std=c++20 -O3 -DNDEBUG -fPIC -I"$REF/src" -I"$OUT/gen" -c "$s" -o "$o" &
  pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
g++ -shared -o "$OUT/libkutta_ref.so" "${objs[@]}"
echo "$NEWEST" > "$STAMP"
echo "build_ref: built $OUT/libkutta_ref.so"
