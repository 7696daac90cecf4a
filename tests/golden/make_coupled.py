"""Coupled (4x4-block) solve fixtures, with the reference's own results.

For each case the reference built from its sources (oracle/_ref,
oracle/ref_coupled.cpp) generates a box mesh (make_box_hex / make_box_tet),
its geometry, device mesh, stencil and pressure least-squares fit; seeded flow
fields are made on it (kutta_b200/coupled_harness.flow_fields); then the
reference's CoupledSolver is constructed, captures the three momentum
diagonals, solves once and updates zero fields. Each fixture stores the mesh
arrays, the fields, and what the reference's kernels saw and wrote: the packed
27-plane cell data, the face coefficients, the edge cache, the right-hand side,
every coarse level's operator and transfer, the solution, its iterations,
residuals and describe() string.

Needs the reference sources on this machine; the fixtures are committed and the
tests read them without the reference.

    python tests/golden/make_coupled.py [case ...]
"""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from kutta_b200 import coupled_harness as H  # noqa: E402
from oracle import ref  # noqa: E402

OPEN = (H.INLET, H.OUTLET, H.WALL, H.WALL, H.SYMMETRY, H.SYMMETRY)
OPEN_NORMAL = (H.INLET, H.OUTLET_NORMAL, H.WALL, H.SYMMETRY, H.WALL, H.WALL)
CLOSED = (H.WALL,) * 6

# name: (tet, dims, patch kinds, reference cell, seed, options, control, extras)
CASES = {
    "coupled_hex8x6x5_open": (False, (8, 6, 5), OPEN, -1, 1, {}, (0.1, 1e-12, 20), {}),
    "coupled_tet4x4x3_open": (True, (4, 4, 3), OPEN, -1, 2, {}, (0.1, 1e-12, 20), {}),
    "coupled_hex12x10x8_closed": (False, (12, 10, 8), CLOSED, 0, 3, {}, (0.1, 1e-12, 20), {}),
    "coupled_tet6x5x4_tight": (True, (6, 5, 4), OPEN_NORMAL, -1, 4, {}, (1e-4, 1e-12, 200),
                               {}),
    "coupled_hex10x8x6_v22_net": (False, (10, 8, 6), OPEN, -1, 5,
                                  {"pre_sweeps": 2, "post_sweeps": 2, "coarsest_rows": 20,
                                   "recompute": True},
                                  (1e-3, 1e-12, 60), {"net_outflow": True}),
    # Cells flagged with low-order pressure faces (no extrapolation in Q),
    # and the float-pair update on seeded hi/lo fields.
    "coupled_tet5x4x3_loworder_paired": (True, (5, 4, 3), OPEN, -1, 6, {}, (1e-3, 1e-12, 60),
                                         {"low_order": 0.15, "pairs": True}),
}

MESH_KEYS = ("sizes", "owner", "neighbour", "area_x", "area_y", "area_z", "face_area",
             "cell_centroid", "cell_face_offsets", "cell_faces", "cell_face_sign", "adjacent",
             "diffusion", "pattern_row_ptr", "pattern_col", "pattern_diag", "lsq_x", "lsq_y",
             "lsq_z", "boundary_delta_x", "boundary_delta_y", "boundary_delta_z", "lsq_inverse",
             "owner_to_face_x", "owner_to_face_y", "owner_to_face_z", "neighbour_to_face_x",
             "neighbour_to_face_y", "neighbour_to_face_z", "volume", "boundary_kind")
FIELD_KEYS = ("momentum_u", "momentum_v", "momentum_w", "physical_u", "physical_v",
              "physical_w", "ru", "rv", "rw", "mass", "viscosity", "physical_diagonal",
              "face_weights")


def make(name: str) -> None:
    tet, dims, kinds, reference, seed, options, control, extras = CASES[name]
    case = ref.CoupledCase(tet, *dims, patch_kinds=kinds)
    fields = H.flow_fields(case.arrays, seed, reference=reference)
    if extras.get("net_outflow"):
        # The float-pair continuity's net outflow: the mass imbalance with a
        # seeded perturbation, so it differs from the summed mass fluxes.
        rng = np.random.default_rng(seed + 100)
        m = case.arrays
        n = int(m["sizes"][0])
        net = np.zeros(n)
        np.add.at(net, m["owner"], fields["mass"].astype(np.float64))
        np.add.at(net, m["neighbour"], -fields["mass"][: len(m["neighbour"])].astype(np.float64))
        fields["net_outflow"] = (net * (1 + 0.1 * rng.standard_normal(n))).astype(np.float32)
    rel_tol, abs_tol, max_iter = control
    n = int(case.arrays["sizes"][0])
    rng = np.random.default_rng(seed + 200)
    low = None
    if extras.get("low_order"):
        low = (rng.random(n) < extras["low_order"]).astype(np.int32)
    pairs = None
    if extras.get("pairs"):
        hi = (rng.standard_normal(4 * n) * 10).astype(np.float32)
        lo = (rng.standard_normal(4 * n) * 1e-6).astype(np.float32)
        pairs = (hi, lo, 0.7, 0.3, 1e-4, 3e-5)
    out = case.solve(fields, ref.coupled_options(**options), rel_tol=rel_tol, abs_tol=abs_tol,
                     max_iter=max_iter, low_order=low, pairs=pairs)
    arrays = {}
    for k in MESH_KEYS:
        arrays["mesh_" + k] = case.arrays[k]
    for k in FIELD_KEYS:
        arrays["field_" + k] = fields[k]
    if fields.get("net_outflow") is not None:
        arrays["field_net_outflow"] = fields["net_outflow"]
    if low is not None:
        arrays["mesh_low_order"] = low
    if pairs is not None:
        arrays["pair_hi"], arrays["pair_lo"] = pairs[0], pairs[1]
    for k, v in out.items():
        if isinstance(v, np.ndarray) and k not in case.arrays:
            arrays["ref_" + k] = v
    meta = {
        "tet": tet, "dims": dims, "patch_kinds": kinds, "reference": reference, "seed": seed,
        "options": options, "control": control, "density": fields["density"],
        "velocity_scale": fields["velocity_scale"], "iterations": out["iterations"],
        "converged": out["converged"], "initial_residual": out["initial_residual"],
        "final_residual": out["final_residual"], "describe": out["describe"],
        "net_outflow": bool(extras.get("net_outflow")),
        "pairs": list(pairs[2:]) if pairs is not None else None,
    }
    np.savez_compressed(HERE / f"{name}.npz", meta=np.frombuffer(json.dumps(meta).encode(), np.uint8),
                        **arrays)
    print(f"{name}: {out['describe']}; {out['iterations']} iterations, "
          f"{out['initial_residual']:.4e} -> {out['final_residual']:.4e}")


def main(names):
    if not ref.available():
        raise SystemExit("oracle/_ref/libkutta_ref.so is missing: run oracle/build_ref.sh")
    for name in names or CASES:
        make(name)


if __name__ == "__main__":
    main(sys.argv[1:])
