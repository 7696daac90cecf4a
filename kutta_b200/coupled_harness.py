"""Synthetic inputs for the Coupled 4x4-block solve: the per-solve flow fields
a pseudo-transient Coupled step hands the block solver
(src/kutta/fv/steady_solver.cpp:1268-1294), made on a given mesh.

A mesh is a dict of the device-mesh, stencil and least-squares arrays by name
(`sizes`, `owner`, `neighbour`, `area_x`.., `face_area`, `cell_centroid`,
`cell_face_offsets`, `cell_faces`, `cell_face_sign`, `adjacent`, `diffusion`,
`pattern_row_ptr` / `_col` / `_diag`, `lsq_x`.., `boundary_delta_x`..,
`lsq_inverse`, `owner_to_face_x`.., `neighbour_to_face_x`.., `volume`,
`boundary_kind`), as the reference builds them for a box
(src/kutta/fv/device_mesh.cpp, src/kutta/fv/operators.cpp:43-90) and as
`box_hex` below builds them for a structured hex box without the reference.

The fields follow the steady solver's assembly in form, with seeded values:
a swirling velocity field, its face mass fluxes, an effective viscosity that
varies over three decades, upwind momentum rows over the stencil pattern
(off-diagonal -mu_f D_f + min(s F_f, 0), fv_coupled.kern.h:9), their
physical diagonals (plus a pseudo-time term in the assembled diagonal),
momentum residuals, and the floored physical diagonal as the face-velocity
weights. They are not a converged flow; they are the same kind of inputs.
"""
from __future__ import annotations

import numpy as np

WALL, INLET, OUTLET, SYMMETRY, OUTLET_NORMAL = 0, 1, 2, 3, 4


def flow_fields(mesh: dict, seed: int = 1, *, density: float = 1.2, speed: float = 10.0,
                viscosity: float = 1e-3, pseudo_time: float = 1.0, reference: int = -1) -> dict:
    n, nf, ni = (int(v) for v in mesh["sizes"][:3])
    rng = np.random.default_rng(seed)
    owner = mesh["owner"].astype(np.int64)
    neighbour = mesh["neighbour"].astype(np.int64)
    kind = mesh["boundary_kind"]
    c = mesh["cell_centroid"].reshape(n, 3)
    S = mesh["face_area"].reshape(nf, 3)
    lo, hi = c.min(0), c.max(0)
    t = (c - lo) / np.maximum(hi - lo, 1e-30)
    two_pi = 2 * np.pi
    u = speed * (1 + 0.3 * np.sin(two_pi * t[:, 1]) * np.sin(two_pi * t[:, 2]))
    v = 0.1 * speed * np.sin(two_pi * t[:, 0]) * np.cos(two_pi * t[:, 2])
    w = 0.1 * speed * np.cos(two_pi * t[:, 0]) * np.sin(two_pi * t[:, 1])
    vel = np.stack([u, v, w], 1) * (1 + 0.05 * rng.standard_normal((n, 1)))
    # Face velocities: the mean across internal faces, the owner's at outlets,
    # the free stream at inlets, none at walls and symmetry planes.
    face_vel = np.zeros((nf, 3))
    face_vel[:ni] = 0.5 * (vel[owner[:ni]] + vel[neighbour])
    b_owner = owner[ni:]
    face_vel[ni:] = np.where(np.isin(kind, (OUTLET, OUTLET_NORMAL))[:, None], vel[b_owner], 0.0)
    face_vel[ni:][kind == INLET] = (speed, 0.0, 0.0)
    mass = density * np.einsum("fk,fk->f", face_vel, S)
    mu = viscosity * np.exp(1.2 * rng.standard_normal(nf))
    D = mesh["diffusion"].astype(np.float64)
    mass32 = mass.astype(np.float32)
    mu32 = mu.astype(np.float32)
    # Upwind momentum rows: the off-diagonal of row i toward j over face f is
    # -mu_f D_f + min(s F_f, 0) with s = +1 out of i; the physical diagonal sums
    # mu_f D_f + max(s F_f, 0) over internal faces, mu_f D_f at walls and
    # inlets and the outflow at outlets.
    m_d = (mu32.astype(np.float64) * D)
    rows = mesh["pattern_row_ptr"]
    cols = mesh["pattern_col"]
    diag = mesh["pattern_diag"]
    nnz = len(cols)
    off = np.zeros(nnz)
    a_p = np.zeros(n)

    # Entry of (row, col): the pattern is sorted by row, then column, so the
    # keys row * n + col are sorted too.
    keys = np.repeat(np.arange(n, dtype=np.int64), np.diff(rows)) * n + cols
    i, j = owner[:ni], neighbour
    F = mass32[:ni].astype(np.float64)
    np.add.at(off, np.searchsorted(keys, i * n + j), -m_d[:ni] + np.minimum(F, 0.0))
    np.add.at(off, np.searchsorted(keys, j * n + i), -m_d[:ni] + np.minimum(-F, 0.0))
    np.add.at(a_p, i, m_d[:ni] + np.maximum(F, 0.0))
    np.add.at(a_p, j, m_d[:ni] + np.maximum(-F, 0.0))
    bd = np.where(np.isin(kind, (WALL, INLET)), m_d[ni:], 0.0) + \
        np.where(np.isin(kind, (OUTLET, OUTLET_NORMAL)), np.maximum(mass[ni:], 0.0), 0.0)
    np.add.at(a_p, b_owner, bd)
    volume = mesh["volume"].astype(np.float64)
    length = float(np.cbrt(volume.sum()))
    dt = pseudo_time * length / speed
    fields = {}
    physical = []
    for k in range(3):
        phys = a_p * (1 + 0.05 * k)
        vals = off.copy()
        vals[diag] = phys + density * volume / dt
        fields["momentum_" + "uvw"[k]] = vals.astype(np.float32)
        fields["physical_" + "uvw"[k]] = phys.astype(np.float32)
        physical.append(phys)
    # The floored physical diagonal (coupled_floor_physical): at least the
    # off-diagonal magnitude sum of the shared momentum rows.
    off32 = fields["momentum_u"].copy()
    off32[diag] = 0
    off_sum = np.add.reduceat(np.abs(off32.astype(np.float64)), rows[:-1]) if n else np.zeros(0)
    off_sum = np.where(np.diff(rows) > 0, off_sum, 0.0)
    floored = np.maximum(physical[0], off_sum).astype(np.float32)
    scale = 0.01 * speed * a_p
    for k, name in enumerate(("ru", "rv", "rw")):
        fields[name] = (scale * (np.sin(two_pi * (t[:, k] + 0.1 * k)) +
                                 0.3 * rng.standard_normal(n))).astype(np.float32)
    fields.update(mass=mass32, viscosity=mu32, physical_diagonal=floored,
                  face_weights=floored.copy(), net_outflow=None, density=density,
                  velocity_scale=speed, reference=reference)
    return fields


def box_hex(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
            patch_kinds=(INLET, OUTLET, WALL, WALL, SYMMETRY, SYMMETRY)) -> dict:
    """A structured hex box [lo, hi] with nx x ny x nz cells and the arrays a
    Coupled solve reads, in the reference's conventions for such a box
    (src/kutta/io/generators.cpp make_box_hex, src/kutta/fv/device_mesh.cpp,
    src/kutta/fv/operators.cpp:43-90): cell i + nx (j + ny k); internal faces
    sorted by (owner, neighbour); boundary faces by patch (xmin, xmax, ymin,
    ymax, zmin, zmax), each in cell order; each cell's faces in face order;
    least-squares rows d / |d|^2 toward the neighbour centroid or the boundary
    face centroid, with every boundary face observed at its centroid (on a box
    the normal foot of the cell centroid is the face centroid)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    dims = np.array([nx, ny, nz])
    h = (hi - lo) / dims
    n = int(nx * ny * nz)
    cells = np.arange(n, dtype=np.int64)
    ijk = np.stack([cells % nx, (cells // nx) % ny, cells // (nx * ny)], 1)
    centroid = lo + (ijk + 0.5) * h
    strides = np.array([1, nx, nx * ny])
    face_area_axis = np.array([h[1] * h[2], h[0] * h[2], h[0] * h[1]])
    # Internal faces, sorted by (owner, neighbour).
    own, nei, axis = [], [], []
    for a in range(3):
        c = cells[ijk[:, a] < dims[a] - 1]
        own.append(c)
        nei.append(c + strides[a])
        axis.append(np.full(len(c), a))
    own, nei, axis = (np.concatenate(v) for v in (own, nei, axis))
    order = np.argsort(own * n + nei, kind="stable")
    own, nei, axis = own[order], nei[order], axis[order]
    ni = len(own)
    # Boundary faces by patch, each in cell order.
    b_owner, b_axis, b_side, b_kind = [], [], [], []
    for a in range(3):
        for side, at in ((-1, 0), (1, dims[a] - 1)):
            c = cells[ijk[:, a] == at]
            b_owner.append(c)
            b_axis.append(np.full(len(c), a))
            b_side.append(np.full(len(c), side))
            b_kind.append(np.full(len(c), patch_kinds[2 * a + (side > 0)]))
    b_owner, b_axis, b_side, b_kind = (np.concatenate(v) for v in (b_owner, b_axis, b_side,
                                                                   b_kind))
    nb = len(b_owner)
    nf = ni + nb
    owner = np.concatenate([own, b_owner])
    f_axis = np.concatenate([axis, b_axis])
    sign_b = np.concatenate([np.ones(ni), b_side])
    S = np.zeros((nf, 3))
    S[np.arange(nf), f_axis] = face_area_axis[f_axis] * sign_b
    fc = np.empty((nf, 3))
    fc[:ni] = 0.5 * (centroid[own] + centroid[nei])
    fc[ni:] = centroid[b_owner]
    fc[ni + np.arange(nb), b_axis] += 0.5 * h[b_axis] * b_side
    # Cell-face entries: each cell's faces in face order.
    e_cell = np.concatenate([own, nei, b_owner])
    e_face = np.concatenate([np.arange(ni), np.arange(ni), ni + np.arange(nb)])
    e_sign = np.concatenate([np.ones(ni), -np.ones(ni), np.ones(nb)])
    order = np.argsort(e_cell * nf + e_face, kind="stable")
    e_cell, e_face, e_sign = e_cell[order], e_face[order], e_sign[order]
    offsets = np.zeros(n + 1, np.int64)
    np.add.at(offsets, e_cell + 1, 1)
    offsets = np.cumsum(offsets)
    internal = e_face < ni
    other = np.where(internal, np.where(owner[e_face] == e_cell,
                                        np.concatenate([nei, np.zeros(nb, np.int64)])[e_face],
                                        owner[e_face]), -1)
    adjacent = np.where(internal, other, -(e_face - ni + 1))
    target = np.where(internal[:, None], centroid[np.maximum(other, 0)], fc[e_face])
    d = target - centroid[e_cell]
    w = 1.0 / np.einsum("ek,ek->e", d, d)
    rows = d * w[:, None]
    m = np.zeros((n, 6))
    for k, (p, q) in enumerate(((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        np.add.at(m[:, k], e_cell, w * d[:, p] * d[:, q])
    a = m.T
    det = a[0] * (a[3] * a[5] - a[4] * a[4]) - a[1] * (a[1] * a[5] - a[4] * a[2]) + \
        a[2] * (a[1] * a[4] - a[3] * a[2])
    inverse = np.stack([(a[3] * a[5] - a[4] * a[4]) / det, (a[2] * a[4] - a[1] * a[5]) / det,
                        (a[1] * a[4] - a[2] * a[3]) / det, (a[0] * a[5] - a[2] * a[2]) / det,
                        (a[1] * a[2] - a[0] * a[4]) / det, (a[0] * a[3] - a[1] * a[1]) / det])
    dfc = np.empty((nf, 3))
    dfc[:ni] = centroid[nei] - centroid[own]
    dfc[ni:] = fc[ni:] - centroid[b_owner]
    diffusion = np.einsum("fk,fk->f", S, S) / np.einsum("fk,fk->f", S, dfc)
    bd = dfc[ni:] / np.einsum("fk,fk->f", dfc[ni:], dfc[ni:])[:, None]
    otf = fc - centroid[owner]
    ntf = fc[:ni] - centroid[nei]
    # The stencil pattern: each cell's face neighbours and itself, sorted.
    p_cell = np.concatenate([own, nei, cells])
    p_col = np.concatenate([nei, own, cells])
    order = np.argsort(p_cell * n + p_col, kind="stable")
    p_cell, p_col = p_cell[order], p_col[order]
    p_rows = np.zeros(n + 1, np.int64)
    np.add.at(p_rows, p_cell + 1, 1)
    p_rows = np.cumsum(p_rows)
    p_diag = np.nonzero(p_col == p_cell)[0]
    f32, i32 = np.float32, np.int32
    return {
        "sizes": np.array([n, nf, ni, len(e_cell), len(p_col)], i32),
        "owner": owner.astype(i32), "neighbour": nei.astype(i32),
        "area_x": S[:, 0].astype(f32), "area_y": S[:, 1].astype(f32),
        "area_z": S[:, 2].astype(f32), "face_area": S.reshape(-1),
        "cell_centroid": centroid.reshape(-1),
        "cell_face_offsets": offsets.astype(i32), "cell_faces": e_face.astype(i32),
        "cell_face_sign": e_sign.astype(f32), "adjacent": adjacent.astype(i32),
        "diffusion": diffusion.astype(f32),
        "pattern_row_ptr": p_rows.astype(i32), "pattern_col": p_col.astype(i32),
        "pattern_diag": p_diag.astype(i32),
        "lsq_x": rows[:, 0].astype(f32), "lsq_y": rows[:, 1].astype(f32),
        "lsq_z": rows[:, 2].astype(f32),
        "boundary_delta_x": bd[:, 0].astype(f32), "boundary_delta_y": bd[:, 1].astype(f32),
        "boundary_delta_z": bd[:, 2].astype(f32),
        "lsq_inverse": inverse.reshape(-1).astype(f32),
        "owner_to_face_x": otf[:, 0].astype(f32), "owner_to_face_y": otf[:, 1].astype(f32),
        "owner_to_face_z": otf[:, 2].astype(f32),
        "neighbour_to_face_x": ntf[:, 0].astype(f32), "neighbour_to_face_y": ntf[:, 1].astype(f32),
        "neighbour_to_face_z": ntf[:, 2].astype(f32),
        "volume": np.full(n, np.prod(h), f32), "boundary_kind": b_kind.astype(i32),
    }
