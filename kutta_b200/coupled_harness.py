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
`box_hex` / `box_tet` below build them, bit for bit, for a structured hex box and
its six-tet split without the reference.

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


def _mesh_arrays(centroid, volume, owner, neighbour, S, fc, b_kind) -> dict:
    """The device-mesh, stencil and pressure least-squares arrays of a mesh
    given by its cells (centroids, volumes) and faces (owner for every face,
    neighbour for the internal ones, which come first; area vectors out of
    the owner; centroids; the kind of each boundary face), in the reference's
    conventions (src/kutta/fv/device_mesh.cpp, src/kutta/fv/operators.cpp):
    each cell's faces in face order; least-squares rows d / |d|^2 toward the
    neighbour centroid or the boundary face centroid (make_stencil); the
    pressure fit observes pressure-specified faces at their centroid and every
    other boundary face at the normal foot of the cell centroid
    (operators.cpp cell_fit, steady_solver.cpp:348-356)."""
    n = len(centroid)
    ni = len(neighbour)
    nf = len(owner)
    nb = nf - ni
    b_owner = owner[ni:]
    # Cell-face entries: each cell's faces in face order.
    e_cell = np.concatenate([owner[:ni], neighbour, b_owner])
    e_face = np.concatenate([np.arange(ni), np.arange(ni), ni + np.arange(nb)])
    e_sign = np.concatenate([np.ones(ni), -np.ones(ni), np.ones(nb)])
    order = np.argsort(e_cell * nf + e_face, kind="stable")
    e_cell, e_face, e_sign = e_cell[order], e_face[order], e_sign[order]
    offsets = np.zeros(n + 1, np.int64)
    np.add.at(offsets, e_cell + 1, 1)
    offsets = np.cumsum(offsets)
    internal = e_face < ni
    nei_full = np.concatenate([neighbour, np.zeros(nb, np.int64)])
    other = np.where(internal, np.where(owner[e_face] == e_cell, nei_full[e_face],
                                        owner[e_face]), -1)
    adjacent = np.where(internal, other, -(e_face - ni + 1))
    target = np.where(internal[:, None], centroid[np.maximum(other, 0)], fc[e_face])
    d = target - centroid[e_cell]
    w = 1.0 / np.einsum("ek,ek->e", d, d)
    rows = d * w[:, None]
    # The pressure fit's boundary observations.
    db = fc[ni:] - centroid[b_owner]
    prescribed = np.isin(b_kind, (OUTLET, OUTLET_NORMAL))
    sb = S[ni:]
    foot = sb * (np.einsum("bk,bk->b", db, sb) / np.einsum("bk,bk->b", sb, sb))[:, None]
    db = np.where(prescribed[:, None], db, foot)
    wb = 1.0 / np.einsum("bk,bk->b", db, db)
    bd = db * wb[:, None]
    m = np.zeros((n, 6))
    ci, di, wi = e_cell[internal], d[internal], w[internal]
    for k, (p, q) in enumerate(((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        np.add.at(m[:, k], ci, wi * di[:, p] * di[:, q])
        np.add.at(m[:, k], b_owner, wb * db[:, p] * db[:, q])
    a = m.T
    det = a[0] * (a[3] * a[5] - a[4] * a[4]) - a[1] * (a[1] * a[5] - a[4] * a[2]) + \
        a[2] * (a[1] * a[4] - a[3] * a[2])
    inverse = np.stack([(a[3] * a[5] - a[4] * a[4]) / det, (a[2] * a[4] - a[1] * a[5]) / det,
                        (a[1] * a[4] - a[2] * a[3]) / det, (a[0] * a[5] - a[2] * a[2]) / det,
                        (a[1] * a[2] - a[0] * a[4]) / det, (a[0] * a[3] - a[1] * a[1]) / det])
    dfc = np.empty((nf, 3))
    dfc[:ni] = centroid[neighbour] - centroid[owner[:ni]]
    dfc[ni:] = fc[ni:] - centroid[b_owner]
    diffusion = np.einsum("fk,fk->f", S, S) / np.einsum("fk,fk->f", S, dfc)
    otf = fc - centroid[owner]
    ntf = fc[:ni] - centroid[neighbour]
    # The stencil pattern: each cell's face neighbours and itself, sorted.
    cells = np.arange(n, dtype=np.int64)
    p_cell = np.concatenate([owner[:ni], neighbour, cells])
    p_col = np.concatenate([neighbour, owner[:ni], cells])
    order = np.argsort(p_cell * n + p_col, kind="stable")
    p_cell, p_col = p_cell[order], p_col[order]
    p_rows = np.zeros(n + 1, np.int64)
    np.add.at(p_rows, p_cell + 1, 1)
    p_rows = np.cumsum(p_rows)
    p_diag = np.nonzero(p_col == p_cell)[0]
    f32, i32 = np.float32, np.int32
    return {
        "sizes": np.array([n, nf, ni, len(e_cell), len(p_col)], i32),
        "owner": owner.astype(i32), "neighbour": neighbour.astype(i32),
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
        "volume": volume.astype(f32), "boundary_kind": b_kind.astype(i32),
    }


def box_hex(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
            patch_kinds=(INLET, OUTLET, WALL, WALL, SYMMETRY, SYMMETRY)) -> dict:
    """A structured hex box [lo, hi] with nx x ny x nz cells and the arrays a
    Coupled solve reads, as the reference builds them for the same box
    (src/kutta/io/generators.cpp make_box_hex): cell i + nx (j + ny k);
    patches xmin, xmax, ymin, ymax, zmin, zmax with the given kinds."""
    return _box(nx, ny, nz, lo, hi, patch_kinds, tet=False)


def box_tet(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
            patch_kinds=(INLET, OUTLET, WALL, WALL, SYMMETRY, SYMMETRY)) -> dict:
    """The same box split into six tets per hex around its (0,0,0)-(1,1,1)
    diagonal (generators.cpp make_box_tet): cell 6 (hex index) + t."""
    return _box(nx, ny, nz, lo, hi, patch_kinds, tet=True)


def _box(nx, ny, nz, lo, hi, patch_kinds, tet):
    """The box's cells as the generator lists them, then the reference's
    face construction (src/kutta/mesh/topology.cpp from_cells and pack):
    faces numbered by first appearance over the cells' local faces, stored
    with the first cell's node order, reversed where its normal points into
    that cell; the lower cell owns an internal face; internal faces sorted by
    (owner, neighbour), boundary faces by patch (the first box side all the
    face's nodes lie on), each in order of first appearance. The geometry
    follows in the reference's double operations (`_face_geometry`,
    `_cell_geometry`), so the arrays are the reference's bit for bit, the
    least-squares inverse aside (the reference inverts by a Jacobi
    eigensolve; the two agree to double round-off)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    dims = np.array([nx, ny, nz])
    hexes = np.arange(int(nx * ny * nz), dtype=np.int64)
    i, j, k = hexes % nx, (hexes // nx) % ny, hexes // (nx * ny)

    def node(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    v = np.stack([node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k),
                  node(i, j, k + 1), node(i + 1, j, k + 1), node(i + 1, j + 1, k + 1),
                  node(i, j + 1, k + 1)], 1)
    if tet:
        ring = (1, 2, 3, 7, 4, 5)
        cells = np.stack([np.stack([v[:, 0], v[:, ring[t]], v[:, ring[(t + 1) % 6]], v[:, 6]], 1)
                          for t in range(6)], 1).reshape(-1, 4)
        local = [[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]]
    else:
        cells = v
        local = [[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6],
                 [3, 0, 4, 7]]
    n = len(cells)
    npts = (nx + 1) * (ny + 1) * (nz + 1)
    pid = np.arange(npts, dtype=np.int64)
    pijk = np.stack([pid % (nx + 1), (pid // (nx + 1)) % (ny + 1),
                     pid // ((nx + 1) * (ny + 1))], 1)
    points = lo + (hi - lo) * pijk / dims
    # Every cell's local faces; occurrence (local faces) cell + local face.
    occ = cells[:, local].reshape(-1, len(local[0]))
    per_cell = len(local)
    cell_mid = np.zeros((n, 3))
    for c in range(cells.shape[1]):
        cell_mid += points[cells[:, c]]
    cell_mid /= cells.shape[1]
    del cells
    srt = np.sort(occ, axis=1)
    key_hi = srt[:, 0] * npts + srt[:, 1]
    key_lo = srt[:, 2] * npts + (srt[:, 3] if srt.shape[1] > 3 else 0)
    del srt
    order = np.lexsort((key_lo, key_hi))  # stable: each key's first occurrence leads
    ks_hi, ks_lo = key_hi[order], key_lo[order]
    del key_hi, key_lo
    lead = np.ones(len(order), bool)
    lead[1:] = (ks_hi[1:] != ks_hi[:-1]) | (ks_lo[1:] != ks_lo[:-1])
    del ks_hi, ks_lo
    first = order[lead]
    group = np.cumsum(lead) - 1
    owner_f = first // per_cell
    second = np.full(len(first), -1, np.int64)
    repeat = ~lead
    second[group[repeat]] = order[repeat] // per_cell
    del order, lead, group, repeat
    # Stored node order: the first cell's, reversed where the polygon's normal
    # points into that cell (the sign needs no exact doubles).
    ns = occ[first]
    del occ
    corners = points[ns]
    normal = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    inward = np.einsum("fk,fk->f", normal, corners.mean(axis=1) - cell_mid[owner_f]) < 0
    del corners, normal
    ns[inward] = ns[inward, ::-1]
    internal = second >= 0
    nijk = pijk[ns]
    patch = np.full(len(first), -1)
    for side in range(6):
        axis = side // 2
        at = 0 if side % 2 == 0 else dims[axis]
        on = np.all(nijk[:, :, axis] == at, axis=1) & ~internal & (patch < 0)
        patch[on] = side
    del nijk
    ii = np.nonzero(internal)[0]
    ii = ii[np.lexsort((second[ii], owner_f[ii]))]
    bb = np.nonzero(~internal)[0]
    bb = bb[np.lexsort((first[bb], patch[bb]))]
    order = np.concatenate([ii, bb])
    owner, neighbour = owner_f[order], second[ii]
    fc, area = _face_geometry(points[ns[order]])
    centroid, volume = _cell_geometry(fc, area, owner, neighbour, n)
    b_kind = np.asarray(patch_kinds)[patch[bb]]
    return _mesh_arrays(centroid, volume, owner, neighbour, area, fc, b_kind)


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def _face_geometry(corners):
    """Centroid and area vector of each polygon (faces x nodes x 3), in the
    reference's double operations and their order (src/kutta/mesh/mesh.cpp
    face_geometry, src/kutta/mesh/detail.hpp face_center): the node mean
    about the first node; the area vector as the fan of half cross products
    about it; the centroid as the fan triangles' moments weighted by their
    areas projected on the unit normal. A division by s is a product with
    1 / s, as there."""
    k = corners.shape[1]
    origin = corners[:, 0]
    d = np.zeros_like(origin)
    for j in range(k):
        d = d + (corners[:, j] - origin)
    center = origin + d * (1 / float(k))
    av = np.zeros_like(origin)
    for j in range(k):
        av = av + _cross(corners[:, j] - center, corners[:, (j + 1) % k] - center) * 0.5
    normal = av * (1 / np.sqrt(_dot(av, av)))[:, None]
    area = np.zeros(len(origin))
    moment = np.zeros_like(origin)
    for j in range(k):
        a, b = corners[:, j] - center, corners[:, (j + 1) % k] - center
        w = _dot(_cross(a, b) * 0.5, normal)
        area = area + w
        moment = moment + (a + b) * (w / 3)[:, None]
    return center + moment * (1 / area)[:, None], av


def _cell_geometry(fc, area, owner, neighbour, n):
    """Cell centroids and volumes from the face centroids and area vectors, in
    the reference's double operations and their order (src/kutta/mesh/mesh.cpp
    cell_geometry): a first estimate, the mean of the cell's face centroids
    about its first; then one pyramid per face from that estimate, with volume
    (sign) S.r / 3 and centroid 3/4 of the way to the face, each cell summed
    in face order."""
    ni = len(neighbour)
    e_cell = np.concatenate([owner[:ni], neighbour, owner[ni:]])
    e_face = np.concatenate([np.arange(ni), np.arange(ni), np.arange(ni, len(owner))])
    e_sign = np.concatenate([np.ones(ni), -np.ones(ni), np.ones(len(owner) - ni)])
    order = np.lexsort((e_face, e_cell))
    e_cell, e_face, e_sign = e_cell[order], e_face[order], e_sign[order]
    start = np.searchsorted(e_cell, np.arange(n + 1))
    count = np.diff(start)
    anchor = fc[e_face[start[:-1]]]
    estimate = np.zeros((n, 3))
    for k in range(int(count.max())):
        c = np.nonzero(count > k)[0]
        estimate[c] = estimate[c] + (fc[e_face[start[c] + k]] - anchor[c])
    estimate = anchor + estimate * (1 / count.astype(np.float64))[:, None]
    volume = np.zeros(n)
    centroid = np.zeros((n, 3))
    for k in range(int(count.max())):
        c = np.nonzero(count > k)[0]
        e = start[c] + k
        r = fc[e_face[e]] - estimate[c]
        v = e_sign[e] * _dot(area[e_face[e]], r) / 3
        volume[c] = volume[c] + v
        centroid[c] = centroid[c] + r * (0.75 * v)[:, None]
    return estimate + centroid * (1 / volume)[:, None], volume
