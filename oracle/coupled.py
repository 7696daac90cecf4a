"""Test infrastructure only: a numpy restatement of the reference's Coupled
(4x4-block) row kernels, src/kutta/kernels/fv_coupled.kern.h, in float32
with the reference's operation order (numpy's float32 elementwise operations
round exactly like the reference's CPU build, which contracts nothing), so its
results are bit-exact. Vectors are planes [u | v | w | p~] of n floats, as
the reference stores them.

Pinned against the reference itself by tests/test_coupled.py: the edge cache
it rebuilds equals the one the reference's kernels wrote, and the residual of
the reference's returned solution reproduces the reference's final residual.
The product never imports this module.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def _rows(offsets):
    counts = np.diff(offsets)
    return counts, int(counts.max()) if len(counts) else 0


def share(weight, i, c):
    """fv_coupled.kern.h:86-91 (coupled_share)."""
    return weight[c] / np.maximum(weight[i] + weight[c], f32(1e-30))


def fine_coefficients(m: dict, cell, mu, mass, weight, wc):
    """fv_coupled.kern.h:229-256: the five directed-edge planes [a | gx | gy |
    gz | h] per cell-face entry (boundary entries untouched, zero here)."""
    n = int(m["sizes"][0])
    offsets, faces, adjacent, sign = m["cell_face_offsets"], m["cell_faces"], m["adjacent"], \
        m["cell_face_sign"]
    entries = len(faces)
    wc = f32(wc)
    edge = np.zeros(5 * entries, f32)
    rows = np.repeat(np.arange(n), np.diff(offsets))
    q = [wc * cell[k * n + rows] for k in range(10, 19)]
    half = f32(0.5) * wc
    inner = adjacent >= 0
    f = faces
    s = sign
    a = -mu[f] * m["diffusion"][f] + np.minimum(s * mass[f], f32(0))
    bx, by, bz = half * s * m["area_x"][f], half * s * m["area_y"][f], half * s * m["area_z"][f]
    dx, dy, dz = m["lsq_x"], m["lsq_y"], m["lsq_z"]
    gx = bx + q[0] * dx + q[1] * dy + q[2] * dz
    gy = by + q[3] * dx + q[4] * dy + q[5] * dz
    gz = bz + q[6] * dx + q[7] * dy + q[8] * dz
    c = np.where(inner, adjacent, 0)
    h = wc * s * share(weight, rows, c)
    for k, plane in enumerate((a, gx, gy, gz, h)):
        edge[k * entries:(k + 1) * entries] = np.where(inner, plane, f32(0))
    return edge


def fine_row(m: dict, cell, edge, coefficient, x, wc):
    """(J x) of the fine level, fv_coupled.kern.h:258-278, as 4 planes."""
    n = int(m["sizes"][0])
    offsets, faces, adjacent = m["cell_face_offsets"], m["cell_faces"], m["adjacent"]
    entries = len(faces)
    wc = f32(wc)
    xu, xv, xw, xp = (x[k * n:(k + 1) * n] for k in range(4))
    ex, ey, ez = (wc * cell[k * n:(k + 1) * n] for k in (4, 5, 6))
    hx, hy, hz = (wc * cell[k * n:(k + 1) * n] for k in (7, 8, 9))
    yu = cell[:n] * xu + ex * xp
    yv = cell[n:2 * n] * xv + ey * xp
    yw = cell[2 * n:3 * n] * xw + ez * xp
    yp = cell[3 * n:4 * n] * xp + hx * xu + hy * xv + hz * xw
    counts, width = _rows(offsets)
    sx, sy, sz = m["area_x"], m["area_y"], m["area_z"]
    for k in range(width):
        i = np.nonzero(counts > k)[0]
        j = offsets[i] + k
        c = adjacent[j]
        keep = c >= 0
        i, j, c = i[keep], j[keep], c[keep]
        f = faces[j]
        a, gx, gy, gz, h = (edge[p * entries + j] for p in range(5))
        pu, pv, pw, pp = xu[c], xv[c], xw[c], xp[c]
        yu[i] = yu[i] + (a * pu + gx * pp)
        yv[i] = yv[i] + (a * pv + gy * pp)
        yw[i] = yw[i] + (a * pw + gz * pp)
        yp[i] = yp[i] + (h * (sx[f] * pu + sy[f] * pv + sz[f] * pw) - coefficient[f] * pp)
    return np.concatenate([yu, yv, yw, yp])


def fine_residual(m, cell, edge, coefficient, x, b, wc):
    return (b - fine_row(m, cell, edge, coefficient, x, wc)).astype(f32)


def block_solve(r, ex, ey, ez, cache, n, base):
    """fv_coupled.kern.h:61-66 with the block inverse planes base..base+6."""
    ru, rv, rw, rp = (r[k * n:(k + 1) * n] for k in range(4))
    iu, iv, iw, hu, hv, hw, schur = (cache[(base + k) * n:(base + k + 1) * n] for k in range(7))
    p = (rp - hu * ru - hv * rv - hw * rw) / schur
    return np.concatenate([iu * (ru - ex * p), iv * (rv - ey * p), iw * (rw - ez * p), p])


def fine_smooth(m, cell, edge, coefficient, x, b, wc, omega, first):
    """fv_coupled.kern.h:294-309 (coupled_fine_smooth)."""
    n = int(m["sizes"][0])
    wcf = f32(wc)
    r = b.copy()
    base = np.zeros(4 * n, f32)
    if not first:
        r = b - fine_row(m, cell, edge, coefficient, x, wc)
        base = x
    ex, ey, ez = (wcf * cell[k * n:(k + 1) * n] for k in (4, 5, 6))
    d = block_solve(r, ex, ey, ez, cell, n, 20)
    return (base + f32(omega) * d).astype(f32)


def coarse_row(level: dict, x):
    """fv_coupled.kern.h:376-392 (coupled_coarse_row), as 4 planes."""
    rows, cols, diag = level["rows"], level["cols"], level["diag"]
    a, c, g, h, d = level["a"], level["c"], level["g"], level["h"], level["d"]
    n, nnz = len(diag), len(cols)
    xu, xv, xw, xp = (x[k * n:(k + 1) * n] for k in range(4))
    k = diag
    yu = d[:n] * xu + g[k] * xp
    yv = d[n:2 * n] * xv + g[nnz + k] * xp
    yw = d[2 * n:3 * n] * xw + g[2 * nnz + k] * xp
    yp = c[k] * xp + h[k] * xu + h[nnz + k] * xv + h[2 * nnz + k] * xw
    counts, width = _rows(rows)
    for s in range(width):
        i = np.nonzero(counts > s)[0]
        j = rows[i] + s
        keep = j != diag[i]
        i, j = i[keep], j[keep]
        mm = cols[j]
        pu, pv, pw, pp = xu[mm], xv[mm], xw[mm], xp[mm]
        yu[i] = yu[i] + (a[j] * pu + g[j] * pp)
        yv[i] = yv[i] + (a[j] * pv + g[nnz + j] * pp)
        yw[i] = yw[i] + (a[j] * pw + g[2 * nnz + j] * pp)
        yp[i] = yp[i] + (h[j] * pu + h[nnz + j] * pv + h[2 * nnz + j] * pw + c[j] * pp)
    return np.concatenate([yu, yv, yw, yp])


def coarse_smooth(level: dict, x, b, omega, first):
    """fv_coupled.kern.h:401-416 (coupled_coarse_smooth)."""
    n, nnz = len(level["diag"]), len(level["cols"])
    g, k = level["g"], level["diag"]
    r = b.copy()
    base = np.zeros(4 * n, f32)
    if not first:
        r = b - coarse_row(level, x)
        base = x
    s = block_solve(r, g[k], g[nnz + k], g[2 * nnz + k], level["d"], n, 4)
    return (base + f32(omega) * s).astype(f32)


def restrict(offsets, members, fine, nf):
    """fv_coupled.kern.h:554-561: member-order float sums per component."""
    nc = len(offsets) - 1
    out = np.zeros(4 * nc, f32)
    counts, width = _rows(offsets)
    for comp in range(4):
        acc = np.zeros(nc, f32)
        for s in range(width):
            i = np.nonzero(counts > s)[0]
            acc[i] = acc[i] + fine[comp * nf + members[offsets[i] + s]]
        out[comp * nc:(comp + 1) * nc] = acc
    return out


def pair_add(hi, lo, d, slack):
    """prelude.h:139-149 (kpair_add), elementwise."""
    hi, lo, d = (np.asarray(v, f32) for v in (hi, lo, d))
    low = lo + d
    keep = np.abs(low) <= f32(slack)
    s = hi + d
    part = s - hi
    e = (hi - (s - part)) + (d - part)
    t = e + lo
    out_hi = s + t
    part2 = out_hi - s
    out_lo = (s - (out_hi - part2)) + (t - part2)
    return np.where(keep, hi, out_hi).astype(f32), np.where(keep, low, out_lo).astype(f32)
