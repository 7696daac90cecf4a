"""Synthetic pressure-correction systems (host side, numpy).

Thin ctypes front end over ``csrc/harness/systems.c``: jittered hex / six-tet box
meshes assembled into the finite-volume pressure M-matrix, the non-symmetric
upwind convection-diffusion twin, and the reference's own linear-algebra test
matrices (``poisson``, tests/linalg/matrices.hpp:17-62 of the reference).

A system is a :class:`HostSystem` holding a host CSR matrix in the reference's
``CsrMatrixHost`` form (int32 ``row_ptr``/``col``/``diag``, float-representable
float64 ``val``) plus a right-hand side.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import pathlib

import numpy as np

_LIB_DIR = pathlib.Path(__file__).resolve().parent / "_lib"


class _KhSystem(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("nnz", ctypes.c_int),
        ("row_ptr", ctypes.POINTER(ctypes.c_int)), ("col", ctypes.POINTER(ctypes.c_int)),
        ("diag", ctypes.POINTER(ctypes.c_int)), ("val", ctypes.POINTER(ctypes.c_double)),
        ("b", ctypes.POINTER(ctypes.c_float)), ("volume", ctypes.POINTER(ctypes.c_double)),
        ("new_to_old", ctypes.POINTER(ctypes.c_int)), ("faces", ctypes.c_int),
        ("centroid", ctypes.POINTER(ctypes.c_double)), ("boundary", ctypes.POINTER(ctypes.c_double)),
        ("geometry", ctypes.POINTER(ctypes.c_double)),
    ]


_lib = None


def _load():
    global _lib
    if _lib is None:
        path = _LIB_DIR / "libkutta_harness.so"
        if not path.exists():
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        lib = ctypes.CDLL(str(path))
        lib.kh_poisson.restype = ctypes.POINTER(_KhSystem)
        lib.kh_poisson.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.kh_box_system.restype = ctypes.POINTER(_KhSystem)
        lib.kh_box_system.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_uint64, ctypes.c_double, ctypes.c_double]
        lib.kh_free.argtypes = [ctypes.POINTER(_KhSystem)]
        lib.kh_hash.restype = ctypes.c_uint32
        lib.kh_hash.argtypes = [ctypes.c_uint32]
        _lib = lib
    return _lib


@dataclasses.dataclass
class HostSystem:
    """Host CSR (the reference's CsrMatrixHost layout) plus a right-hand side."""
    row_ptr: np.ndarray   # int32[n+1]
    col: np.ndarray       # int32[nnz], sorted per row
    diag: np.ndarray      # int32[n], index of (i, i)
    val: np.ndarray       # float64[nnz], float-representable
    b: np.ndarray         # float32[n]
    volume: np.ndarray | None = None
    new_to_old: np.ndarray | None = None
    name: str = ""
    centroid: np.ndarray | None = None   # float64[n, 3] (box meshes)
    boundary: np.ndarray | None = None   # float64[n], Dirichlet term in each diagonal
    geometry: np.ndarray | None = None   # float64[nnz], |A_f| / |c_N - c_P| per off-diagonal

    @property
    def n(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def val32(self) -> np.ndarray:
        return self.val.astype(np.float32)


def _take(ptr) -> HostSystem:
    if not ptr:
        raise ValueError("system generation failed (invalid sizes)")
    s = ptr.contents
    n, nnz = s.n, s.nnz

    def arr(p, count, dtype):
        if count == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(p, shape=(count,)).astype(dtype, copy=True)

    out = HostSystem(
        row_ptr=arr(s.row_ptr, n + 1, np.int32), col=arr(s.col, nnz, np.int32),
        diag=arr(s.diag, n, np.int32), val=arr(s.val, nnz, np.float64),
        b=arr(s.b, n, np.float32), volume=arr(s.volume, n, np.float64),
        new_to_old=arr(s.new_to_old, n, np.int32))
    if s.centroid:
        out.centroid = arr(s.centroid, 3 * n, np.float64).reshape(n, 3)
        out.boundary = arr(s.boundary, n, np.float64)
    if s.geometry:
        out.geometry = arr(s.geometry, nnz, np.float64)
    _load().kh_free(ptr)
    return out


def ref_hash(x: int) -> int:
    """The reference test suite's integer hash (tests/linalg/matrices.hpp:13-15)."""
    return int(_load().kh_hash(ctypes.c_uint32(x & 0xFFFFFFFF)))


def ref_hash_array(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint32)
    x = x ^ (x >> np.uint32(16))
    x = (x * np.uint32(0x7FEB352D)).astype(np.uint32)
    x = x ^ (x >> np.uint32(15))
    x = (x * np.uint32(0x846CA68B)).astype(np.uint32)
    return x ^ (x >> np.uint32(16))


def poisson(nx: int, ny: int, nz: int = 1, anisotropy: float = 1.0, random: bool = False,
            neumann: bool = False, wind: float = 0.0) -> HostSystem:
    """The reference's poisson() test matrix (tests/linalg/matrices.hpp:17-62)."""
    s = _take(_load().kh_poisson(nx, ny, nz, anisotropy, int(random), int(neumann), wind))
    s.name = f"poisson({nx},{ny},{nz},{anisotropy},{int(random)},{int(neumann)},{wind})"
    return s


def random_forcing(n: int, offset: int = 53) -> np.ndarray:
    """b_i = (hash(i + 53) % 2001 - 1000) / 1024 (bench/bench_linalg.cpp:57-58)."""
    h = ref_hash_array(np.arange(n, dtype=np.uint64) + offset).astype(np.int64)
    return ((h % 2001) - 1000).astype(np.float32) / np.float32(1024.0)


def random_solution(n: int) -> np.ndarray:
    """tests/linalg/matrices.hpp:71-75."""
    return random_forcing(n, 19)


def box_system(nx: int, ny: int, nz: int, *, tet: bool, seed: int, jitter: float = 0.15,
               band_layers: int = 0, aspect: float = 1000.0, ratio: float = 1.2,
               dmin: float = 1e-3, dmax: float = 1.0, convection: float = 0.0,
               renumber: bool = True, coeff_seed: int = 0, field_sigma: float = 0.0,
               field_corr: float = 0.1) -> HostSystem:
    """Finite-volume pressure (or convection-diffusion) system on a jittered box.
    `seed` fixes the mesh; a nonzero `coeff_seed` draws the coefficient field
    and right-hand side from a stream of its own (same mesh, another field).
    field_sigma > 0: D = exp(field_sigma g) for a smooth unit-variance Gaussian
    field g of correlation length field_corr, instead of per-cell log-uniform
    D in [dmin, dmax]."""
    s = _take(_load().kh_box_system(nx, ny, nz, int(tet), jitter, band_layers, aspect, ratio,
                                    dmin, dmax, convection, int(renumber), seed, coeff_seed,
                                    field_sigma, field_corr))
    s.name = (f"{'tet6' if tet else 'hex'}{nx}x{ny}x{nz}-seed{seed}"
              + (f"-band{band_layers}" if band_layers else "")
              + (f"-conv{convection}" if convection > 0 else ""))
    return s


# Named workloads -----------------------------------------------------------

def pressure_hex32(seed: int = 1) -> HostSystem:
    """32^3 jittered hex pressure matrix (32,768 cells, 6-face stencil)."""
    return box_system(32, 32, 32, tet=False, seed=seed)


def pressure_tet96(seed: int = 1, n: int = 96) -> HostSystem:
    """96^3 jittered hex mesh, six tets per hex (5,308,416 cells, 4-face stencil)."""
    return box_system(n, n, n, tet=True, seed=seed)


def convection_tet96(seed: int = 1, n: int = 96) -> HostSystem:
    """Non-symmetric upwind convection-diffusion twin (nu = 1e-3, relaxation 0.7)."""
    return box_system(n, n, n, tet=True, seed=seed, convection=1e-3)


def graded_tet96(seed: int = 1, n: int = 96) -> HostSystem:
    """Tet mesh with a 10-layer graded band at z = 0 (ratio 1.2, first aspect 1000:1),
    D_f log-uniform over [1e-6, 1]."""
    return box_system(n, n, n, tet=True, seed=seed, band_layers=10, aspect=1000.0, ratio=1.2,
                      dmin=1e-6, dmax=1.0)

# Finite-volume face data ------------------------------------------------------
# Synthetic inputs of the reference's pressure assembly and correction kernels
# (src/kutta/kernels/fv_flow.kern.h:164-201) for a CSR pattern, laid out as
# src/kutta/fv/steady_solver.cpp passes them: cell-face slots (offsets, faces,
# sign +1 on the owner side, adjacent cell or -1 on the boundary, CSR entry of
# (cell, adjacent)), internal faces first, per-face coefficients and fluxes.
# Each off-diagonal pair (i, j) becomes an internal face (owner i < j); a
# seeded fraction of pairs gets a second face on the same CSR entry (cells
# sharing several faces); a seeded fraction of cells gets boundary faces.
# Coefficients are log-uniform positive, fluxes normal.

@dataclasses.dataclass
class FvCase:
    n: int
    rows: np.ndarray
    cols: np.ndarray
    diag: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray      # internal faces only
    internal: int
    offsets: np.ndarray
    faces: np.ndarray
    sign: np.ndarray
    adjacent: np.ndarray
    entry: np.ndarray
    coefficient: np.ndarray
    flux: np.ndarray
    reference: int = -1

    @property
    def n_faces(self) -> int:
        return len(self.owner)


def fv_faces(row_ptr, col, diag, seed: int, duplicate: float = 0.1, boundary: float = 0.3,
          reference: int = -1) -> FvCase:
    rng = np.random.default_rng(seed)
    n = len(row_ptr) - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    upper = col > rows
    own, nb = rows[upper].astype(np.int32), col[upper].astype(np.int32)
    extra = rng.random(len(own)) < duplicate
    own = np.concatenate([own, own[extra]])
    nb = np.concatenate([nb, nb[extra]])
    internal = len(own)
    bcells = np.nonzero(rng.random(n) < boundary)[0]
    bcells = np.concatenate([bcells, bcells[rng.random(len(bcells)) < 0.3]])  # some with two
    owner = np.concatenate([own, np.sort(bcells)]).astype(np.int32)
    nf = len(owner)
    # Cell-face slots: every face on its owner's side, internal faces also on
    # the neighbour's, grouped by cell in face order.
    slot_cell = np.concatenate([owner, nb])
    slot_face = np.concatenate([np.arange(nf), np.arange(internal)]).astype(np.int32)
    slot_sign = np.concatenate([np.ones(nf), -np.ones(internal)]).astype(np.float32)
    slot_adj = np.concatenate([np.concatenate([nb, -np.ones(nf - internal, np.int32)]), own])
    order = np.lexsort((slot_face, slot_cell))
    slot_cell, slot_face = slot_cell[order], slot_face[order]
    slot_sign, slot_adj = slot_sign[order], slot_adj[order].astype(np.int32)
    offsets = np.zeros(n + 1, np.int32)
    np.add.at(offsets, slot_cell + 1, 1)
    offsets = np.cumsum(offsets).astype(np.int32)
    # CSR keys row * n + col are sorted, so one search finds every entry.
    keys = rows.astype(np.int64) * n + np.asarray(col, np.int64)
    entry = np.full(len(slot_cell), -1, np.int32)
    inner = slot_adj >= 0
    entry[inner] = np.searchsorted(keys, slot_cell[inner].astype(np.int64) * n + slot_adj[inner])
    coefficient = np.exp(rng.uniform(np.log(1e-3), 0.0, nf)).astype(np.float32)
    flux = rng.normal(size=nf).astype(np.float32)
    return FvCase(n=n, rows=np.asarray(row_ptr, np.int32), cols=np.asarray(col, np.int32),
                  diag=np.asarray(diag, np.int32), owner=owner, neighbour=nb.astype(np.int32),
                  internal=internal, offsets=offsets, faces=slot_face, sign=slot_sign,
                  adjacent=slot_adj, entry=entry, coefficient=coefficient, flux=flux,
                  reference=reference)
