"""Test infrastructure only: the finite-volume kernels around the pressure
solve (src/kutta/kernels/fv_flow.kern.h:164-201) from the two CPU sources of
truth: the C restatement in kutta_oracle.c (ko_fv_*) and the reference's own
kernels compiled into oracle/_ref (kref_fv_*). Arrays are numpy; outputs are
updated in place, as the kernels do."""
from __future__ import annotations

import ctypes

import numpy as np

from oracle import ref
from oracle.kutta_oracle import lib as oracle_lib

_P = ctypes.c_void_p
_I = ctypes.c_int


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a.size else None


def _check(code, lib):
    if code != 0:
        raise RuntimeError(lib.kref_last_error().decode())


def oracle_assemble(case, values, rhs):
    lib = oracle_lib()
    lib.ko_fv_pressure_assemble.argtypes = [_I] + [_P] * 11 + [_I]
    lib.ko_fv_pressure_assemble(case.n, *(_p(getattr(case, k)) for k in (
        "offsets", "faces", "sign", "adjacent", "entry", "rows", "diag", "coefficient", "flux")),
        _p(values), _p(rhs), case.reference)


def oracle_correct_flux(case, correction, flux):
    lib = oracle_lib()
    lib.ko_fv_correct_flux.argtypes = [_I, _P, _P, _P, _P, _P, _I]
    lib.ko_fv_correct_flux(case.n_faces, _p(case.owner), _p(case.neighbour), _p(correction),
                           _p(case.coefficient), _p(flux), case.internal)


def oracle_correct_velocity(n, volume, inverse, diagonal, g, correction, uvwp, alpha):
    lib = oracle_lib()
    lib.ko_fv_correct_velocity.argtypes = [_I] + [_P] * 11 + [ctypes.c_float]
    lib.ko_fv_correct_velocity(n, _p(volume), _p(inverse), _p(diagonal), _p(g[0]), _p(g[1]),
                               _p(g[2]), _p(correction), *(_p(a) for a in uvwp), alpha)


def ref_assemble(case, values, rhs):
    lib = ref._load()
    lib.kref_fv_pressure_assemble.argtypes = [_I] * 4 + [_P] * 11 + [_I]
    lib.kref_last_error.restype = ctypes.c_char_p
    _check(lib.kref_fv_pressure_assemble(case.n, case.n_faces, len(case.faces), len(values),
                                         *(_p(getattr(case, k)) for k in (
                                             "offsets", "faces", "sign", "adjacent", "entry",
                                             "rows", "diag", "coefficient", "flux")),
                                         _p(values), _p(rhs), case.reference), lib)


def ref_correct_flux(case, correction, flux):
    lib = ref._load()
    lib.kref_fv_correct_flux.argtypes = [_I, _I, _P, _P, _P, _P, _P, _I]
    lib.kref_last_error.restype = ctypes.c_char_p
    _check(lib.kref_fv_correct_flux(case.n_faces, case.n, _p(case.owner), _p(case.neighbour),
                                    _p(correction), _p(case.coefficient), _p(flux),
                                    case.internal), lib)


def ref_correct_velocity(n, volume, inverse, diagonal, g, correction, uvwp, alpha):
    lib = ref._load()
    lib.kref_fv_correct_velocity.argtypes = [_I] + [_P] * 11 + [ctypes.c_float]
    lib.kref_last_error.restype = ctypes.c_char_p
    _check(lib.kref_fv_correct_velocity(n, _p(volume), _p(inverse), _p(diagonal), _p(g[0]),
                                        _p(g[1]), _p(g[2]), _p(correction),
                                        *(_p(a) for a in uvwp), alpha), lib)
