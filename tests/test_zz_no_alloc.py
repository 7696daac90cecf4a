"""b2_dense_inverse_noalloc: the dense coarsest-level inverse for callers that
cannot allocate device memory, called through the C ABI and compared with
b2_dense_inverse (which allocates its factor scratch) on two calls in a row.

The file name sorts last so pytest collects it after every other test; it also
passes alone in a fresh process, where its first call is also the call that
looks up the built-in scratch array."""
import ctypes

import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L

# The tolerance of the dense inverse tests against numpy FP64, relative to the
# largest entry of the inverse.
REL_TOL = 1e-9

# b2_status values (include/kutta_b200.h).
B2_OK = 0
B2_INVALID_ARGUMENT = 1


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _call(name, a, inverse, flag):
    import torch
    lib = L._load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return getattr(lib, name)(a.n_rows, _ptr(a.row_ptr), _ptr(a.col), _ptr(a.val),
                              _ptr(inverse), _ptr(flag), stream)


def _both(s):
    """(no-allocation result, flag), (allocating result, flag) for one system."""
    import torch
    a = L.upload(s)
    n = s.n
    got = torch.full((n * n,), float("nan"), dtype=torch.float64, device="cuda")
    want = torch.full((n * n,), float("nan"), dtype=torch.float64, device="cuda")
    got_flag = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    want_flag = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    assert _call("b2_dense_inverse_noalloc", a, got, got_flag) == B2_OK, L.last_error()
    assert _call("b2_dense_inverse", a, want, want_flag) == B2_OK, L.last_error()
    torch.cuda.synchronize()
    return ((got.cpu().numpy().reshape(n, n), got_flag.item()),
            (want.cpu().numpy().reshape(n, n), want_flag.item()))


# Operators of up to ON_CHIP_ROWS rows are factored in shared memory and never
# touch the built-in scratch array; every case below is larger, so each call
# factors through that array.
ON_CHIP_ROWS = 236


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda):
    # First a larger operator, then a smaller one with other values: the second
    # call reuses the part of the array the first one filled, and must not see
    # its leftovers.
    first = harness.box_system(4, 4, 4, tet=True, seed=4)    # 384 rows
    second = harness.box_system(7, 7, 7, tet=False, seed=9)  # 343 rows
    assert ON_CHIP_ROWS < second.n < first.n <= 512
    for s in (first, second):
        (got, got_flag), (want, want_flag) = _both(s)
        assert got_flag == want_flag == 0.0
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - want)) <= REL_TOL * np.max(np.abs(want))


@pytest.mark.gpu
def test_noalloc_at_its_size_limit(cuda):
    s = harness.box_system(8, 8, 8, tet=False, seed=5)  # 512 rows: the whole array
    assert s.n == 512
    (got, got_flag), (want, want_flag) = _both(s)
    assert got_flag == want_flag == 0.0
    assert np.max(np.abs(got - want)) <= REL_TOL * np.max(np.abs(want))


@pytest.mark.gpu
def test_noalloc_flags_non_spd_like_allocating_entry_point(cuda):
    s = harness.box_system(7, 7, 6, tet=False, seed=4)  # 294 rows
    assert s.n > ON_CHIP_ROWS
    bad = s.val.copy()
    bad[s.diag[0]] = -1.0
    (_, got_flag), (_, want_flag) = _both(harness.HostSystem(s.row_ptr, s.col, s.diag, bad, s.b))
    assert got_flag == want_flag == 1.0
    # The next call on the same array, with an SPD operator, is unaffected.
    (got, got_flag), (want, want_flag) = _both(s)
    assert got_flag == want_flag == 0.0
    assert np.max(np.abs(got - want)) <= REL_TOL * np.max(np.abs(want))


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    s = harness.box_system(3, 3, 3, tet=True, seed=4)
    a = L.upload(s)
    inverse = torch.zeros(s.n * s.n, dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = L._load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # The size check comes before any device work, so the small arrays are
    # never read.
    status = lib.b2_dense_inverse_noalloc(513, _ptr(a.row_ptr), _ptr(a.col), _ptr(a.val),
                                          _ptr(inverse), _ptr(flag), stream)
    assert status == B2_INVALID_ARGUMENT
    assert "513" in L.last_error() and "512" in L.last_error()
