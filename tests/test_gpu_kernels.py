"""Kernel-level parity: each CUDA kernel bit-for-bit against the oracle's
restatement of the reference kernel, on the same inputs, through the C ABI."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import kutta_oracle as O

pytestmark = pytest.mark.gpu
p = O.p


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _systems():
    rng = np.random.default_rng(5)
    out = [harness.box_system(10, 10, 10, tet=True, seed=1),
           harness.box_system(12, 12, 12, tet=False, seed=2),
           harness.poisson(31, 17, 5, 1, True)]
    # Skewed rows: a few dense rows (hundreds of entries) among short ones, so
    # some 256-row tiles exceed the staging capacity and take the row path.
    n = 6000
    lens = np.where(rng.random(n) < 0.02, rng.integers(200, 900, n), rng.integers(1, 9, n))
    row_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    val = rng.standard_normal(row_ptr[-1]).astype(np.float32).astype(np.float64)
    out.append(harness.HostSystem(row_ptr, col, np.zeros(n, np.int32), val,
                                  rng.standard_normal(n).astype(np.float32)))
    return out


@pytest.mark.parametrize("k", range(4))
def test_csr_kernels_bitwise(cuda, k):
    import torch
    s = _systems()[k]
    n = s.n
    rng = np.random.default_rng(k)
    x = (rng.standard_normal(n) * 10).astype(np.float32)
    b = s.b.astype(np.float32)
    inv = (rng.random(n) + 0.1).astype(np.float32)
    vals = s.val.astype(np.float32)
    a = L.CsrMatrix(n, s.nnz, torch.from_numpy(s.row_ptr).cuda(), torch.from_numpy(s.col).cuda(),
                    torch.from_numpy(s.diag).cuda(), torch.from_numpy(vals).cuda())
    tx, tb, ti = (torch.from_numpy(v).cuda() for v in (x, b, inv))
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    lib = O.lib()
    ref = np.zeros(n, np.float32)

    L.spmv(a, tx, out)
    lib.ko_spmv(n, p(s.row_ptr), p(s.col), p(vals), p(x), p(ref))
    assert np.array_equal(bits(out.cpu().numpy()), bits(ref))

    L.residual(a, tx, tb, out)
    lib.ko_residual(n, p(s.row_ptr), p(s.col), p(vals), p(x), p(b), p(ref))
    assert np.array_equal(bits(out.cpu().numpy()), bits(ref))

    status = np.zeros(3, np.int32)
    for zero in (0, 1):
        L.amg_smooth(a, tx, tb, ti, out, zero_start=bool(zero))
        xin = np.zeros(n, np.float32) if zero else x
        lib.ko_smooth(n, p(s.row_ptr), p(s.col), p(vals), p(xin), p(b), p(inv), p(ref), p(status), zero)
        assert np.array_equal(bits(out.cpu().numpy()), bits(ref)), zero


def test_zero_start_sweep_special_values_bitwise(cuda):
    """test_amg_zero.cpp:11-48 of the reference, on the device: the zero-start
    sweep equals the full sweep from x = 0 bit for bit, and both equal the
    oracle, for signed zeros, subnormals, infinities and NaN payloads."""
    import torch
    rhs_values = np.array([0.0, -0.0, 1, -1, 1e30, -1e30, 1e-30, -1e-30,
                           np.finfo(np.float32).smallest_subnormal, np.inf, -np.inf, 0], np.float32)
    rhs_values[11] = np.frombuffer(np.uint32(0x7FC01234).tobytes(), np.float32)[0]
    mvals = np.array([0.0, -0.0, 1, -1, 1e30, -1e30, 1e-30, -1e-30], np.float32)
    for n in (513, 2053):
        i = np.arange(n)
        row_ptr = (7 * np.arange(n + 1)).astype(np.int32)
        cols = ((i[:, None] + np.arange(7)[None, :] * 31) % n).astype(np.int32).ravel()
        vals = mvals[(i[:, None] + np.arange(7)[None, :]) % 8].astype(np.float32).ravel()
        b = rhs_values[i % 12]
        inv = mvals[(i // 12) % 8]
        a = L.CsrMatrix(n, 7 * n, torch.from_numpy(row_ptr).cuda(), torch.from_numpy(cols).cuda(),
                        torch.zeros(n, dtype=torch.int32, device="cuda"), torch.from_numpy(vals).cuda())
        x = torch.zeros(n, dtype=torch.float32, device="cuda")
        tb, ti = torch.from_numpy(b).cuda(), torch.from_numpy(inv).cuda()
        full = torch.empty_like(x)
        zero = torch.empty_like(x)
        L.amg_smooth(a, x, tb, ti, full, zero_start=False)
        L.amg_smooth(a, x, tb, ti, zero, zero_start=True)
        f, z = full.cpu().numpy(), zero.cpu().numpy()
        assert np.array_equal(bits(f), bits(z))
        ref = np.zeros(n, np.float32)
        x0 = np.zeros(n, np.float32)
        status = np.zeros(3, np.int32)
        O.lib().ko_smooth(n, p(row_ptr), p(cols), p(vals), p(x0), p(b), p(inv), p(ref), p(status), 0)
        # The GPU returns the canonical NaN where the CPU propagates an input
        # NaN's payload; every other value must match bit for bit.
        nan = np.isnan(ref)
        assert np.array_equal(np.isnan(f), nan)
        assert np.array_equal(bits(f)[~nan], bits(ref)[~nan])


def test_launch_counter_counts_native_kernels(cuda):
    import torch
    s = harness.poisson(8, 8, 8)
    a = L.upload(s)
    x = torch.ones(s.n, device="cuda")
    y = torch.empty_like(x)
    before = L.kernel_launches()
    L.spmv(a, x, y)
    L.spmv(a, x, y)
    torch.cuda.synchronize()
    assert L.kernel_launches() - before == 2
