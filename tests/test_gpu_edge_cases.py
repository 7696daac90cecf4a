"""The reference solver tests' exact edge cases, run by the CUDA solver and
compared with the reference library (oracle/_ref) and the oracle on the same
inputs. These drive the device's (hi,lo) float-pair scalar epilogue into its
guard states: a residual that cannot shrink below float representability, a
reference term of 2^-20 that must not be projected away, an exact one-step
exit, BiCGStab's frozen state after a zero omega or a zero shadow product, and
residual-check intervals that must change no bits.

- test_solvers.cpp:214-229: representability limit is not convergence;
- test_solvers.cpp:255-272: a small reference term is kept;
- test_solvers.cpp:359-391: reused solves, interval invariance;
- test_solvers.cpp:393-407: exact one-step exit;
- test_solvers.cpp:603-629: BiCGStab freezes on a zero omega / shadow product.

On these one- and two-row systems every FP64 reduction adds at most two
nonzero terms, so the device's reduction tree cannot reorder anything: the
bar is bit equality with the reference library in iterations, flags, both
residuals and x. The interval case (192 rows) compares the device with itself
bit for bit and with the reference at the usual tolerances."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import kutta_oracle as O
from oracle import ref

pytestmark = pytest.mark.gpu

PCG_JACOBI, BICGSTAB_JACOBI, AMG_PCG = 1, 2, 3


def _system(row_ptr, col, diag, val, b):
    return harness.HostSystem(np.array(row_ptr, np.int32), np.array(col, np.int32),
                              np.array(diag, np.int32), np.array(val, np.float64),
                              np.array(b, np.float32))


def _gpu(s, kind, rel_tol, abs_tol, max_iter, interval=8):
    import torch
    a = L.upload(s)
    if kind >= AMG_PCG:
        solver = L.make_amg_solver(L.SolverKind(kind), s, L.AmgOptions())
    else:
        solver = L.make_solver(L.SolverKind(kind), s, L.SolverOptions())
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    x = torch.zeros(s.n, dtype=torch.float32, device="cuda")
    st = solver.solve(a, x, b, L.SolveControl(rel_tol, abs_tol, max_iter, interval))
    torch.cuda.synchronize()
    return st, x.cpu().numpy(), solver.describe()


def _expected(s, kind, rel_tol, abs_tol, max_iter, interval=8):
    """The reference library's result where it is built, else the oracle's
    (the two are equal bit for bit on these cases, tests/test_oracle_edge_cases.py)."""
    if ref.available():
        return ref.solve(s, opts=ref.options(kind), rel_tol=rel_tol, abs_tol=abs_tol,
                         max_iter=max_iter, interval=interval)
    return O.solve(s, kind, rel_tol=rel_tol, abs_tol=abs_tol, max_iter=max_iter,
                   interval=interval)


def _bitwise(st, x, r):
    assert (st.iterations, st.converged) == (r.iterations, r.converged)
    assert (st.initial_residual, st.final_residual) == (r.initial_residual, r.final_residual)
    assert np.array_equal(x.view(np.uint32), np.asarray(r.x, np.float32).view(np.uint32))


def test_representability_limit_is_not_convergence(cuda):
    s = _system([0, 1], [0], [0], [7.0], [1.0])
    st, x, _ = _gpu(s, PCG_JACOBI, 1e-10, 0.0, 100)
    assert not st.converged
    assert st.final_residual > 1e-10
    assert st.final_residual == pytest.approx(abs(1 - 7 * float(x[0])), rel=1e-6)
    _bitwise(st, x, _expected(s, PCG_JACOBI, 1e-10, 0.0, 100))


@pytest.mark.parametrize("kind", [PCG_JACOBI, AMG_PCG], ids=["pcg_jacobi", "amg_pcg"])
def test_small_reference_term_is_kept(cuda, kind):
    d = 1 + 2.0 ** -20
    s = _system([0, 2, 4], [0, 1, 0, 1], [0, 3], [d, -1, -1, d], [1, 1])
    st, x, describe = _gpu(s, kind, 1e-6, 0.0, 100)
    assert "nullspace" not in describe
    assert st.converged
    assert float(x[0]) == pytest.approx(2.0 ** 20, rel=1e-6)
    r = _expected(s, kind, 1e-6, 0.0, 100)
    assert describe == r.describe
    _bitwise(st, x, r)


@pytest.mark.parametrize("interval", [1, 8, 31])
@pytest.mark.parametrize("zero_omega", [True, False], ids=["zero_omega", "zero_shadow"])
def test_bicgstab_freezes_on_breakdown(cuda, zero_omega, interval):
    # A [1, 1] = [4, 0] with alpha = 1/2 gives s = [-1, 1] and A s = [2, 2]:
    # t.s = 0 while t.t = 8, an exact omega breakdown after one step. The
    # second matrix makes the shadow product rhat.v zero before any step.
    val = [1, 3, -1, 1] if zero_omega else [1, 2, -4, 1]
    s = _system([0, 2, 4], [0, 1, 0, 1], [0, 3], val, [1, 1])
    st, x, _ = _gpu(s, BICGSTAB_JACOBI, 1e-8, 0.0, 31, interval)
    assert not st.converged
    assert st.iterations == (1 if zero_omega else 0)
    assert st.final_residual == st.initial_residual
    assert x.tolist() == [0.0, 0.0]
    _bitwise(st, x, _expected(s, BICGSTAB_JACOBI, 1e-8, 0.0, 31, interval))


@pytest.mark.parametrize("kind", [PCG_JACOBI, BICGSTAB_JACOBI], ids=["pcg_jacobi", "bicgstab"])
def test_exact_one_step_exit(cuda, kind):
    s = _system([0, 1], [0], [0], [2.0], [1.0])
    st, x, _ = _gpu(s, kind, 1e-6, 1e-12, 20)
    assert st.converged and st.iterations == 1
    assert st.final_residual == 0 and x.tolist() == [0.5]
    _bitwise(st, x, _expected(s, kind, 1e-6, 1e-12, 20))


def test_residual_check_interval_changes_no_bits(cuda):
    """A diagonally boosted upwind BiCGStab-Jacobi solve gives the same
    iterations, final residual and x at residual-check intervals 8 and 1 on the
    device (the interval only batches host status polls), and matches the
    reference at both."""
    s = harness.poisson(8, 6, 4, 1, False, False, 5)
    s.val[s.diag] += 100
    s.b = harness.random_solution(s.n)
    st8, x8, _ = _gpu(s, BICGSTAB_JACOBI, 1e-4, 1e-12, 100, 8)
    st1, x1, _ = _gpu(s, BICGSTAB_JACOBI, 1e-4, 1e-12, 100, 1)
    assert st8.converged
    assert (st8.iterations, st8.final_residual) == (st1.iterations, st1.final_residual)
    assert np.array_equal(x8.view(np.uint32), x1.view(np.uint32))
    for st, x, interval in ((st8, x8, 8), (st1, x1, 1)):
        r = _expected(s, BICGSTAB_JACOBI, 1e-4, 1e-12, 100, interval)
        assert (st.iterations, st.converged) == (r.iterations, r.converged)
        assert st.final_residual == pytest.approx(r.final_residual, rel=1e-3)
        err = np.linalg.norm(x.astype(np.float64) - r.x) / np.linalg.norm(r.x)
        assert err <= 1e-5, err
