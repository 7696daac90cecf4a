"""Small exact cases of the reference's own solver tests, run on the oracle
and, where oracle/_ref is built, on the reference library too. Each case
asserts what the reference test asserts, and the oracle must match the
reference bit for bit: iterations, flags, both residuals and x. CPU only.

- test_solvers.cpp:214-229: float representability limits never produce
  false convergence (1x1 system, PCG-Jacobi, relative 1e-10);
- test_solvers.cpp:255-272: a small reference term is kept, not projected
  away (2x2, diagonal 1 + 2^-20; PCG-Jacobi and AMG-PCG);
- test_solvers.cpp:603-629: BiCGStab freezes on a zero omega and on a zero
  shadow product, at residual-check intervals 1, 8 and 31;
- test_solvers.cpp:393-407: an exact one-step exit (2 x = 1);
- test_solvers.cpp:359-391: the residual-check interval changes no bits."""
import numpy as np
import pytest

from kutta_b200 import harness
from oracle import kutta_oracle as O
from oracle import ref

PCG_JACOBI, BICGSTAB_JACOBI = 1, 2


def _system(row_ptr, col, diag, val, b):
    return harness.HostSystem(np.array(row_ptr, np.int32), np.array(col, np.int32),
                              np.array(diag, np.int32), np.array(val, np.float64),
                              np.array(b, np.float32))


def _both(s, kind, rel_tol, abs_tol, max_iter, interval=8):
    o = O.solve(s, kind, rel_tol=rel_tol, abs_tol=abs_tol, max_iter=max_iter, interval=interval)
    if not ref.available():
        return o, None
    r = ref.solve(s, opts=ref.options(kind), rel_tol=rel_tol, abs_tol=abs_tol,
                  max_iter=max_iter, interval=interval)
    return o, r


def _same(o, r):
    if r is None:
        return
    assert (o.iterations, o.converged) == (r.iterations, r.converged)
    assert (o.initial_residual, o.final_residual) == (r.initial_residual, r.final_residual)
    assert np.array_equal(o.x.view(np.uint32), r.x.view(np.uint32))


def test_representability_limit_is_not_convergence():
    s = _system([0, 1], [0], [0], [7.0], [1.0])
    o, r = _both(s, PCG_JACOBI, 1e-10, 0.0, 100)
    assert not o.converged
    assert o.final_residual > 1e-10
    assert o.final_residual == pytest.approx(abs(1 - 7 * float(o.x[0])), rel=1e-6)
    _same(o, r)


@pytest.mark.parametrize("kind", [PCG_JACOBI, O.AMG_PCG], ids=["pcg_jacobi", "amg_pcg"])
def test_small_reference_term_is_kept(kind):
    d = 1 + 2.0 ** -20
    s = _system([0, 2, 4], [0, 1, 0, 1], [0, 3], [d, -1, -1, d], [1, 1])
    o, r = _both(s, kind, 1e-6, 0.0, 100)
    assert "nullspace" not in o.describe
    assert o.converged
    assert float(o.x[0]) == pytest.approx(2.0 ** 20, rel=1e-6)
    _same(o, r)
    if r is not None:
        assert o.describe == r.describe


@pytest.mark.parametrize("interval", [1, 8, 31])
@pytest.mark.parametrize("zero_omega", [True, False], ids=["zero_omega", "zero_shadow"])
def test_bicgstab_freezes_on_breakdown(zero_omega, interval):
    # A [1, 1] = [4, 0], alpha = 1/2, s = [-1, 1], A s = [2, 2]: t.s = 0 while
    # t.t = 8, an exact omega breakdown after one step; the second matrix makes
    # the shadow product rhat.v zero before any step.
    val = [1, 3, -1, 1] if zero_omega else [1, 2, -4, 1]
    s = _system([0, 2, 4], [0, 1, 0, 1], [0, 3], val, [1, 1])
    o, r = _both(s, BICGSTAB_JACOBI, 1e-8, 0.0, 31, interval)
    assert not o.converged
    assert o.iterations == (1 if zero_omega else 0)
    assert o.final_residual == o.initial_residual
    assert o.x.tolist() == [0.0, 0.0]
    _same(o, r)


@pytest.mark.parametrize("kind", [PCG_JACOBI, BICGSTAB_JACOBI], ids=["pcg_jacobi", "bicgstab"])
def test_exact_one_step_exit(kind):
    """test_solvers.cpp:393-407: 2 x = 1 converges in one step with a zero
    final residual and x = 0.5."""
    s = _system([0, 1], [0], [0], [2.0], [1.0])
    o, r = _both(s, kind, 1e-6, 1e-12, 20)
    assert o.converged and o.iterations == 1
    assert o.final_residual == 0 and o.x.tolist() == [0.5]
    _same(o, r)


def test_residual_check_interval_changes_no_bits():
    """test_solvers.cpp:359-391: a diagonally boosted upwind BiCGStab-Jacobi
    solve gives the same iterations, final residual and x at residual-check
    intervals 8 and 1 (the interval only batches host polls)."""
    s = harness.poisson(8, 6, 4, 1, False, False, 5)
    s.val[s.diag] += 100
    s.b = harness.random_solution(s.n)
    o8, r8 = _both(s, BICGSTAB_JACOBI, 1e-4, 1e-12, 100, 8)
    o1, r1 = _both(s, BICGSTAB_JACOBI, 1e-4, 1e-12, 100, 1)
    assert o8.converged
    assert (o8.iterations, o8.final_residual) == (o1.iterations, o1.final_residual)
    assert np.array_equal(o8.x.view(np.uint32), o1.x.view(np.uint32))
    _same(o8, r8)
    _same(o1, r1)
