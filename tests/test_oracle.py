"""The oracle (C restatement) against the reference's golden vectors: the
known-answer values of the reference's own kernel tests, its published
benchmark residual, and the committed fixtures generated from the reference's
CPU path (tests/golden/make_golden.py). CPU only."""
import ctypes

import numpy as np
import pytest

import golden_cases as G
from kutta_b200 import harness
from oracle import kutta_oracle as O
from oracle import ref

L = O.lib()
p = O.p


def f32(*v):
    return np.array(v, np.float32)


def i32(*v):
    return np.array(v, np.int32)


@pytest.mark.parametrize("name", G.names())
def test_oracle_reproduces_reference_fixture(name):
    meta, arrays = G.load(name)
    s = G.system(name)
    opts = O.options(meta["kind"], m_matrix=bool(meta["m_matrix"]), **meta.get("options", {}))
    r = O.solve(s, opts=opts, rel_tol=meta["rel_tol"], abs_tol=meta["abs_tol"],
                max_iter=meta["max_iter"])
    assert r.iterations == meta["iterations"]
    assert r.converged == meta["converged"]
    assert r.initial_residual == meta["initial_residual"]
    assert r.final_residual == meta["final_residual"]
    assert r.describe == meta["describe"]
    assert G.digest(r.x) == meta["x_sha"]
    if "x" in arrays:
        assert np.array_equal(r.x.view(np.uint32), arrays["x"].view(np.uint32))
    if meta["kind"] >= 3:
        solver = O.Solver(s, opts)
        solver.refresh(s.val.astype(np.float32))
        levels = solver.levels()
        assert [lv["n"] for lv in levels] == meta["levels"]
        for i, (lv, sha) in enumerate(zip(levels, meta["level_sha"])):
            assert G.digest(lv["row_ptr"]) == sha["row_ptr"]
            assert G.digest(lv["col"]) == sha["col"]
            assert G.digest(lv["l1"]) == sha["l1"]
            if i > 0:
                assert G.digest(lv["val"]) == sha["val"]
            if sha["aggregate"] is not None:
                assert G.digest(lv["aggregate"]) == sha["aggregate"]


def test_published_64cube_residual():
    """bench_linalg.log:3 of the reference: 64^3 Poisson, random forcing, AMG-PCG,
    15 iterations, relative residual 7.91394974e-07 (x86, bitwise)."""
    s = harness.poisson(64, 64, 64)
    s.b = harness.random_forcing(s.n)
    r = O.solve(s, O.AMG_PCG, rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert r.iterations == 15
    assert f"{r.final_residual / r.initial_residual:.8e}" == "7.91394974e-07"


@pytest.mark.parametrize("anisotropy,kind,iterations,converged,relative", [
    (1, 1, 278, True, "6.85768115e-07"),
    (1000, 1, 354, False, "1.53025686e-06"),
    (1000, 3, 38, False, "1.51536251e-06"),
], ids=["pcg_jacobi", "pcg_jacobi_aniso1000", "amg_pcg_aniso1000"])
def test_published_64cube_lines(anisotropy, kind, iterations, converged, relative):
    """The other 64^3 lines of the reference's published CPU log
    (validation/results/colab_t4/logs/bench_linalg.log, x86, bitwise): random
    forcing, SolveControl{1e-6, 1e-12, 2000}, isotropic PCG-Jacobi and the
    1:1000 anisotropic case, where both solvers stop unconverged."""
    s = harness.poisson(64, 64, 64, anisotropy)
    s.b = harness.random_forcing(s.n)
    r = O.solve(s, kind, rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert (r.iterations, r.converged) == (iterations, converged)
    assert f"{r.final_residual / r.initial_residual:.8e}" == relative


@pytest.mark.slow
def test_published_128cube_residual():
    """bench_linalg.log of the reference, its largest line: 128^3 Poisson
    (2.1M rows), random forcing, AMG-PCG, 21 iterations, relative residual
    8.66568009e-07 (x86, bitwise). About half a minute on one core."""
    s = harness.poisson(128, 128, 128)
    s.b = harness.random_forcing(s.n)
    r = O.solve(s, O.AMG_PCG, rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert (r.iterations, r.converged) == (21, True)
    assert f"{r.final_residual / r.initial_residual:.8e}" == "8.66568009e-07"


def test_published_32cube_iterations():
    """linalg/README.md:483-484 of the reference: 32^3 random forcing, 11 iterations."""
    s = harness.poisson(32, 32, 32)
    s.b = harness.random_forcing(s.n)
    r = O.solve(s, O.AMG_PCG, rel_tol=1e-6, abs_tol=0, max_iter=300)
    assert r.iterations == 11 and r.converged


def test_kernel_known_answers():
    """tests/linalg/test_kernels.cpp:11-64 of the reference."""
    offsets, members = i32(0, 2, 5), i32(0, 2, 1, 3, 4)
    agg, fine = i32(0, 1, 0, 1, 1), f32(1, 2, 3, 4, 5)
    coarse = np.zeros(2, np.float32)
    L.ko_restrict(2, p(offsets), p(members), p(fine), p(coarse))
    assert coarse.tolist() == [4, 11]
    L.ko_prolong(5, p(agg), p(coarse), p(fine))
    assert fine.tolist() == [5, 13, 7, 15, 16]
    L.ko_galerkin(2, p(offsets), p(members), p(fine), p(coarse))
    assert coarse.tolist() == [12, 44]
    rows, diag, vals = i32(0, 2, 5, 7), i32(0, 3, 6), f32(2, -1, -1, 4, -2, -2, 8)
    out, invalid, l1 = (np.zeros(3, np.float32) for _ in range(3))
    L.ko_diagonal(3, p(rows), p(diag), p(vals), p(out), p(invalid), 0)
    assert out.tolist() == [0.5, 0.25, 0.125]
    L.ko_diagonal(3, p(rows), p(diag), p(vals), p(l1), p(invalid), 1)
    assert l1.tolist() == out.tolist() and invalid.max() == 0
    vals[:] = 0
    L.ko_diagonal(3, p(rows), p(diag), p(vals), p(out), p(invalid), 0)
    assert invalid.tolist() == [1, 1, 1]


def test_galerkin_keeps_weak_term_across_cancellation():
    """test_kernels.cpp:154-170: Neumaier keeps the 1 in {1e8, 1, -1e8}."""
    offsets, entries, fine = i32(0, 3), i32(0, 1, 2), f32(1e8, 1, -1e8)
    coarse = np.zeros(1, np.float32)
    L.ko_galerkin(1, p(offsets), p(entries), p(fine), p(coarse))
    assert coarse[0] == 1


def test_compensated_residual_resolves_cancellation():
    """test_kernels.cpp:66-90."""
    rows, cols = i32(0, 3, 6, 9), i32(0, 1, 2, 0, 1, 2, 0, 1, 2)
    vals = f32(6, -1, -1, -1, 6, -1, -1, -1, 6)
    x = f32(np.nextafter(np.float32(1), np.float32(2)), -1, 1)
    b = f32(6, -8, 6)
    r = np.zeros(3, np.float32)
    L.ko_residual(3, p(rows), p(cols), p(vals), p(x), p(b), p(r))
    expect = [float(b[i]) - sum(float(vals[j]) * float(x[cols[j]]) for j in range(rows[i], rows[i + 1]))
              for i in range(3)]
    np.testing.assert_allclose(r, np.float32(expect), rtol=1e-6)


@pytest.mark.parametrize("count", [1, 17, 24])
def test_fused_coarse_solve_equals_ordinary_sweeps(count):
    """test_kernels.cpp:92-127."""
    s = harness.poisson(count, 1)
    rows, cols, vals = s.row_ptr, s.col, s.val.astype(np.float32)
    b = harness.random_solution(count)
    inv = (np.float32(1) / vals[s.diag]).astype(np.float32)
    status = i32(0)
    for sweeps in (1, 5, 32):
        y = np.zeros(count, np.float32)
        r = np.zeros(count, np.float32)
        for _ in range(sweeps):
            L.ko_residual(count, p(rows), p(cols), p(vals), p(y), p(b), p(r))
            y = (y + np.float32(2.0 / 3.0) * inv * r).astype(np.float32)
        x = np.zeros(count, np.float32)
        L.ko_coarse_solve(p(rows), p(cols), p(vals), p(x), p(b), p(inv), p(status), count, sweeps)
        assert np.array_equal(x, y)
    frozen = i32(2)
    x = np.full(count, 42, np.float32)
    L.ko_coarse_solve(p(rows), p(cols), p(vals), p(x), p(b), p(inv), p(frozen), count, 32)
    assert np.all(x == 42)


def test_zero_start_sweep_preserves_full_sweep_bits():
    """test_amg_zero.cpp:11-48: signed zeros, subnormals, infinities, NaN payloads."""
    rhs_values = np.array([0.0, -0.0, 1, -1, 1e30, -1e30, 1e-30, -1e-30,
                           np.finfo(np.float32).smallest_subnormal, np.inf, -np.inf, 0], np.float32)
    rhs_values[11] = np.frombuffer(np.uint32(0x7FC01234).tobytes(), np.float32)[0]
    mvals = np.array([0.0, -0.0, 1, -1, 1e30, -1e30, 1e-30, -1e-30], np.float32)
    for n in (513, 2053):
        rows = (7 * np.arange(n + 1)).astype(np.int32)
        i = np.arange(n)
        cols = ((i[:, None] + np.arange(7)[None, :] * 31) % n).astype(np.int32).ravel()
        vals = mvals[(i[:, None] + np.arange(7)[None, :]) % 8].astype(np.float32).ravel()
        b = rhs_values[i % 12]
        inv = mvals[(i // 12) % 8]
        x = np.zeros(n, np.float32)
        for phase in (0, 1, 2):
            st = i32(phase, 0, 0)
            e = np.full(n, 42, np.float32)
            a = np.full(n, 42, np.float32)
            L.ko_smooth(n, p(rows), p(cols), p(vals), p(x), p(b), p(inv), p(e), p(st), 0)
            L.ko_smooth(n, p(rows), p(cols), p(vals), p(x), p(b), p(inv), p(a), p(st), 1)
            assert np.array_equal(e.view(np.uint32), a.view(np.uint32))


def test_coefficient_guards_hold_on_zero_or_nonfinite():
    """test_kernels.cpp:129-152: bicg_beta freezes on zero/NaN/Inf rho or omega."""
    for slot in (0, 12):
        for bad in (0.0, np.nan, np.inf):
            sc = np.zeros(24, np.float32)
            sc[[0, 8, 12, 14]] = 1
            sc[slot] = bad
            st = i32(0, 0, 0)
            L.ko_scalar(3, p(sc), p(st), 0)
            x, r, pv = f32(2, -3), f32(4, 5), f32(1, 1)
            L.ko_solver_step(2, p(x), p(r), p(pv), p(pv), p(sc), p(st))
            assert st[0] == 2
            assert x.tolist() == [2, -3] and r.tolist() == [4, 5]


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built on this machine")
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_bitwise_equals_reference_library(seed):
    """Direct pin against the reference CPU library when it is present."""
    s = harness.box_system(10, 10, 10, tet=True, seed=seed)
    r = ref.solve(s, opts=ref.options(3, structure=1), rel_tol=1e-6, abs_tol=1e-12, max_iter=500)
    o = O.solve(s, O.AMG_PCG, m_matrix=True, rel_tol=1e-6, abs_tol=1e-12, max_iter=500)
    assert (o.iterations, o.final_residual) == (r.iterations, r.final_residual)
    assert np.array_equal(o.x.view(np.uint32), r.x.view(np.uint32))


def test_fp64_oracle_solves_to_tolerance():
    s = harness.box_system(8, 8, 8, tet=True, seed=4)
    x, it = O.cg64(s, rel_tol=1e-12)
    A_res = O.true_residual(s, x.astype(np.float32))
    assert it > 0
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    assert np.linalg.norm(s.b.astype(np.float64) - A @ x) <= 1e-11 * np.linalg.norm(s.b)
    assert A_res < 1e-4 * np.linalg.norm(s.b)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built on this machine")
@pytest.mark.parametrize("sweeps", [1, 2, 3])
def test_oracle_equals_reference_library_at_other_sweep_counts(sweeps):
    """V(s,s) pressure solves; the steady solver runs V(2,2) with the SST model
    (steady_solver.cpp:578-580)."""
    s = harness.box_system(10, 10, 10, tet=True, seed=3)
    r = ref.solve(s, opts=ref.options(3, structure=1, pre_sweeps=sweeps, post_sweeps=sweeps),
                  rel_tol=1e-6, abs_tol=1e-12, max_iter=500)
    o = O.solve(s, opts=O.options(O.AMG_PCG, m_matrix=True, pre_sweeps=sweeps,
                                  post_sweeps=sweeps),
                rel_tol=1e-6, abs_tol=1e-12, max_iter=500)
    assert (o.iterations, o.converged) == (r.iterations, r.converged)
    assert (o.initial_residual, o.final_residual) == (r.initial_residual, r.final_residual)
    assert np.array_equal(o.x.view(np.uint32), r.x.view(np.uint32))
    assert o.describe == r.describe


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built on this machine")
@pytest.mark.parametrize("kind", [1, O.AMG_PCG], ids=["pcg_jacobi", "amg_pcg"])
def test_oracle_equals_reference_library_with_constant_nullspace(kind):
    """A pure-Neumann pressure system (constant null space projected at every
    level, test_solvers.cpp:102-115) with a compatible right-hand side."""
    import scipy.sparse as sp
    s = harness.poisson(12, 10, 6, 1, False, True)
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    s.b = (A @ harness.random_solution(s.n).astype(np.float64)).astype(np.float32)
    r = ref.solve(s, opts=ref.options(kind, nullspace=1), rel_tol=1e-6, abs_tol=1e-12,
                  max_iter=500)
    o = O.solve(s, kind, nullspace=True, rel_tol=1e-6, abs_tol=1e-12, max_iter=500)
    assert r.converged
    assert (o.iterations, o.converged) == (r.iterations, r.converged)
    assert (o.initial_residual, o.final_residual) == (r.initial_residual, r.final_residual)
    assert np.array_equal(o.x.view(np.uint32), r.x.view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built on this machine")
def test_oracle_equals_reference_library_on_a_graded_mesh():
    """The graded near-wall band (aspect 1000:1, D_f over [1e-6, 1]) where the
    FP32 solve stalls: the stall itself (iterations, final residual, best x)
    must be the reference's."""
    s = harness.box_system(12, 12, 12, tet=True, seed=4, band_layers=5, dmin=1e-6, dmax=1.0)
    r = ref.solve(s, opts=ref.options(3, structure=1), rel_tol=1e-8, abs_tol=1e-30, max_iter=300)
    o = O.solve(s, O.AMG_PCG, m_matrix=True, rel_tol=1e-8, abs_tol=1e-30, max_iter=300)
    assert (o.iterations, o.converged) == (r.iterations, r.converged)
    assert (o.initial_residual, o.final_residual) == (r.initial_residual, r.final_residual)
    assert np.array_equal(o.x.view(np.uint32), r.x.view(np.uint32))
