"""GPU solves against the reference's own CPU path (oracle/_ref, built from the
reference sources): iteration counts, residuals and solutions, for every solver
kind, on the reference's own test matrices and on synthetic pressure systems."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import ref

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

M = L.OperatorStructure.SymmetricMMatrix


def _solve_gpu(system, kind, amg_options=None, solver_options=None, rel_tol=1e-6, abs_tol=1e-12,
               max_iter=2000, interval=8, x0=None):
    import torch
    a = L.upload(system)
    if amg_options is not None:
        solver = L.make_amg_solver(kind, system, amg_options)
    else:
        solver = L.make_solver(kind, system, solver_options)
    solver.refresh(a)
    b = torch.from_numpy(system.b).cuda()
    x = torch.zeros(system.n, dtype=torch.float32, device="cuda") if x0 is None else \
        torch.from_numpy(np.asarray(x0, np.float32)).cuda()
    st = solver.solve(a, x, b, L.SolveControl(rel_tol, abs_tol, max_iter, interval))
    torch.cuda.synchronize()
    solver._matrix = a  # level 0's values are the caller's matrix: keep it alive
    return st, x.cpu().numpy(), solver


def _compare(st, x, r, xtol=1e-5):
    assert st.iterations == r.iterations
    assert st.converged == r.converged
    assert st.initial_residual == pytest.approx(r.initial_residual, rel=1e-9)
    assert st.final_residual == pytest.approx(r.final_residual, rel=1e-3)
    err = np.linalg.norm(x.astype(np.float64) - r.x) / max(np.linalg.norm(r.x), 1e-300)
    assert err <= xtol, err
    return err


CASES = [
    ("poisson32_random_forcing", lambda: _forced(harness.poisson(32, 32, 32)), 3, False),
    ("poisson_aniso1000", lambda: _rhs(harness.poisson(12, 9, 5, 1000)), 3, False),
    ("poisson_random2d", lambda: _rhs(harness.poisson(8, 7, 1, 1, True)), 3, False),
    ("hex16_pressure", lambda: harness.box_system(16, 16, 16, tet=False, seed=5), 3, True),
    ("tet12_pressure", lambda: harness.box_system(12, 12, 12, tet=True, seed=7), 3, True),
    ("poisson_wind3_bicg", lambda: _rhs(harness.poisson(20, 18, 1, 1, False, False, 3)), 4, False),
    ("tet10_convection_bicg", lambda: harness.box_system(10, 10, 10, tet=True, seed=2,
                                                          convection=1e-3), 4, False),
]


def _forced(s):
    s.b = harness.random_forcing(s.n)
    return s


def _rhs(s):
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    x = harness.random_solution(s.n).astype(np.float64)
    s.b = (A @ x).astype(np.float32)
    return s


@needs_ref
@pytest.mark.parametrize("name,make,kind,m_matrix", CASES, ids=[c[0] for c in CASES])
def test_amg_matches_reference(cuda, name, make, kind, m_matrix):
    s = make()
    opts = L.AmgOptions(structure=M if m_matrix else L.OperatorStructure.General)
    st, x, solver = _solve_gpu(s, L.SolverKind(kind), amg_options=opts)
    r = ref.solve(s, opts=ref.options(kind, structure=int(m_matrix)), rel_tol=1e-6, abs_tol=1e-12,
                  max_iter=2000)
    assert solver.describe() == r.describe
    _compare(st, x, r)


@needs_ref
@pytest.mark.parametrize("sweeps", [1, 2], ids=["V11", "V22"])
@pytest.mark.parametrize("make,kind,m_matrix", [
    (lambda: harness.box_system(12, 12, 12, tet=True, seed=7), 3, True),
    (lambda: harness.pressure_hex32(1), 3, True),
    (lambda: _rhs(harness.poisson(20, 18, 1, 1, False, False, 3)), 4, False),
], ids=["tet12_pcg", "hex32_pcg", "poisson_wind3_bicg"])
def test_other_sweep_counts_match_reference(cuda, make, kind, m_matrix, sweeps):
    """V(1,1), where the single zero-start pre-sweep and the residual run as one
    fused pass, and V(2,2), the pressure solver of the SST configuration
    (src/kutta/fv/steady_solver.cpp:575-578): iterations, residuals and x must
    still be the reference's."""
    s = make()
    opts = L.AmgOptions(pre_sweeps=sweeps, post_sweeps=sweeps,
                        structure=M if m_matrix else L.OperatorStructure.General)
    st, x, solver = _solve_gpu(s, L.SolverKind(kind), amg_options=opts)
    r = ref.solve(s, opts=ref.options(kind, structure=int(m_matrix), pre_sweeps=sweeps,
                                      post_sweeps=sweeps),
                  rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert solver.describe() == r.describe
    _compare(st, x, r)


@needs_ref
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_jacobi_kinds_match_reference(cuda, kind):
    s = _rhs(harness.poisson(16, 12, 8, 1, False, False, 5 if kind == 2 else 0))
    st, x, solver = _solve_gpu(s, L.SolverKind(kind), rel_tol=1e-5, max_iter=500)
    r = ref.solve(s, opts=ref.options(kind), rel_tol=1e-5, abs_tol=1e-12, max_iter=500)
    assert solver.describe() == r.describe
    _compare(st, x, r)


@needs_ref
def test_device_hierarchy_matches_reference_bitwise(cuda):
    s = harness.box_system(16, 16, 16, tet=True, seed=11)
    opts = L.AmgOptions(structure=M)
    st, x, solver = _solve_gpu(s, L.SolverKind.AmgPcg, amg_options=opts, max_iter=1)
    mine = solver.levels()
    theirs = ref.hierarchy(s, ref.options(structure=1))
    assert len(mine) == len(theirs)
    for (n, rp, cl, vl, l1, ag), r in zip(mine, theirs):
        assert n == r.n
        assert np.array_equal(rp, r.row_ptr) and np.array_equal(cl, r.col)
        assert np.array_equal(vl.view(np.uint32), r.val.view(np.uint32))
        assert np.array_equal(l1.view(np.uint32), r.l1.view(np.uint32))
        if r.aggregate is not None:
            assert np.array_equal(ag, r.aggregate)


def _neumann_forcing(s):
    """Integer-valued compatible forcing (tests/linalg/test_solvers.cpp:20-23)."""
    s.b = np.zeros(s.n, np.float32)
    s.b[0], s.b[-1] = 1.0, -1.0
    return s


K_CASES = [
    # test_solvers.cpp:97-98: K-cycle AMG-BiCGStab on the upwind Poisson matrix.
    ("poisson_wind3_bicg", lambda: _rhs(harness.poisson(20, 18, 1, 1, False, False, 3)), 4,
     False, False),
    # test_solvers.cpp:146-151: K-cycle AMG-PCG on poisson(14, 13, 8).
    ("poisson14x13x8", lambda: _rhs(harness.poisson(14, 13, 8)), 3, False, False),
    # test_solvers.cpp:634-647: K-cycle with the constant-nullspace projection.
    ("poisson12x10x4_neumann", lambda: _neumann_forcing(harness.poisson(12, 10, 4, 1, False, True)),
     3, False, True),
    ("poisson32_random_forcing", lambda: _forced(harness.poisson(32, 32, 32)), 3, False, False),
    ("hex16_pressure", lambda: harness.box_system(16, 16, 16, tet=False, seed=5), 3, True, False),
    ("tet12_pressure", lambda: harness.box_system(12, 12, 12, tet=True, seed=7), 3, True, False),
    ("tet10_convection_bicg", lambda: harness.box_system(10, 10, 10, tet=True, seed=2,
                                                          convection=1e-3), 4, False, False),
]


@needs_ref
@pytest.mark.parametrize("name,make,kind,m_matrix,neumann", K_CASES, ids=[c[0] for c in K_CASES])
def test_k_cycle_matches_reference(cuda, name, make, kind, m_matrix, neumann):
    """amg.cpp:283-338: the K-cycle's two inner Krylov corrections per coarse
    level (flexible CG for SPD, GCR otherwise), against the reference library."""
    s = make()
    opts = L.AmgOptions(cycle=L.AmgCycle.K,
                        structure=M if m_matrix else L.OperatorStructure.General,
                        nullspace=L.NullSpace.Constant if neumann else L.NullSpace.None_)
    st, x, solver = _solve_gpu(s, L.SolverKind(kind), amg_options=opts)
    r = ref.solve(s, opts=ref.options(kind, cycle=1, structure=int(m_matrix), nullspace=int(neumann)),
                  rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert "K-cycle" in r.describe
    assert solver.describe() == r.describe
    _compare(st, x, r)
