"""Solver parity on the GPU against the oracle (the C restatement of the
reference's path) and the golden fixtures generated from the reference itself:
iteration counts, convergence flags, residuals, solutions and the refreshed AMG
hierarchy; plus the reference's behavioural tests (refresh == fresh setup,
controls, breakdown honesty, best-iterate restore, Neumann projection, empty
systems) and size-independent properties at full size.

Tolerances: aggregates, coarse patterns, coarse values and L1 diagonals are
compared bit for bit. Iterates may differ from the oracle only through the
order of FP64 reduction trees (the oracle sums serially), which can move a
float-pair scalar by one unit in its low word; x is required to match within
relative 1e-5 at the returned residual and the residuals within 1e-3 relative
(the reference's own bar: rel 1e-5 on x at relative residual 1e-6, FP32)."""
import numpy as np
import pytest

import golden_cases as G
from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import kutta_oracle as O

pytestmark = pytest.mark.gpu
M = L.OperatorStructure.SymmetricMMatrix
XTOL = 1e-5


def run(system, kind, m_matrix=False, rel_tol=1e-6, abs_tol=1e-12, max_iter=2000, interval=8,
        amg=None, nullspace=False, refresh=True, b=None, x0=None):
    import torch
    a = L.upload(system)
    ns = L.NullSpace.Constant if nullspace else L.NullSpace.None_
    if amg is not None:
        solver = L.make_amg_solver(kind, system, amg)
    else:
        solver = L.make_solver(kind, system, L.SolverOptions(nullspace=ns,
                                                             structure=M if m_matrix else L.OperatorStructure.General))
    if refresh:
        solver.refresh(a)
    tb = torch.from_numpy(np.asarray(system.b if b is None else b, np.float32)).cuda()
    x = torch.zeros(system.n, device="cuda") if x0 is None else torch.from_numpy(np.asarray(x0, np.float32)).cuda()
    st = solver.solve(a, x, tb, L.SolveControl(rel_tol, abs_tol, max_iter, interval))
    torch.cuda.synchronize()
    return st, x.cpu().numpy(), solver


def rel_err(x, ref):
    return float(np.linalg.norm(x.astype(np.float64) - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.mark.parametrize("name", G.names())
def test_fixture_parity(cuda, name):
    meta, arrays = G.load(name)
    s = G.system(name)
    m_matrix = bool(meta["m_matrix"])
    amg = None
    if "options" in meta:  # make_amg_solver with the fixture's AmgOptions overrides
        amg = L.AmgOptions(structure=M if m_matrix else L.OperatorStructure.General,
                           **meta["options"])
    st, x, solver = run(s, L.SolverKind(meta["kind"]), m_matrix, meta["rel_tol"],
                        meta["abs_tol"], meta["max_iter"], amg=amg)
    assert solver.describe() == meta["describe"]
    assert st.iterations == meta["iterations"]
    assert st.converged == meta["converged"]
    assert st.initial_residual == pytest.approx(meta["initial_residual"], rel=1e-9)
    assert st.final_residual == pytest.approx(meta["final_residual"], rel=1e-3)
    if "x" in arrays:
        ref_x = arrays["x"].astype(np.float64)
        assert rel_err(x, ref_x) <= XTOL
        if m_matrix:
            # Error against an FP64 solution, stated for the GPU x and the
            # reference's x alike (FP32 AMG-PCG stops near its rounding floor).
            x64, _ = O.cg64(s, rel_tol=1e-13)
            print(f"{name}: it={st.iterations} |x-x_ref|/|x_ref|={rel_err(x, ref_x):.3e} "
                  f"|x-x64|/|x64|={rel_err(x, x64):.3e} |x_ref-x64|/|x64|="
                  f"{rel_err(arrays['x'], x64):.3e}")
    if meta["kind"] >= 3:
        levels = solver.levels()
        assert [lv[0] for lv in levels] == meta["levels"]
        for i, ((n, rp, cl, vl, l1, ag), sha) in enumerate(zip(levels, meta["level_sha"])):
            assert G.digest(rp) == sha["row_ptr"] and G.digest(cl) == sha["col"]
            assert G.digest(l1) == sha["l1"], f"L1 diagonal differs on level {i}"
            if i > 0:
                assert G.digest(vl) == sha["val"], f"Galerkin values differ on level {i}"
            if sha["aggregate"] is not None:
                assert G.digest(ag) == sha["aggregate"]


@pytest.mark.parametrize("name", G.hierarchy_names())
def test_scale_hierarchy_matches_reference(cuda, name):
    """The 5.3M-row tet pressure matrix: the hierarchy set up on the device
    (pairing, coarsening, Galerkin refresh) against the one the reference
    library sets up and refreshes on the same matrix (amg.cpp:200-256):
    level sizes, aggregates, coarse row pointers and columns, coarse values
    and L1 inverse diagonals, all bit for bit through their SHA-256 digests."""
    import torch
    meta, _ = G.load(name)
    s = G.system(name)
    opts = L.AmgOptions(structure=M if meta["m_matrix"] else L.OperatorStructure.General,
                        **meta["options"])
    a = L.upload(s)
    solver = L.make_amg_solver(L.SolverKind(meta["kind"]), s, opts)
    solver.refresh(a)
    torch.cuda.synchronize()
    levels = solver.levels()
    assert [lv[0] for lv in levels] == meta["levels"]
    for i, ((n, rp, cl, vl, l1, ag), sha) in enumerate(zip(levels, meta["level_sha"])):
        assert int(rp[-1]) == meta["level_nnz"][i]
        assert G.digest(rp) == sha["row_ptr"], f"row pointers differ on level {i}"
        assert G.digest(cl) == sha["col"], f"columns differ on level {i}"
        if i > 0:  # level 0's values are the caller's matrix
            assert G.digest(vl) == sha["val"], f"values differ on level {i}"
        assert G.digest(l1) == sha["l1"], f"L1 diagonal differs on level {i}"
        if sha["aggregate"] is not None:
            assert G.digest(ag) == sha["aggregate"], f"aggregates differ on level {i}"


ORACLE_CASES = [
    ("hex24_pressure", lambda: harness.box_system(24, 24, 24, tet=False, seed=31), 3, True),
    ("tet16_pressure", lambda: harness.box_system(16, 16, 16, tet=True, seed=32), 3, True),
    ("tet16_graded", lambda: harness.box_system(16, 16, 16, tet=True, seed=33, band_layers=4,
                                                dmin=1e-6, dmax=1.0), 3, True),
    ("tet14_convection", lambda: harness.box_system(14, 14, 14, tet=True, seed=34,
                                                    convection=1e-3), 4, False),
]


@pytest.mark.parametrize("name,make,kind,m", ORACLE_CASES, ids=[c[0] for c in ORACLE_CASES])
def test_oracle_parity(cuda, name, make, kind, m):
    s = make()
    st, x, solver = run(s, L.SolverKind(kind), m)
    o = O.solve(s, kind, m_matrix=m, rel_tol=1e-6, abs_tol=1e-12, max_iter=2000)
    assert solver.describe() == o.describe
    assert st.iterations == o.iterations
    assert st.converged == o.converged
    assert st.final_residual == pytest.approx(o.final_residual, rel=1e-3)
    assert rel_err(x, o.x.astype(np.float64)) <= XTOL
    # Error against an FP64 solution, stated (not bounded: plain FP32 may stall).
    if kind == 3:
        x64, _ = O.cg64(s, rel_tol=1e-13)
    else:
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n)).tocsc()
        x64 = spl.spsolve(A, s.b.astype(np.float64))
    print(f"{name}: it={st.iterations} rel={st.final_residual / st.initial_residual:.3e} "
          f"|x-x64|/|x64|={rel_err(x, x64):.3e}")


def test_refresh_equals_fresh_setup(cuda):
    """test_solvers.cpp:145-175: refresh after a value change gives the same
    iterations, residual and x as a solver set up from the new values."""
    import torch
    s = harness.poisson(14, 13, 8)
    scaled = harness.HostSystem(s.row_ptr, s.col, s.diag, s.val.copy(), s.b.copy())
    scaled.val = (scaled.val * 1.37).astype(np.float32).astype(np.float64)
    h = harness.ref_hash_array(np.arange(s.n))
    scaled.val[s.diag] = (scaled.val[s.diag] + 0.031 * (1 + h % 17)).astype(np.float32)
    import scipy.sparse as sp
    A = sp.csr_matrix((scaled.val, s.col, s.row_ptr), shape=(s.n, s.n))
    b = (A @ harness.random_solution(s.n).astype(np.float64)).astype(np.float32)
    a = L.upload(s)
    solver = L.make_amg_solver(L.SolverKind.AmgPcg, s, L.AmgOptions())
    a.val.copy_(torch.from_numpy(scaled.val.astype(np.float32)).cuda())
    solver.refresh(a)
    fresh = L.make_amg_solver(L.SolverKind.AmgPcg, scaled, L.AmgOptions())
    tb = torch.from_numpy(b).cuda()
    x = torch.zeros(s.n, device="cuda")
    y = torch.zeros(s.n, device="cuda")
    st = solver.solve(a, x, tb, L.SolveControl(1e-6, 1e-12, 400))
    ft = fresh.solve(a, y, tb, L.SolveControl(1e-6, 1e-12, 400))
    assert st.converged and ft.converged and st.iterations == ft.iterations
    assert st.final_residual == ft.final_residual
    assert torch.equal(x, y)


def test_controls_and_breakdown_are_truthful(cuda):
    """test_solvers.cpp:117-143."""
    import torch
    s = harness.poisson(5, 4)
    a = L.upload(s)
    solver = L.make_solver(L.SolverKind.PcgJacobi, s)
    x = torch.zeros(s.n, device="cuda")
    b = torch.zeros(s.n, device="cuda")
    assert solver.solve(a, x, b).iterations == 0
    assert solver.solve(a, x, b).converged
    b.fill_(1)
    st = solver.solve(a, x, b, L.SolveControl(0, 0, 0))
    assert st.iterations == 0 and not st.converged
    assert st.final_residual == pytest.approx(np.sqrt(s.n))
    assert solver.solve(a, x, b, L.SolveControl(0, 10, 0)).converged
    with pytest.raises(L.KuttaError):
        solver.solve(a, x, b, L.SolveControl(-1, 0, 10))
    x.fill_(0.5)
    assert solver.solve(a, x, b, L.SolveControl(1e-5, 1e-10, 100)).converged
    neg = harness.poisson(5, 4)
    neg.val = -neg.val
    an = L.upload(neg)
    solver.refresh(an)
    x.zero_()
    st = solver.solve(an, x, b)
    assert not st.converged and np.isfinite(st.final_residual)
    an.val.zero_()
    with pytest.raises(L.KuttaError):
        solver.refresh(an)


def test_best_iterate_restored_on_divergence(cuda):
    """test_solvers.cpp:467-483: a violated SPD contract returns the best
    verified iterate (x = 0) and a truthful residual."""
    import torch
    bad = harness.HostSystem(np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                             np.array([0, 3], np.int32), np.array([1, 999999, -999998, 1.0]),
                             np.array([1, 1], np.float32))
    for kind in (L.SolverKind.PcgJacobi, L.SolverKind.BicgstabJacobi):
        st, x, _ = run(bad, kind, rel_tol=1e-8, abs_tol=0, max_iter=8)
        assert not st.converged
        assert st.final_residual <= st.initial_residual
        assert x.tolist() == [0, 0]
        assert st.iterations == 1


def test_nonfinite_rhs_raises_nonfinite_error(cuda):
    s = harness.poisson(6, 5)
    b = np.ones(s.n, np.float32)
    b[3] = np.nan
    with pytest.raises(L.NonfiniteError):
        run(s, L.SolverKind.AmgPcg, b=b)


@pytest.mark.parametrize("kind", [1, 3])
def test_neumann_projection(cuda, kind):
    """test_solvers.cpp:102-115, 409-448: constant nullspace projected; an
    incompatible RHS is rejected."""
    s = harness.poisson(8, 7, 1, 1, False, True)
    f = np.zeros(s.n, np.float32)
    f[0], f[-1] = 1, -1
    st, x, solver = run(s, L.SolverKind(kind), rel_tol=2e-6, max_iter=2000, nullspace=True, b=f)
    assert "nullspace" in solver.describe()
    assert st.converged and abs(float(x.astype(np.float64).sum())) < 1e-5
    o = O.solve(s, kind, nullspace=True, b=f, rel_tol=2e-6, max_iter=2000)
    assert st.iterations == o.iterations
    assert rel_err(x, o.x.astype(np.float64)) <= XTOL
    with pytest.raises(L.KuttaError, match="incompatible RHS"):
        run(s, L.SolverKind(kind), nullspace=True, b=np.ones(s.n, np.float32), x0=np.full(s.n, 4.0))


def test_empty_system(cuda):
    import torch
    e = harness.HostSystem(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                           np.zeros(0), np.zeros(0, np.float32))
    for kind in range(5):
        solver = L.make_solver(L.SolverKind(kind), e)
        a = L.upload(e)
        st = solver.solve(a, torch.zeros(0, device="cuda"), torch.zeros(0, device="cuda"))
        assert st.converged and st.iterations == 0 and st.final_residual == 0


def test_large_pressure_properties(cuda):
    """A 48^3 x 6-tet pressure matrix (663,552 rows): the device hierarchy after
    refresh equals the host-built one bit for bit; the reported residual equals
    the FP64 true residual of the returned x; repeated solves are bitwise
    deterministic."""
    s = harness.box_system(48, 48, 48, tet=True, seed=9)
    st, x, solver = run(s, L.SolverKind.AmgPcg, True, max_iter=400)
    host = L.build_hierarchy(s, L.AmgOptions(structure=M))
    dev = solver.levels()
    assert [d[0] for d in dev] == [h.n for h in host]
    for (n, rp, cl, vl, l1, ag), h in zip(dev[1:], host[1:]):
        assert np.array_equal(cl, h.col) and np.array_equal(vl.view(np.uint32), h.val.view(np.uint32))
        assert np.array_equal(l1.view(np.uint32), h.inverse_l1.view(np.uint32))
    true = O.true_residual(s, x)
    assert true == pytest.approx(st.final_residual, rel=1e-4)
    st2, x2, _ = run(s, L.SolverKind.AmgPcg, True, max_iter=400)
    assert st2.iterations == st.iterations and np.array_equal(x.view(np.uint32), x2.view(np.uint32))
