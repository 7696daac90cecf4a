"""The mixed-precision solve (no reference counterpart).

CPU: its hierarchy (pairing with singleton absorption) equals the oracle's
restatement bit for bit and reaches the dense size where the reference's
pairing stalls. GPU: it converges below the FP32 rounding floor, measured by the
FP64 true residual of the returned FP64 solution and by the error against the
FP64 CG oracle."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import kutta_oracle as O


def _oracle_levels(s, dense_rows=112):
    o = O.Solver(s, O.options(O.AMG_PCG, pre_sweeps=2, post_sweeps=2, coarse_rows=dense_rows,
                              m_matrix=True, absorb=True))
    return o.levels()


@pytest.mark.parametrize("seed,tet", [(1, True), (2, False)])
def test_mixed_hierarchy_matches_oracle(seed, tet):
    s = harness.box_system(20, 20, 20, tet=tet, seed=seed)
    mine = L.build_mixed_hierarchy(s)
    theirs = _oracle_levels(s)
    assert [m.n for m in mine] == [t["n"] for t in theirs]
    assert mine[-1].n <= 112
    for i, (m, t) in enumerate(zip(mine, theirs)):
        assert np.array_equal(m.row_ptr, t["row_ptr"]) and np.array_equal(m.col, t["col"])
        if i > 0:
            assert np.array_equal(m.val.view(np.uint32), t["val"].view(np.uint32))
        assert np.array_equal(m.inverse_l1.view(np.uint32), t["l1"].view(np.uint32))
        if t["aggregate"] is not None:
            assert np.array_equal(m.aggregate, t["aggregate"])


def test_absorption_removes_the_stall():
    """The reference's pairing stops coarsening at a large level on random
    coefficients; absorption keeps coarsening down to the dense size."""
    s = harness.box_system(24, 24, 24, tet=True, seed=3)
    plain = L.build_hierarchy(s, L.AmgOptions(structure=L.OperatorStructure.SymmetricMMatrix,
                                              coarse_rows=512))
    mixed = L.build_mixed_hierarchy(s)
    assert plain[-1].n > 2000
    assert mixed[-1].n <= 112
    assert sum(lv.row_ptr[-1] for lv in mixed) < sum(lv.row_ptr[-1] for lv in plain)


def _fp64_true(s, x64, b):
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    return float(np.linalg.norm(b.astype(np.float64) - A @ x64))


CASES = [
    ("hex20", lambda: harness.box_system(20, 20, 20, tet=False, seed=5), 1e-6),
    ("tet16", lambda: harness.box_system(16, 16, 16, tet=True, seed=6), 1e-6),
    ("tet16_graded_1e-8", lambda: harness.box_system(16, 16, 16, tet=True, seed=7, band_layers=6,
                                                     dmin=1e-6, dmax=1.0), 1e-8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,tol", CASES, ids=[c[0] for c in CASES])
def test_mixed_converges_below_fp32_floor(cuda, name, make, tol):
    import torch
    s = make()
    solver = L.make_mixed_solver(s)
    a = L.upload(s)
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    st = solver.solve(a, x, b, L.SolveControl(tol, 1e-30, 3000))
    torch.cuda.synchronize()
    xr = x.cpu().numpy()
    true = _fp64_true(s, xr, s.b)
    assert st.converged, st
    assert true <= tol * st.initial_residual * 1.0001
    assert true == pytest.approx(st.final_residual, rel=1e-3)
    x64, _ = O.cg64(s, rel_tol=1e-14)
    err = np.linalg.norm(xr - x64) / np.linalg.norm(x64)
    # A float32 x cannot reach this residual: the rounded exact solution sits above it.
    floor = _fp64_true(s, x64.astype(np.float32).astype(np.float64), s.b) / st.initial_residual
    print(f"{name}: refinements={st.refinements} inner iterations={st.iterations} "
          f"rel={true / st.initial_residual:.2e} |x-x64|/|x64|={err:.2e} fp32 floor={floor:.2e}")
    assert err < 1e-3


@pytest.mark.gpu
def test_mixed_refresh_tracks_new_values(cuda):
    """After a value change and refresh the solve meets the tolerance for the
    new matrix (BF16 copies and the dense inverse are rebuilt)."""
    import torch
    s = harness.box_system(14, 14, 14, tet=True, seed=8)
    solver = L.make_mixed_solver(s)
    a = L.upload(s)
    scaled = s.val * 1.5
    scaled[s.diag] += 0.01 * np.abs(s.val[s.diag])
    a.val.copy_(torch.from_numpy(scaled.astype(np.float32)))
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    st = solver.solve(a, x, b, L.SolveControl(1e-7, 1e-30, 2000))
    t = harness.HostSystem(s.row_ptr, s.col, s.diag, scaled.astype(np.float32).astype(np.float64), s.b)
    assert st.converged
    assert _fp64_true(t, x.cpu().numpy(), s.b) <= 1e-7 * st.initial_residual * 1.0001


def _coarsest(n_side=6, seed=4):
    s = harness.box_system(n_side, n_side, n_side, tet=True, seed=seed)
    return s


DENSE_SYSTEMS = {
    # Up to 112 rows the factor and inverse live in shared memory; up to 236
    # rows the packed lower triangle does, inverted in place; above, a blocked
    # Cholesky, block inverse and Gram product over many CTAs (32-row blocks:
    # 237, 384 and 750 rows leave ragged last blocks).
    "tet2_48": lambda: _coarsest(2),
    "poisson_112": lambda: harness.poisson(7, 4, 4),
    "poisson_113": lambda: harness.poisson(113, 1, 1),
    "poisson_236": lambda: harness.poisson(59, 4, 1),
    "poisson_237": lambda: harness.poisson(79, 3, 1),
    "tet3_162": lambda: _coarsest(3),
    "tet4_384": lambda: _coarsest(4),
    "tet5_750": lambda: _coarsest(5),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(DENSE_SYSTEMS))
def test_dense_inverse_matches_fp64(cuda, name):
    """The coarsest-level dense FP64 Cholesky inverse against numpy in FP64."""
    import torch
    s = DENSE_SYSTEMS[name]()
    n = s.n
    assert n <= 1024
    a = L.upload(s)
    inv = torch.empty(n * n, dtype=torch.float64, device="cuda")
    flag = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    L.dense_inverse(a, inv, flag)
    torch.cuda.synchronize()
    assert flag.item() == 0.0
    dense = np.zeros((n, n))
    for i in range(n):
        for j in range(s.row_ptr[i], s.row_ptr[i + 1]):
            dense[i, s.col[j]] = np.float32(s.val[j])
    got = inv.cpu().numpy().reshape(n, n)
    want = np.linalg.inv(dense)
    assert np.max(np.abs(got - want)) <= 1e-9 * np.max(np.abs(want))


@pytest.mark.gpu
@pytest.mark.parametrize("n_side", [2, 3, 4])
def test_dense_inverse_flags_non_spd(cuda, n_side):
    import torch
    s = _coarsest(n_side)
    bad = s.val.copy()
    bad[s.diag[0]] = -1.0
    a = L.upload(harness.HostSystem(s.row_ptr, s.col, s.diag, bad, s.b))
    inv = torch.empty(s.n * s.n, dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.dense_inverse(a, inv, flag)
    torch.cuda.synchronize()
    assert flag.item() == 1.0


@pytest.mark.gpu
def test_mixed_rejects_nonfinite_rhs(cuda):
    import torch
    s = harness.box_system(6, 6, 6, tet=True, seed=1)
    solver = L.make_mixed_solver(s)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    b[3] = float("nan")
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    with pytest.raises(L.NonfiniteError):
        solver.solve(a, x, b)


def _v11():
    return L.AmgOptions(pre_sweeps=1, post_sweeps=1, structure=L.OperatorStructure.SymmetricMMatrix)


def _default_amg():
    return L.MixedOptions().amg


FUSED_CASES = [
    # V-cycle: the tail starts at level 1.
    ("tet16_v", lambda: harness.box_system(16, 16, 16, tet=True, seed=6), _v11),
    ("hex24_v", lambda: harness.box_system(24, 24, 24, tet=False, seed=12), _v11),
    # Default K-cycle with the inner step on level 1: the tail starts below it.
    # (Well conditioned on purpose: over hundreds of iterations the different
    # summation orders of the two forms drift apart without either being wrong.)
    ("tet40_k", lambda: harness.box_system(40, 40, 40, tet=True, seed=13), _default_amg),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,amg", FUSED_CASES, ids=[c[0] for c in FUSED_CASES])
def test_fused_coarse_levels_match_separate_launches(cuda, name, make, amg):
    """The small coarse levels as one thread-block-cluster launch give the same
    solve as their separate BF16 kernels: same convergence, iteration counts
    within one, and both solutions within the tolerance of the FP64 oracle."""
    import torch
    s = make()
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    results = {}
    for fused in (True, False):
        solver = L.make_mixed_solver(s, L.MixedOptions(amg=amg(), fused_coarse=fused))
        assert ("cluster launch" in solver.describe()) == fused, solver.describe()
        solver.refresh(a)
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
        torch.cuda.synchronize()
        assert st.converged, (fused, st)
        xr = x.cpu().numpy()
        assert _fp64_true(s, xr, s.b) <= 1e-8 * st.initial_residual * 1.0001
        results[fused] = (st, xr)
    (sf, xf), (su, xu) = results[True], results[False]
    assert abs(sf.iterations - su.iterations) <= max(1, su.iterations // 20), (sf, su)
    x64, _ = O.cg64(s, rel_tol=1e-14)
    for xr in (xf, xu):
        assert np.linalg.norm(xr - x64) / np.linalg.norm(x64) < 1e-5


PACKED_CASES = [
    # Tets: at most 4 off-diagonal entries per row (packed width 4).
    ("tet40", lambda: harness.box_system(40, 40, 40, tet=True, seed=13)),
    # Hexes: 6 off-diagonal entries (width 8, two slots unused).
    ("hex32", lambda: harness.box_system(32, 32, 32, tet=False, seed=15)),
    ("tet24_graded", lambda: harness.box_system(24, 24, 24, tet=True, seed=16, band_layers=6,
                                                dmin=1e-6, dmax=1.0)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", PACKED_CASES, ids=[c[0] for c in PACKED_CASES])
def test_packed_fine_rows_give_the_csr_results_bitwise(cuda, name, make):
    """The fine level's packed rows (diagonal apart, 16-bit column offsets)
    visit each row's terms in CSR column order with the same arithmetic,
    grids and reductions: the mixed solve's statistics and FP64 solution equal
    the CSR kernels' bit for bit, through refresh and two solves."""
    import torch
    s = make()
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    out = {}
    for packed in (True, False):
        solver = L.make_mixed_solver(s, L.MixedOptions(packed_rows=packed))
        assert ("packed fine rows" in solver.describe()) == packed, solver.describe()
        solver.refresh(a)
        runs = []
        for _ in range(2):
            x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
            torch.cuda.synchronize()
            runs.append((st, x.cpu().numpy()))
        out[packed] = runs
    for (sp, xp), (sc, xc) in zip(out[True], out[False]):
        assert (sp.refinements, sp.iterations, sp.converged) == (sc.refinements, sc.iterations,
                                                                 sc.converged)
        assert (sp.initial_residual, sp.final_residual) == (sc.initial_residual, sc.final_residual)
        assert np.array_equal(xp.view(np.uint64), xc.view(np.uint64))
    assert out[True][0][0].converged


@pytest.mark.gpu
@pytest.mark.parametrize("k_levels", [1, 0], ids=["k_cycle_level1", "k_cycle_all"])
def test_cuda_graph_replay_is_bitwise_identical(cuda, k_levels):
    """Captured-graph replay runs the same kernels with the same arguments as
    direct launches: equal statistics and a bitwise-equal FP64 solution, over
    two solves (the second replays graphs captured by the first)."""
    import torch
    s = harness.box_system(24, 24, 24, tet=True, seed=14)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    out = {}
    for graphs in (True, False):
        solver = L.make_mixed_solver(s, L.MixedOptions(cuda_graphs=graphs, k_cycle_levels=k_levels))
        solver.refresh(a)
        runs = []
        for _ in range(2):
            x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 2000))
            torch.cuda.synchronize()
            runs.append((st, x.cpu().numpy()))
        out[graphs] = runs
    for (sg, xg), (sd, xd) in zip(out[True], out[False]):
        assert sg == sd
        assert np.array_equal(xg.view(np.uint64), xd.view(np.uint64))


@pytest.mark.gpu
def test_fused_post_sweep_reductions_are_exact(cuda):
    """The flexible PCG's r.z and z.q ride on the fine post-sweep when nothing
    changes z after it. A learned stage with all-zero weights turns that
    fusion off (it acts after the cycle) but adds nothing to z (G = 0, step
    0), so the fused and the unfused solves must agree bit for bit."""
    import torch
    s = harness.box_system(20, 20, 20, tet=True, seed=15)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    out = []
    for zero_stage in (False, True):
        solver = L.make_mixed_solver(s)
        solver.refresh(a)
        if zero_stage:
            g = L.LearnedStage(seed=1)
            g.set_weights(np.zeros(L.LearnedStage.parameter_count(), np.float32))
            solver.set_learned(g, L.LEARNED_CYCLE)
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
        out.append((st.iterations, st.final_residual, x.cpu().numpy()))
        if zero_stage:
            solver.set_learned(None)
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2].view(np.uint64), out[1][2].view(np.uint64))


@pytest.mark.gpu
def test_fp32_solution_is_the_rounded_fp64_solution(cuda):
    """b2_mixed_solve_f32, the form LinearSolver.solve has (x in FP32): the same
    solve as b2_mixed_solve from the widened guess, with the FP64 solution
    rounded to nearest on return."""
    import torch
    s = harness.box_system(16, 16, 16, tet=True, seed=6)
    solver = L.make_mixed_solver(s)
    a = L.upload(s)
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    rng = np.random.default_rng(3)
    for guess in (np.zeros(s.n, np.float32), rng.normal(size=s.n).astype(np.float32)):
        x64 = torch.from_numpy(guess.astype(np.float64)).cuda()
        st64 = solver.solve(a, x64, b, L.SolveControl(1e-6, 1e-30, 2000))
        x32 = torch.from_numpy(guess.copy()).cuda()
        st32 = solver.solve(a, x32, b, L.SolveControl(1e-6, 1e-30, 2000))
        torch.cuda.synchronize()
        assert st64.converged
        assert (st32.refinements, st32.iterations, st32.converged) == \
            (st64.refinements, st64.iterations, st64.converged)
        assert (st32.initial_residual, st32.final_residual) == \
            (st64.initial_residual, st64.final_residual)
        rounded = x64.cpu().numpy().astype(np.float32)
        assert np.array_equal(x32.cpu().numpy().view(np.uint32), rounded.view(np.uint32))
