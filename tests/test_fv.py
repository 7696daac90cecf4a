"""The finite-volume steps on either side of the pressure solve
(src/kutta/kernels/fv_flow.kern.h:164-201): the C restatement against the
reference's own kernels (CPU), the CUDA kernels against both (bit for bit),
and the assembly fused with the solver's refresh against assembly followed
by a separate refresh."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L
from oracle import fv, ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

SYSTEMS = [
    ("tet8", lambda: harness.box_system(8, 8, 8, tet=True, seed=3)),
    ("hex10", lambda: harness.box_system(10, 10, 10, tet=False, seed=4)),
    ("graded_tet8", lambda: harness.box_system(8, 8, 8, tet=True, seed=5, band_layers=4,
                                               aspect=1000.0, ratio=1.2, dmin=1e-6, dmax=1.0)),
]


def _case(make, seed, reference=-1):
    s = make()
    if reference == "middle":
        reference = s.n // 2
    elif reference == "last":
        reference = s.n - 1
    return s, harness.fv_faces(s.row_ptr, s.col, s.diag, seed=seed, reference=reference)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _velocity_inputs(n, seed):
    rng = np.random.default_rng(seed)
    pos = lambda: rng.uniform(0.1, 2.0, n).astype(np.float32)  # noqa: E731
    g = [rng.normal(size=n).astype(np.float32) for _ in range(3)]
    uvwp = [rng.normal(size=n).astype(np.float32) for _ in range(4)]
    return pos(), pos(), pos(), g, rng.normal(size=n).astype(np.float32), uvwp


@needs_ref
@pytest.mark.parametrize("reference", [-1, 0, "middle", "last"])
@pytest.mark.parametrize("name,make", SYSTEMS, ids=[c[0] for c in SYSTEMS])
def test_oracle_assembly_matches_reference(name, make, reference):
    s, c = _case(make, seed=11, reference=reference)
    v1 = np.full(len(s.col), 3.0, np.float32)
    r1 = np.zeros(s.n, np.float32)
    v2, r2 = v1.copy(), r1.copy()
    fv.oracle_assemble(c, v1, r1)
    fv.ref_assemble(c, v2, r2)
    assert np.array_equal(_bits(v1), _bits(v2)) and np.array_equal(_bits(r1), _bits(r2))


@needs_ref
def test_oracle_corrections_match_reference():
    s, c = _case(SYSTEMS[0][1], seed=12)
    rng = np.random.default_rng(5)
    correction = rng.normal(size=s.n).astype(np.float32)
    f1 = c.flux.copy()
    f2 = c.flux.copy()
    fv.oracle_correct_flux(c, correction, f1)
    fv.ref_correct_flux(c, correction, f2)
    assert np.array_equal(_bits(f1), _bits(f2))
    volume, inverse, diagonal, g, corr, uvwp = _velocity_inputs(s.n, 6)
    a = [x.copy() for x in uvwp]
    b = [x.copy() for x in uvwp]
    fv.oracle_correct_velocity(s.n, volume, inverse, diagonal, g, corr, a, 0.3)
    fv.ref_correct_velocity(s.n, volume, inverse, diagonal, g, corr, b, 0.3)
    for x, y in zip(a, b):
        assert np.array_equal(_bits(x), _bits(y))


def test_assembled_matrix_is_a_symmetric_m_matrix():
    import scipy.sparse as sp
    for reference in (-1, "middle"):
        s, c = _case(SYSTEMS[0][1], seed=13, reference=reference)
        v = np.zeros(len(s.col), np.float32)
        r = np.zeros(s.n, np.float32)
        fv.oracle_assemble(c, v, r)
        A = sp.csr_matrix((v.astype(np.float64), s.col, s.row_ptr), shape=(s.n, s.n))
        assert abs(A - A.T).max() == 0
        assert (A - sp.diags(A.diagonal())).max() <= 0
        assert A.sum(axis=1).min() >= 0
        if reference != -1:
            # The eliminated cell: a unit row, its column removed, zero rhs.
            k = s.n // 2
            row = A.getrow(k).toarray().ravel()
            column = A.getcol(k).toarray().ravel()
            assert row[k] == 1 and np.count_nonzero(row) == 1 and np.count_nonzero(column) == 1
            assert r[k] == 0


def _device_fv(c):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return L.FvPressure(t(c.offsets), t(c.faces), t(c.sign), t(c.adjacent), t(c.entry),
                        t(c.coefficient), t(c.flux), int(c.reference))


@pytest.mark.gpu
@pytest.mark.parametrize("reference", [-1, "middle"])
@pytest.mark.parametrize("name,make", SYSTEMS + [
    ("tet40", lambda: harness.box_system(40, 40, 40, tet=True, seed=7))],
    ids=[c[0] for c in SYSTEMS] + ["tet40"])
def test_device_assembly_matches_oracle(cuda, name, make, reference):
    import torch
    s, c = _case(make, seed=21, reference=reference)
    a = L.upload(s)
    a.val.fill_(3.0)
    rhs = torch.zeros(s.n, device="cuda")
    L.fv_pressure_assemble(a, _device_fv(c), rhs)
    v = np.full(len(s.col), 3.0, np.float32)
    r = np.zeros(s.n, np.float32)
    fv.oracle_assemble(c, v, r)
    assert np.array_equal(_bits(a.val.cpu().numpy()), _bits(v))
    assert np.array_equal(_bits(rhs.cpu().numpy()), _bits(r))


@pytest.mark.gpu
def test_device_corrections_match_oracle(cuda):
    import torch
    s, c = _case(lambda: harness.box_system(20, 20, 20, tet=True, seed=8), seed=22)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    rng = np.random.default_rng(9)
    correction = rng.normal(size=s.n).astype(np.float32)
    flux = t(c.flux)
    L.fv_correct_flux(t(c.owner), t(c.neighbour), t(correction), t(c.coefficient), flux, c.internal)
    f = c.flux.copy()
    fv.oracle_correct_flux(c, correction, f)
    assert np.array_equal(_bits(flux.cpu().numpy()), _bits(f))
    volume, inverse, diagonal, g, corr, uvwp = _velocity_inputs(s.n, 10)
    dev = [t(x) for x in uvwp]
    L.fv_correct_velocity(t(volume), t(inverse), t(diagonal), *(t(x) for x in g), t(corr), *dev,
                          0.3)
    host = [x.copy() for x in uvwp]
    fv.oracle_correct_velocity(s.n, volume, inverse, diagonal, g, corr, host, 0.3)
    for x, y in zip(dev, host):
        assert np.array_equal(_bits(x.cpu().numpy()), _bits(y))


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True], ids=["plain", "mixed"])
def test_assemble_refresh_equals_assemble_then_refresh(cuda, mixed):
    """The fused pass (assembly + level-0 L1 diagonal) and the separate
    assembly followed by refresh give the same matrix, right-hand side and
    hierarchy values, and the same solve, bit for bit."""
    import torch
    s, c = _case(lambda: harness.box_system(24, 24, 24, tet=True, seed=14), seed=23)
    fvd = _device_fv(c)
    results = []
    for fused in (False, True):
        a = L.upload(s)
        rhs = torch.zeros(s.n, device="cuda")
        if mixed:
            solver = L.make_mixed_solver(s)
        else:
            solver = L.make_amg_solver(L.SolverKind.AmgPcg, s, L.AmgOptions(
                structure=L.OperatorStructure.SymmetricMMatrix))
        if fused:
            solver.assemble_refresh(a, fvd, rhs)
        else:
            L.fv_pressure_assemble(a, fvd, rhs)
            solver.refresh(a)
        levels = [] if mixed else [(lv[3].copy(), lv[4].copy()) for lv in solver.levels()]
        x = torch.zeros(s.n, dtype=torch.float64 if mixed else torch.float32, device="cuda")
        st = solver.solve(a, x, rhs, L.SolveControl(1e-6, 1e-30, 2000))
        results.append((a.val.cpu().numpy(), rhs.cpu().numpy(), levels, st.iterations,
                        x.cpu().numpy()))
    (v0, r0, l0, i0, x0), (v1, r1, l1, i1, x1) = results
    assert np.array_equal(_bits(v0), _bits(v1)) and np.array_equal(_bits(r0), _bits(r1))
    for (va, ia), (vb, ib) in zip(l0, l1):
        assert np.array_equal(_bits(va), _bits(vb)) and np.array_equal(_bits(ia), _bits(ib))
    assert i0 == i1 and i0 > 0
    assert np.array_equal(x0.view(np.uint8), x1.view(np.uint8))


@pytest.mark.gpu
def test_assemble_refresh_rejects_a_bad_reference_cell(cuda):
    import torch
    s, c = _case(SYSTEMS[0][1], seed=24)
    a = L.upload(s)
    rhs = torch.zeros(s.n, device="cuda")
    solver = L.make_amg_solver(L.SolverKind.AmgPcg, s, L.AmgOptions(
        structure=L.OperatorStructure.SymmetricMMatrix))
    bad = _device_fv(c)
    bad.reference = s.n
    with pytest.raises(L.KuttaError):
        solver.assemble_refresh(a, bad, rhs)
    with pytest.raises(L.KuttaError):
        L.fv_pressure_assemble(a, bad, rhs)


def test_face_data_is_consistent():
    """harness.fv_faces: every internal face sits in exactly two cell-face
    slots (owner +1, neighbour -1) whose CSR entries are (cell, other cell);
    every boundary face in one owner slot; shared entries occur."""
    s = harness.box_system(6, 6, 6, tet=True, seed=1)
    c = harness.fv_faces(s.row_ptr, s.col, s.diag, seed=2)
    assert c.offsets[-1] == len(c.faces) == 2 * c.internal + (c.n_faces - c.internal)
    cell = np.repeat(np.arange(c.n), np.diff(c.offsets))
    seen = np.zeros(c.n_faces, np.int64)
    np.add.at(seen, c.faces, 1)
    assert np.all(seen[:c.internal] == 2) and np.all(seen[c.internal:] == 1)
    inner = c.adjacent >= 0
    assert np.all(inner == (c.faces < c.internal))
    f = c.faces[inner]
    own = c.sign[inner] > 0
    assert np.all(np.where(own, c.owner[f], c.neighbour[f]) == cell[inner])
    assert np.all(np.where(own, c.neighbour[f], c.owner[f]) == c.adjacent[inner])
    assert np.all(c.cols[c.entry[inner]] == c.adjacent[inner])
    rows = np.repeat(np.arange(c.n), np.diff(c.rows))
    assert np.all(rows[c.entry[inner]] == cell[inner])
    assert len(np.unique(c.entry[inner])) < inner.sum()  # some entries shared
