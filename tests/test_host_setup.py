"""The product's host side without a GPU: the C ABI library loads and exports
every symbol include/kutta_b200.h declares; the host AMG setup reproduces the
reference's hierarchy bit for bit; usage errors follow the reference's rules."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

import golden_cases as G
from kutta_b200 import harness
from kutta_b200 import linalg as L

HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "kutta_b200.h"
M = L.OperatorStructure.SymmetricMMatrix


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(b2_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(L.library_path()))
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(L._SIGNATURES), "ctypes signatures out of sync with the header"


def test_defaults_match_reference_structs():
    lib = L._load()
    o = L._Options()
    lib.b2_options_default(ctypes.byref(o))
    assert (o.cycle, o.pre_sweeps, o.post_sweeps, o.coarse_sweeps, o.coarse_rows, o.max_levels,
            o.aggregation_passes, o.strength_threshold) == (0, 5, 5, 32, 24, 24, 3, 0.25)
    c = L._Control()
    lib.b2_control_default(ctypes.byref(c))
    assert (c.rel_tol, c.abs_tol, c.max_iter, c.residual_check_interval) == (1e-2, 1e-12, 200, 8)


@pytest.mark.parametrize("name", [n for n in G.names() if G.load(n)[0]["kind"] >= 3]
                         + G.hierarchy_names())
def test_host_hierarchy_matches_reference_fixture(name):
    """Every AMG fixture, and the 5.3M-row tet pressure matrix's hierarchy
    (about 20 s: generating the matrix and the host setup)."""
    meta, arrays = G.load(name)
    s = G.system(name)
    opts = L.AmgOptions(structure=M if meta["m_matrix"] else L.OperatorStructure.General,
                        **meta.get("options", {}))
    levels = L.build_hierarchy(s, opts, spd=meta["kind"] == 3)
    assert [lv.n for lv in levels] == meta["levels"]
    for i, (lv, sha) in enumerate(zip(levels, meta["level_sha"])):
        assert G.digest(lv.row_ptr) == sha["row_ptr"], i
        assert G.digest(lv.col) == sha["col"], i
        assert G.digest(lv.inverse_l1) == sha["l1"], i
        if i > 0:
            assert G.digest(lv.val) == sha["val"], i
        if sha["aggregate"] is not None:
            assert G.digest(lv.aggregate) == sha["aggregate"], i
        if f"l{i}_aggregate" in arrays:
            assert np.array_equal(lv.aggregate, arrays[f"l{i}_aggregate"])


def test_host_hierarchy_matches_oracle_on_upwind_and_isolated_rows():
    """Strong upwind couplings under permutation (test_solvers.cpp:288-306) and
    isolated diagonal rows (:308-322) coarsen as in the restated reference."""
    from oracle import kutta_oracle as O
    s = harness.poisson(24, 16, 8, 1, False, False, 20.0)
    rng = np.random.default_rng(3)
    perm = rng.permutation(s.n).astype(np.int32)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(s.n, dtype=np.int32)
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))[perm][:, perm].tocsr()
    A.sort_indices()
    t = harness.HostSystem(A.indptr.astype(np.int32), A.indices.astype(np.int32),
                           np.array([A.indptr[i] + np.searchsorted(A.indices[A.indptr[i]:A.indptr[i + 1]], i)
                                     for i in range(s.n)], np.int32), A.data.astype(np.float64),
                           np.ones(s.n, np.float32))
    for system, m in ((s, False), (t, False)):
        mine = L.build_hierarchy(system, L.AmgOptions(), spd=False)
        o = O.Solver(system, O.options(O.AMG_BICGSTAB))
        theirs = o.levels()
        assert len(mine) == len(theirs) > 1
        for a, b in zip(mine, theirs):
            assert np.array_equal(a.col, b["col"])
            if b["aggregate"] is not None:
                assert np.array_equal(a.aggregate, b["aggregate"])
    # isolated rows
    p = harness.poisson(8, 8)
    n0 = p.n
    extra = 1024
    p.row_ptr = np.concatenate([p.row_ptr, p.row_ptr[-1] + np.arange(1, extra + 1)]).astype(np.int32)
    p.col = np.concatenate([p.col, np.arange(n0, n0 + extra)]).astype(np.int32)
    p.diag = np.concatenate([p.diag, p.row_ptr[n0:-1]]).astype(np.int32)
    p.val = np.concatenate([p.val, np.full(extra, 2.0)])
    levels = L.build_hierarchy(p, L.AmgOptions(), spd=True)
    assert len(levels) > 1
    assert np.all(levels[0].aggregate[n0:] == -1)


def _bad(s, **changes):
    t = harness.HostSystem(s.row_ptr.copy(), s.col.copy(), s.diag.copy(), s.val.copy(), s.b.copy())
    for k, v in changes.items():
        getattr(t, k)[v[0]] = v[1]
    return t


def test_invalid_csr_and_options_are_rejected_like_the_reference():
    """test_solvers.cpp:50-78, 450-485 (errors raised before any device work)."""
    s = harness.poisson(5, 4, 3, 2, True)
    with pytest.raises(L.KuttaError, match="missing or incorrect diagonal"):
        L.build_hierarchy(_bad(s, diag=(0, -1)))
    with pytest.raises(L.KuttaError, match="columns must be in range"):
        L.build_hierarchy(_bad(s, col=(0, s.n)))
    with pytest.raises(L.KuttaError, match="nonfinite or out-of-range"):
        L.build_hierarchy(_bad(s, val=(0, np.inf)))
    with pytest.raises(L.KuttaError, match="invalid options"):
        L.build_hierarchy(s, L.AmgOptions(aggregation_passes=9))
    with pytest.raises(L.KuttaError, match="equal pre/post"):
        L.build_hierarchy(s, L.AmgOptions(pre_sweeps=2, post_sweeps=3), spd=True)
    neg = harness.poisson(16, 12, 4, 1, False, False, 20)
    for i in range(0, neg.n, 7):
        neg.val[neg.row_ptr[i]:neg.row_ptr[i + 1]] *= -1
    with pytest.raises(L.KuttaError, match="AMG: requires positive diagonals"):
        L.build_hierarchy(neg, L.AmgOptions(), spd=False)
    h = harness.box_system(6, 6, 6, tet=True, seed=1)
    bad = _bad(h, val=(int(h.diag[0]), 0.5 * h.val[h.diag[0]]))
    with pytest.raises(L.KuttaError, match="diagonally dominant"):
        L.build_hierarchy(bad, L.AmgOptions(structure=M), spd=True)


def test_first_failing_row_decides_the_error_on_large_inputs():
    """The host checks scan large inputs in parallel chunks; as in the
    reference's serial loops, the error reported is that of the first failing
    row (or value), whichever chunk finds a later one first."""
    s = harness.poisson(80, 80, 20)  # 128,000 rows: several chunks
    late = s.n - 10
    # Structure: a bad diagonal early, unsorted columns late.
    off = next(j for j in range(s.row_ptr[10], s.row_ptr[11]) if s.col[j] != 10)
    t = _bad(s, diag=(10, int(off)))
    lo = int(s.row_ptr[late])
    t.col[lo], t.col[lo + 1] = t.col[lo + 1], t.col[lo]
    with pytest.raises(L.KuttaError, match="missing or incorrect diagonal"):
        L.build_hierarchy(t)
    # Values: a nonfinite value late only.
    with pytest.raises(L.KuttaError, match="nonfinite or out-of-range"):
        L.build_hierarchy(_bad(s, val=(int(s.row_ptr[late]), np.nan)))
    # M-matrix: a positive edge early (its transpose too, to stay symmetric),
    # a non-dominant row late.
    m = harness.box_system(26, 26, 26, tet=False, seed=2)  # 17,576 rows
    big = harness.box_system(42, 42, 42, tet=False, seed=2)  # 74,088 rows
    for case in (m, big):
        j = next(j for j in range(case.row_ptr[3], case.row_ptr[4]) if case.col[j] != 3)
        c = int(case.col[j])
        k = next(k for k in range(case.row_ptr[c], case.row_ptr[c + 1]) if case.col[k] == 3)
        v = case.val.copy()
        v[j], v[k] = -v[j], -v[k]
        last = case.n - 3
        v[case.diag[last]] *= 0.25
        bad = harness.HostSystem(case.row_ptr, case.col, case.diag, v, case.b)
        with pytest.raises(L.KuttaError, match="symmetric nonpositive edges"):
            L.build_hierarchy(bad, L.AmgOptions(structure=M), spd=True)


def test_empty_system_builds():
    """test_solvers.cpp:274-286: an empty CSR is a valid no-op."""
    e = harness.HostSystem(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                           np.zeros(0), np.zeros(0, np.float32))
    levels = L.build_hierarchy(e, L.AmgOptions(), spd=True)
    assert len(levels) == 1 and levels[0].n == 0
