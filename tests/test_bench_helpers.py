"""Host-side helpers of bench.py's configurations (no GPU)."""
import numpy as np
import scipy.sparse as sp

from kutta_b200 import harness
from kutta_b200 import linalg as L


def test_blend_keeps_a_symmetric_m_matrix():
    """The successive-solve configuration blends the coefficient field toward a
    fresh one (keep 0.7) on the matrix values. The blend must stay a
    float-valued symmetric M-matrix whose rows are weakly diagonally dominant
    by at least the blended boundary term, and the reference's M-matrix check
    (make_amg_solver with SymmetricMMatrix) must accept it."""
    import bench
    kw = dict(tet=True, seed=1, band_layers=3, dmin=1e-6, dmax=1.0)
    s = harness.box_system(8, 8, 8, **kw)
    fresh = harness.box_system(8, 8, 8, coeff_seed=5, **kw)
    assert np.array_equal(s.col, fresh.col)
    vals, bnd = bench._blend(s.val.copy(), s.diag, s.boundary.copy(), s.row_ptr, fresh, 0.7)
    assert np.all(vals.astype(np.float32).astype(np.float64) == vals)
    A = sp.csr_matrix((vals, s.col, s.row_ptr), shape=(s.n, s.n))
    assert abs(A - A.T).max() == 0
    off = A - sp.diags(A.diagonal())
    assert off.max() <= 0
    margin = A.diagonal() - np.asarray(abs(off).sum(axis=1)).ravel()
    assert np.all(margin >= bnd * (1 - 1e-6))
    assert not np.array_equal(vals, s.val)
    t = harness.HostSystem(s.row_ptr, s.col, s.diag, vals, s.b)
    levels = L.build_hierarchy(t, L.AmgOptions(structure=L.OperatorStructure.SymmetricMMatrix))
    assert len(levels) > 1
