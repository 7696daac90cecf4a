"""The device setup's pairing argument, checked on the CPU. The greedy pass
of src/kutta/linalg/amg.cpp:25-75 is equivalent to a triangular system:

    i is a leader unless a leader k < i took it;
    a leader takes the first entry of its preference list (candidates j > i,
    strength descending, column ascending) that no leader k < i took.

A state that one Jacobi sweep of these equations leaves unchanged is its
unique solution. Here the sweeps are restated in numpy, as the device runs
them (setup_kernels.cu), and the fixed point is compared with the host
restatement's sequential pass (setup.cpp), which is pinned to the reference.
The same is done for the mixed hierarchy's singleton absorption, whose
sequential order dependence (a neighbour below i counts where it already
went) is triangular too."""
import numpy as np
import pytest
import scipy.sparse as sp

from kutta_b200 import harness
from kutta_b200 import linalg as L

THRESHOLD = 0.25
NONE = np.iinfo(np.int64).max


def _strength(s):
    A = sp.csr_matrix((np.abs(s.val.astype(np.float32).astype(np.float64)), s.col, s.row_ptr),
                      shape=(s.n, s.n))
    S = A.maximum(A.T).tocsr()
    S.setdiag(0)
    S.eliminate_zeros()
    S.sort_indices()
    rows = np.repeat(np.arange(s.n), np.diff(S.indptr))
    strongest = np.zeros(s.n)
    np.maximum.at(strongest, rows, S.data)
    return rows, S.indices, S.data, strongest


def _pairs(s, exclude_isolated=True):
    """The pairing fixed point: aggregate per row (-1 left out), sweeps used."""
    n = s.n
    rows, cols, w, strongest = _strength(s)
    keep = (cols > rows) & (w >= THRESHOLD * strongest[rows])
    r, c, ww = rows[keep], cols[keep], w[keep]
    order = np.lexsort((c, -ww, r))
    r, c = r[order], c[order]
    left_out = (strongest == 0) if exclude_isolated else np.zeros(n, bool)
    leader = ~left_out
    partner = np.full(n, -1)
    for sweep in range(1, 10_000):
        owner = np.full(n, NONE)
        claimed = leader & (partner >= 0)
        np.minimum.at(owner, partner[claimed], np.nonzero(claimed)[0])
        new_leader = (owner == NONE) & ~left_out
        available = owner[c] >= r  # no leader below r took c
        first = np.full(n, -1)
        idx = np.nonzero(available)[0]
        uniq, pos = np.unique(r[idx], return_index=True)
        first[uniq] = c[idx[pos]]
        new_partner = np.where(new_leader, first, -1)
        if np.array_equal(new_leader, leader) and np.array_equal(new_partner, partner):
            break
        leader, partner = new_leader, new_partner
    ids = np.cumsum(leader) - 1
    agg = np.full(n, -1)
    agg[leader] = ids[leader]
    taken = (~leader) & (owner != NONE)
    agg[taken] = ids[owner[taken]]
    return agg, sweep


def _absorb(s, agg):
    """Singleton absorption (setup.cpp's pairs(), mixed hierarchy) as a fixed
    point: a row alone in its aggregate joins the pair of its strongest
    strongly coupled neighbour; neighbours below i are seen where they went."""
    n = s.n
    rows, cols, w, strongest = _strength(s)
    d = np.abs(s.val.astype(np.float32).astype(np.float64)[s.diag])
    size0 = np.bincount(agg[agg >= 0], minlength=agg.max() + 1)
    single = np.nonzero((agg >= 0) & (size0[np.maximum(agg, 0)] == 1))[0]
    cur = agg.copy()
    for sweep in range(1, 10_000):
        nxt = agg.copy()
        for i in single:
            lo, hi = np.searchsorted(rows, i), np.searchsorted(rows, i, side="right")
            best, weight = agg[i], 0.0
            for k in range(lo, hi):
                j, wj = cols[k], w[k]
                g = cur[j] if j < i else agg[j]
                if (g >= 0 and g != agg[i] and size0[g] >= 2 and wj > weight
                        and wj >= THRESHOLD * strongest[i] and wj >= 0.01 * np.sqrt(d[i] * d[j])):
                    best, weight = g, wj
            nxt[i] = best
        if np.array_equal(nxt, cur):
            break
        cur = nxt
    used = np.zeros(agg.max() + 1, bool)
    used[cur[cur >= 0]] = True
    renumber = np.cumsum(used) - 1
    return np.where(cur >= 0, renumber[np.maximum(cur, 0)], -1), sweep


SYSTEMS = [
    ("poisson24", lambda: harness.poisson(24, 24, 24), L.OperatorStructure.General),
    ("poisson_aniso", lambda: harness.poisson(20, 17, 9, 1000), L.OperatorStructure.General),
    ("poisson_random2d", lambda: harness.poisson(60, 55, 1, 1, True), L.OperatorStructure.General),
    ("poisson_wind", lambda: harness.poisson(30, 28, 1, 1, False, False, 3),
     L.OperatorStructure.General),
    ("hex16", lambda: harness.box_system(16, 16, 16, tet=False, seed=2),
     L.OperatorStructure.SymmetricMMatrix),
    ("tet16", lambda: harness.box_system(16, 16, 16, tet=True, seed=3),
     L.OperatorStructure.SymmetricMMatrix),
    ("graded_tet12", lambda: harness.box_system(12, 12, 12, tet=True, seed=4, band_layers=5,
                                                dmin=1e-6, dmax=1.0),
     L.OperatorStructure.SymmetricMMatrix),
]


@pytest.mark.parametrize("name,make,structure", SYSTEMS, ids=[c[0] for c in SYSTEMS])
def test_pairing_fixed_point_equals_sequential_pass(name, make, structure):
    s = make()
    host = L.build_hierarchy(s, L.AmgOptions(aggregation_passes=1, structure=structure),
                             spd="wind" not in name)
    mine, sweeps = _pairs(s)
    assert np.array_equal(mine, host[0].aggregate)
    assert sweeps < 200


@pytest.mark.parametrize("name,make,structure", SYSTEMS[4:], ids=[c[0] for c in SYSTEMS[4:]])
def test_absorption_fixed_point_equals_sequential_pass(name, make, structure):
    s = make()
    o = L.MixedOptions()
    o.amg.aggregation_passes = 1
    host = L.build_mixed_hierarchy(s, o)
    paired, _ = _pairs(s)
    mine, sweeps = _absorb(s, paired)
    assert np.array_equal(mine, host[0].aggregate)
    assert sweeps < 50
