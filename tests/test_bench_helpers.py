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


def test_clock_samples_are_summarised():
    """bench.Clocks.stop: the median SM clock under sampling, the largest
    reported maximum, and the throttle reasons seen Active in any sample."""
    import bench
    out = L.library_path().parent / "checks"
    out.mkdir(exist_ok=True)
    path = out / "clocks_sample.csv"
    path.write_text(
        "0, 1965, 1965, 640.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n"
        "0, 1800, 1965, 990.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
        "0, 1350, 1965, 998.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
        "garbled line\n")

    class _Proc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    c = bench.Clocks(0)
    c.proc, c.path = _Proc(), str(path)
    summary = c.stop()
    assert summary == {"sm_mhz": 1800.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                       "samples": 3}
    assert not path.exists()


def test_peaks_and_traffic_come_from_the_committed_files():
    import json

    import bench
    peak, source = bench._peaks()
    if (bench.ROOT / "MEASURED_PEAKS.json").exists():
        assert source == "measured"
        assert peak == json.loads((bench.ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
    else:
        assert (peak, source) == (6650.0, "fallback")
    entries = json.loads((bench.ROOT / "profiles" / "traffic.json").read_text())
    for kernel, e in entries.items():
        assert bench._traffic(kernel, e["workload"]) == e["dram_bytes_per_launch"]
        assert bench._traffic(kernel, "another workload") is None


def test_fp64_oracle_error_of_a_solution():
    """bench.fp64_oracle: the relative error of a returned x against the FP64
    CG oracle, and a reported (not raised) failure."""
    import bench
    from oracle import kutta_oracle as O
    s = harness.box_system(8, 8, 8, tet=True, seed=2)
    x64, _ = O.cg64(s, rel_tol=1e-13)
    rng = np.random.default_rng(0)
    x = x64 * (1 + 1e-4 * rng.standard_normal(s.n))
    r = bench.fp64_oracle(s, x)
    expected = np.linalg.norm(x - x64) / np.linalg.norm(x64)
    assert abs(r["relative_error"] - expected) <= 1e-3 * expected
    assert r["oracle_iterations"] > 0 and r["oracle_relative_residual"] < 1e-11
    assert "unavailable" in bench.fp64_oracle(s, x[:-1])
