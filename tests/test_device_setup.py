"""AMG setup on the device against the host setup. The host setup restates
the reference's aggregation (src/kutta/linalg/amg.cpp:25-226) and is pinned to
it bit for bit by the hierarchy tests. For every level the two must give the
same aggregates, coarse patterns, diagonal positions, members, Galerkin entry
maps, coarse values and L1 diagonals, bit for bit. The mixed hierarchy (with
singleton absorption) is checked through bitwise-identical solves."""
import pathlib

import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L

pytestmark = pytest.mark.gpu

M = L.OperatorStructure.SymmetricMMatrix
G = L.OperatorStructure.General
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _tmr(name):
    d = np.load(GOLDEN / f"{name}.npz")
    return harness.HostSystem(d["row_ptr"], d["col"], d["diag"], d["val"], d["b_random"])


def _graded(side, seed):
    return harness.box_system(side, side, side, tet=True, seed=seed, band_layers=10, aspect=1000.0,
                              ratio=1.2, dmin=1e-6, dmax=1.0)


CASES = [
    ("poisson32", lambda: harness.poisson(32, 32, 32), G, {}),
    ("poisson_aniso1000", lambda: harness.poisson(12, 9, 5, 1000), G, {}),
    ("poisson_random2d", lambda: harness.poisson(40, 37, 1, 1, True), G, {}),
    ("poisson_wind3", lambda: harness.poisson(20, 18, 1, 1, False, False, 3), G, {}),
    ("hex16_pressure", lambda: harness.box_system(16, 16, 16, tet=False, seed=5), M, {}),
    ("tet20_pressure", lambda: harness.box_system(20, 20, 20, tet=True, seed=7), M, {}),
    ("tet10_convection", lambda: harness.box_system(10, 10, 10, tet=True, seed=2,
                                                     convection=1e-3), G, {}),
    ("graded_tet16", lambda: _graded(16, 3), M, {}),
    ("tmr_it15", lambda: _tmr("tmr_bump_pressure_it15"), M, {}),
    ("tmr_it18", lambda: _tmr("tmr_bump_pressure_it18"), M, {}),
    ("hex12_one_pass", lambda: harness.box_system(12, 12, 12, tet=False, seed=4), M,
     {"aggregation_passes": 1}),
    ("tet12_two_passes_strong", lambda: harness.box_system(12, 12, 12, tet=True, seed=6), M,
     {"aggregation_passes": 2, "strength_threshold": 0.5}),
    ("tet16_coarse100_k", lambda: harness.box_system(16, 16, 16, tet=True, seed=9), M,
     {"coarse_rows": 100, "cycle": L.AmgCycle.K}),
    ("poisson_neumann", lambda: harness.poisson(14, 13, 8), G,
     {"nullspace": L.NullSpace.Constant}),
]


def _solver(s, structure, extra, setup, kind=L.SolverKind.AmgPcg):
    opts = L.AmgOptions(structure=structure, setup=setup, **extra)
    solver = L.make_amg_solver(kind, s, opts)
    a = L.upload(s)
    solver.refresh(a)
    solver._matrix = a  # level 0's values are the caller's matrix
    return solver


@pytest.mark.parametrize("name,make,structure,extra", CASES, ids=[c[0] for c in CASES])
def test_device_setup_equals_host_setup(cuda, name, make, structure, extra):
    s = make()
    kind = L.SolverKind.AmgBicgstab if ("wind" in name or "convection" in name) \
        else L.SolverKind.AmgPcg
    host = _solver(s, structure, extra, L.Setup.Host, kind)
    device = _solver(s, structure, extra, L.Setup.Device, kind)
    assert device.describe() == host.describe()
    hl, dl = host.levels(), device.levels()
    assert [lv[0] for lv in dl] == [lv[0] for lv in hl]
    assert len(hl) > 1
    for k, ((n, rp, cl, vl, l1, ag), (n2, rp2, cl2, vl2, l12, ag2)) in enumerate(zip(hl, dl)):
        assert np.array_equal(rp, rp2), k
        assert np.array_equal(cl, cl2), k
        assert np.array_equal(vl.view(np.uint32), vl2.view(np.uint32)), k
        assert np.array_equal(l1.view(np.uint32), l12.view(np.uint32)), k
        assert np.array_equal(ag, ag2), k
        th, td = host.level_transfer(k), device.level_transfer(k)
        assert th.keys() == td.keys()
        for key in th:
            assert np.array_equal(th[key], td[key]), (k, key)


@pytest.mark.parametrize("make", [
    lambda: harness.box_system(24, 24, 24, tet=True, seed=12),
    lambda: _graded(20, 5),
    lambda: _tmr("tmr_bump_pressure_it18"),
], ids=["tet24", "graded_tet20", "tmr_it18"])
def test_mixed_solve_identical_with_device_setup(cuda, make):
    """The mixed hierarchy (singleton absorption, BF16 levels, dense coarsest)
    built on the device gives the host-built solver's solve bit for bit."""
    import torch
    s = make()
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    out = {}
    for setup in (L.Setup.Host, L.Setup.Device):
        o = L.MixedOptions()
        o.amg.setup = setup
        solver = L.make_mixed_solver(s, o)
        solver.refresh(a)
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-7, 1e-30, 3000))
        out[setup] = (solver.describe(), st.iterations, st.final_residual, x.cpu().numpy())
    h, d = out[L.Setup.Host], out[L.Setup.Device]
    assert d[0] == h[0] and d[1] == h[1] and d[2] == h[2]
    assert np.array_equal(d[3].view(np.uint64), h[3].view(np.uint64))


def test_nonsymmetric_pattern_falls_back_to_host_setup(cuda):
    """A pattern without its transpose entries takes the host setup (the
    device pairing reads strengths through the transpose)."""
    s = harness.poisson(10, 9, 1, 1, False, False, 3)
    # Drop one off-diagonal entry of row 5 (keeping its transpose).
    rp, col, val = s.row_ptr.copy(), s.col.copy(), s.val.copy()
    j = next(j for j in range(rp[5], rp[6]) if col[j] != 5)
    keep = np.ones(len(col), bool)
    keep[j] = False
    col, val = col[keep], val[keep]
    rp[6:] -= 1
    diag = np.array([rp[i] + np.nonzero(col[rp[i]:rp[i + 1]] == i)[0][0] for i in range(s.n)],
                    np.int32)
    t = harness.HostSystem(rp, col, diag, val, s.b)
    host = _solver(t, G, {}, L.Setup.Host, L.SolverKind.AmgBicgstab)
    device = _solver(t, G, {}, L.Setup.Device, L.SolverKind.AmgBicgstab)
    for a, b in zip(host.levels(), device.levels()):
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[5], b[5])
        assert np.array_equal(a[3].view(np.uint32), b[3].view(np.uint32))


@pytest.mark.parametrize("mixed", [False, True], ids=["plain", "mixed"])
def test_device_setup_equals_host_setup_at_full_size(cuda, mixed):
    """The headline matrix (96^3 x 6 tets, 5,308,416 rows): every level's
    aggregates, pattern, members and entry map, and (plain hierarchy) the
    refreshed values, identical between the device and the host setup. For
    the mixed hierarchy the solve from each is compared bit for bit."""
    import torch
    s = harness.pressure_tet96()
    a = L.upload(s)
    if mixed:
        b = torch.from_numpy(s.b).cuda()
        result = []
        for setup in (L.Setup.Host, L.Setup.Device):
            o = L.MixedOptions()
            o.amg.setup = setup
            solver = L.make_mixed_solver(s, o)
            solver.refresh(a)
            x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
            st = solver.solve(a, x, b, L.SolveControl(1e-6, 1e-30, 3000))
            result.append((solver.describe(), st.iterations, x.cpu().numpy()))
            del solver
        assert result[0][:2] == result[1][:2]
        assert np.array_equal(result[0][2].view(np.uint64), result[1][2].view(np.uint64))
        return
    host = _solver(s, M, {}, L.Setup.Host)
    device = _solver(s, M, {}, L.Setup.Device)
    assert device.describe() == host.describe()
    hl, dl = host.levels(), device.levels()
    assert [lv[0] for lv in hl] == [lv[0] for lv in dl]
    for k, (h, d) in enumerate(zip(hl, dl)):
        for a_h, a_d in zip(h[1:], d[1:]):
            assert np.array_equal(a_h.view(np.uint32), a_d.view(np.uint32)), k
        th, td = host.level_transfer(k), device.level_transfer(k)
        for key in th:
            assert np.array_equal(th[key], td[key]), (k, key)
