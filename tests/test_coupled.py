"""The Coupled (4x4-block) solve (src/kutta/fv/coupled_solver.cpp with
src/kutta/kernels/fv_coupled.kern.h) against the reference's own results.

Fixtures (tests/golden/make_coupled.py) hold box meshes the reference built,
seeded flow fields, and everything the reference's CoupledSolver computed on
them. CPU: the host setup (pressure-force sensitivities, aggregation,
coarse patterns) is bit-exact against the reference; the numpy oracle of the
row kernels is pinned against the reference's edge cache and final residual.
GPU: every assembled array (cell data, face coefficients, right-hand side,
each coarse level's Galerkin operator and block inverse) is bit-exact; the
fine and coarse row kernels are bit-exact against the oracle; the solve
takes the reference's iterations and reaches its residual; the update and
the closed-domain gauge follow."""
from __future__ import annotations

import json
import pathlib

import numpy as np
import pytest

from kutta_b200 import linalg as L
from oracle import coupled as O

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
NAMES = sorted(p.stem for p in GOLDEN.glob("coupled_*.npz"))


def load(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(bytes(d["meta"]).decode())
    mesh = {k[5:]: d[k] for k in d.files if k.startswith("mesh_")}
    fields = {k[6:]: d[k] for k in d.files if k.startswith("field_")}
    refs = {k[4:]: d[k] for k in d.files if k.startswith("ref_")}
    refs.update({k: d[k] for k in d.files if k in ("pair_hi", "pair_lo")})
    fields.setdefault("net_outflow", None)
    fields.update(density=meta["density"], velocity_scale=meta["velocity_scale"],
                  reference=meta["reference"])
    return meta, mesh, fields, refs


def options(meta) -> L.CoupledOptions:
    return L.CoupledOptions(**meta["options"])


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else a.dtype)


def ref_levels(meta, refs):
    """The reference's coarse levels in fine-to-coarse order, from the launch
    captures (keyed by level size)."""
    sizes = [int(s) for s in meta["describe"].split("(")[1].split(" rows")[0].split("/")]
    out = []
    for k, n in enumerate(sizes[1:], start=1):
        lv = {key: refs[f"level{n}_{key}"] for key in ("rows", "cols", "diag", "a", "c", "g",
                                                       "h", "d")}
        lv["n"] = n
        lv["aggregate"] = refs[f"aggregate{sizes[k - 1]}"]
        lv["offsets"] = refs.get(f"restrict{n}_offsets")
        lv["members"] = refs.get(f"restrict{n}_members")
        out.append(lv)
    return sizes, out


def wc_of(meta):
    return np.float32(meta["density"] * meta["velocity_scale"])


# ---- CPU ------------------------------------------------------------------------

def test_fixtures_present():
    assert len(NAMES) >= 5, NAMES


@pytest.mark.parametrize("name", NAMES)
def test_fixture_is_well_formed(name):
    meta, mesh, fields, refs = load(name)
    n, nf, ni, entries, nnz = (int(v) for v in mesh["sizes"])
    assert mesh["cell_face_offsets"][-1] == entries == len(mesh["cell_faces"])
    assert len(mesh["owner"]) == nf and len(mesh["neighbour"]) == ni
    assert np.all(mesh["owner"][:ni] < mesh["neighbour"])
    assert len(fields["momentum_u"]) == nnz and len(fields["mass"]) == nf
    assert refs["cell"].size == 27 * n and refs["rhs"].size == 4 * n and refs["x"].size == 4 * n
    assert meta["converged"], meta


@pytest.mark.parametrize("name", NAMES)
def test_host_setup_matches_reference(name):
    """Sensitivities G and Q (cell planes 4-6, 10-18), aggregates, member lists
    and coarse patterns of b2_coupled_setup_build, bit for bit
    (coupled_solver.cpp:27-289)."""
    meta, mesh, _, refs = load(name)
    n = int(mesh["sizes"][0])
    s = L.build_coupled_setup(mesh, options(meta))
    for k in list(range(4, 7)) + list(range(10, 19)):
        got, want = s["cell"][k * n:(k + 1) * n], refs["cell"][k * n:(k + 1) * n]
        assert np.array_equal(bits(got), bits(want)), k
    sizes, levels = ref_levels(meta, refs)
    assert [lv["n"] for lv in s["levels"]] == sizes
    for k, lv in enumerate(levels, start=1):
        mine = s["levels"][k]
        for key in ("rows", "cols", "diag"):
            assert np.array_equal(mine[key], lv[key][: len(mine[key])]), (k, key)
        assert np.array_equal(s["levels"][k - 1]["aggregate"], lv["aggregate"][:sizes[k - 1]])
        if lv["offsets"] is not None:
            assert np.array_equal(s["levels"][k - 1]["member_offsets"], lv["offsets"][:lv["n"] + 1])
            assert np.array_equal(s["levels"][k - 1]["members"], lv["members"][:sizes[k - 1]])
    inner = np.diff(mesh["cell_face_offsets"])
    assert s["width"] == max(int(np.sum(mesh["adjacent"][a:b] >= 0))
                             for a, b in zip(mesh["cell_face_offsets"][:-1],
                                             mesh["cell_face_offsets"][1:]))
    assert inner.max() >= s["width"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_edge_cache_matches_reference(name):
    meta, mesh, fields, refs = load(name)
    if "edge" not in refs:
        pytest.skip("the reference ran its recompute operator (no edge cache)")
    edge = O.fine_coefficients(mesh, refs["cell"], fields["viscosity"], fields["mass"],
                               fields["face_weights"], wc_of(meta))
    entries = len(mesh["cell_faces"])
    inner = np.tile(mesh["adjacent"] >= 0, 5)
    assert np.array_equal(bits(edge[inner]), bits(refs["edge"][: 5 * entries][inner]))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_residual_reproduces_reference(name):
    """r = b - J x of the reference's returned solution, through the oracle's
    row restatement, has the reference's final residual norm."""
    meta, mesh, fields, refs = load(name)
    edge = O.fine_coefficients(mesh, refs["cell"], fields["viscosity"], fields["mass"],
                               fields["face_weights"], wc_of(meta))
    r = O.fine_residual(mesh, refs["cell"], edge, refs["coefficient"], refs["x"], refs["rhs"],
                        wc_of(meta))
    norm = np.sqrt(np.sum(r.astype(np.float64) ** 2))
    assert norm == pytest.approx(meta["final_residual"], rel=1e-9)
    assert np.sqrt(np.sum(refs["rhs"].astype(np.float64) ** 2)) == \
        pytest.approx(meta["initial_residual"], rel=1e-12)


def test_setup_rejects_bad_mesh():
    meta, mesh, _, _ = load(NAMES[0])
    bad = dict(mesh)
    bad["adjacent"] = mesh["adjacent"].copy()
    bad["adjacent"][0] = int(mesh["sizes"][0])
    with pytest.raises(L.KuttaError, match="adjacent"):
        L.build_coupled_setup(bad)
    with pytest.raises(L.KuttaError, match="invalid options"):
        L.build_coupled_setup(mesh, L.CoupledOptions(smoother_damping=1.5))


def test_setup_matches_reference_live():
    """A case not in the fixtures, against the reference library when it is
    built here."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from kutta_b200 import coupled_harness as H
    case = ref.CoupledCase(True, 5, 3, 4, patch_kinds=(1, 4, 3, 0, 0, 3))
    f = H.flow_fields(case.arrays, 9)
    out = case.solve(f, ref.coupled_options(coarsest_rows=30))
    s = L.build_coupled_setup(case.arrays, L.CoupledOptions(coarsest_rows=30))
    n = int(case.arrays["sizes"][0])
    for k in list(range(4, 7)) + list(range(10, 19)):
        assert np.array_equal(bits(s["cell"][k * n:(k + 1) * n]),
                              bits(out["cell"][k * n:(k + 1) * n]))
    want = [int(v) for v in out["describe"].split("(")[1].split(" rows")[0].split("/")]
    assert [lv["n"] for lv in s["levels"]] == want


# ---- GPU ------------------------------------------------------------------------

def _device(fields):
    import torch
    out = {}
    for k, v in fields.items():
        out[k] = torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v
    return out


def _solver(meta, mesh, fields):
    import torch
    s = L.CoupledSolver(mesh, meta["reference"], options(meta))
    rows = torch.from_numpy(mesh["pattern_row_ptr"]).cuda()
    diag = torch.from_numpy(mesh["pattern_diag"]).cuda()
    d = _device(fields)
    for k, c in enumerate("uvw"):
        s.capture_diagonal(k, rows, diag, d["momentum_" + c], d["physical_" + c])
    rel, abs_, max_iter = meta["control"]
    st = s.solve(d, L.SolveControl(rel, abs_, max_iter))
    torch.cuda.synchronize()
    return s, st, d


def _aos(planes, n):
    return np.ascontiguousarray(planes.reshape(4, n).T).reshape(-1)


def _planes(aos, n):
    return np.ascontiguousarray(aos.reshape(n, 4).T).reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_coupled_assembly_matches_reference(cuda, name):
    """Cell data (captured diagonals, pressure diagonal, G, H, Q, Schur bound,
    block inverse), face coefficients, right-hand side and every coarse
    level's Galerkin operator, Schur bound and block inverse: bit for bit."""
    meta, mesh, fields, refs = load(name)
    s, _, _ = _solver(meta, mesh, fields)
    assert s.describe() == meta["describe"]
    n = int(mesh["sizes"][0])
    cell = s.copy("cell")
    for k in range(27):
        assert np.array_equal(bits(cell[k * n:(k + 1) * n]), bits(refs["cell"][k * n:(k + 1) * n])), k
    assert np.array_equal(bits(s.copy("coefficient")), bits(refs["coefficient"]))
    assert np.array_equal(bits(s.copy("rhs")), bits(refs["rhs"]))
    sizes, levels = ref_levels(meta, refs)
    assert s.levels() == len(sizes)
    for k, lv in enumerate(levels, start=1):
        got = s.level(k)
        for key in ("rows", "cols", "diag", "a", "c", "g", "h", "d"):
            assert np.array_equal(bits(got[key]), bits(lv[key][: len(got[key])])), (k, key)
        assert np.array_equal(got["aggregate"], lv["aggregate"][: len(got["aggregate"])])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_coupled_solve_matches_reference(cuda, name):
    """Iterations, convergence and both residuals of the reference's block
    BiCGStab, and its solution (the Krylov scalars come from FP64 dot
    products whose summation order differs, so x is compared at 1e-4)."""
    meta, mesh, fields, refs = load(name)
    s, st, _ = _solver(meta, mesh, fields)
    print(name, st, meta["iterations"], meta["final_residual"])
    assert st.iterations == meta["iterations"]
    assert st.converged == meta["converged"]
    assert st.initial_residual == pytest.approx(meta["initial_residual"], rel=1e-12)
    assert st.final_residual == pytest.approx(meta["final_residual"], rel=1e-3)
    x = s.copy("x")
    err = np.linalg.norm(x.astype(np.float64) - refs["x"]) / np.linalg.norm(refs["x"])
    assert err <= 1e-4, err


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_coupled_row_kernels_match_oracle(cuda, name):
    """J x, b - J x and the damped block-Jacobi sweep (from x and from zero) on
    seeded vectors: bit for bit against the oracle's restatement."""
    import torch
    meta, mesh, fields, refs = load(name)
    s, _, _ = _solver(meta, mesh, fields)
    n = int(mesh["sizes"][0])
    rng = np.random.default_rng(7)
    x = rng.standard_normal(4 * n).astype(np.float32)
    b = rng.standard_normal(4 * n).astype(np.float32)
    edge = O.fine_coefficients(mesh, refs["cell"], fields["viscosity"], fields["mass"],
                               fields["face_weights"], wc_of(meta))
    wc = wc_of(meta)
    omega = options(meta).smoother_damping
    want = {
        "spmv": O.fine_row(mesh, refs["cell"], edge, refs["coefficient"], x, wc),
        "residual": O.fine_residual(mesh, refs["cell"], edge, refs["coefficient"], x, b, wc),
        "smooth": O.fine_smooth(mesh, refs["cell"], edge, refs["coefficient"], x, b, wc, omega,
                                False),
        "smooth_zero": O.fine_smooth(mesh, refs["cell"], edge, refs["coefficient"], x, b, wc,
                                     omega, True),
    }
    dx = torch.from_numpy(_aos(x, n)).cuda()
    db = torch.from_numpy(_aos(b, n)).cuda()
    for op, w in want.items():
        y = torch.full((4 * n,), float("nan"), dtype=torch.float32, device="cuda")
        s.apply(op, dx, db, y)
        torch.cuda.synchronize()
        got = _planes(y.cpu().numpy(), n)
        assert np.array_equal(bits(got), bits(w.astype(np.float32))), op


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_coupled_update_matches_reference(cuda, name):
    """update(alpha 1, 1) from zero fields: u = du, p = wc dp~, then the closed
    domain's gauge p -= p[reference] (coupled_solver.cpp:514-522)."""
    import torch
    meta, mesh, fields, refs = load(name)
    s, _, _ = _solver(meta, mesh, fields)
    n = int(mesh["sizes"][0])
    u, v, w, p = (torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(4))
    s.update(u, v, w, p, 1.0, 1.0)
    torch.cuda.synchronize()
    x = s.copy("x")
    assert np.array_equal(bits(u.cpu().numpy()), bits(np.float32(0) + x[:n]))
    pw = np.float32(0) + np.float32(1.0 * float(wc_of(meta))) * x[3 * n:]
    if meta["reference"] >= 0:
        pw = pw - pw[meta["reference"]]
        assert p[meta["reference"]].item() == 0.0
    assert np.array_equal(bits(p.cpu().numpy()), bits(pw.astype(np.float32)))
    up = refs["updated_p"]
    err = np.linalg.norm(p.cpu().numpy().astype(np.float64) - up) / max(np.linalg.norm(up), 1e-30)
    assert err <= 1e-4, err


@pytest.mark.gpu
def test_coupled_paired_update_matches_oracle(cuda):
    """The float-pair update (coupled_solver.cpp:524-535) against the oracle's
    kpair_add restatement, with slacks that take both branches."""
    import torch
    meta, mesh, fields, refs = load("coupled_hex12x10x8_closed")
    s, _, _ = _solver(meta, mesh, fields)
    n = int(mesh["sizes"][0])
    rng = np.random.default_rng(3)
    hi = [rng.standard_normal(n).astype(np.float32) * 10 for _ in range(4)]
    lo = [rng.standard_normal(n).astype(np.float32) * 1e-6 for _ in range(4)]
    dev = [torch.from_numpy(a.copy()).cuda() for a in hi + lo]
    vs, ps, au, ap = 1e-4, 3e-5, 0.7, 0.3
    s.paired_update(*dev, au, ap, vs, ps)
    torch.cuda.synchronize()
    x = s.copy("x")
    wc = float(wc_of(meta))
    want = []
    for k in range(3):
        want.append(O.pair_add(hi[k], lo[k], np.float32(au) * x[k * n:(k + 1) * n], vs))
    ph, pl = O.pair_add(hi[3], lo[3], np.float32(ap * wc) * x[3 * n:], ps)
    ref_hi, ref_lo = ph[meta["reference"]], pl[meta["reference"]]
    want.append(O.pair_add(ph, pl, -(np.float32(ref_hi) + np.float32(ref_lo)) * np.ones(n, np.float32), ps))
    for k in range(4):
        assert np.array_equal(bits(dev[k].cpu().numpy()), bits(want[k][0])), k
        assert np.array_equal(bits(dev[4 + k].cpu().numpy()), bits(want[k][1])), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["coupled_tet6x5x4_tight", "coupled_hex12x10x8_closed"])
@pytest.mark.parametrize("wide", [None, "1"], ids=["thread_rows", "warp_rows"])
def test_coupled_coarse_kernels_match_oracle(cuda, name, wide, monkeypatch):
    """On every coarse level: the residual and the damped block-Jacobi sweep
    (from x and from zero), the member-sum restriction and the prolongation,
    on seeded vectors, bit for bit against the oracle on the reference's own
    level operator; with a thread per row (these levels' rows are short) and
    with every level forced to a warp per row."""
    import torch
    if wide is not None:
        monkeypatch.setenv("KUTTA_B200_COUPLED_WIDE_ROWS", wide)
    meta, mesh, fields, refs = load(name)
    s, _, _ = _solver(meta, mesh, fields)
    sizes, levels = ref_levels(meta, refs)
    omega = options(meta).smoother_damping
    rng = np.random.default_rng(11)
    for k, lv in enumerate(levels, start=1):
        n, nf = sizes[k], sizes[k - 1]
        lvr = {key: lv[key][: (n + 1 if key == "rows" else None)] for key in
               ("rows", "cols", "diag", "a", "c", "g", "h", "d")}
        lvr["rows"] = lv["rows"][: n + 1]
        lvr["diag"] = lv["diag"][:n]
        nnz = int(lvr["rows"][-1])
        for key in ("cols", "a", "c"):
            lvr[key] = lv[key][:nnz]
        for key in ("g", "h"):
            lvr[key] = lv[key][: 3 * nnz]
        lvr["d"] = lv["d"][: 11 * n]
        x = rng.standard_normal(4 * n).astype(np.float32)
        b = rng.standard_normal(4 * n).astype(np.float32)
        dx, db = (torch.from_numpy(_aos(v, n)).cuda() for v in (x, b))
        want = {"residual": (b - O.coarse_row(lvr, x)).astype(np.float32),
                "smooth": O.coarse_smooth(lvr, x, b, omega, False),
                "smooth_zero": O.coarse_smooth(lvr, x, b, omega, True)}
        for op, w in want.items():
            y = torch.full((4 * n,), float("nan"), dtype=torch.float32, device="cuda")
            s.level_apply(k, op, dx, db, y)
            torch.cuda.synchronize()
            assert np.array_equal(bits(_planes(y.cpu().numpy(), n)), bits(w)), (k, op)
        fine = rng.standard_normal(4 * nf).astype(np.float32)
        y = torch.zeros(4 * n, dtype=torch.float32, device="cuda")
        s.level_apply(k, "restrict", torch.from_numpy(_aos(fine, nf)).cuda(), None, y)
        torch.cuda.synchronize()
        want_r = O.restrict(lv["offsets"][: n + 1], lv["members"][:nf], fine, nf)
        assert np.array_equal(bits(_planes(y.cpu().numpy(), n)), bits(want_r)), k
        base = rng.standard_normal(4 * nf).astype(np.float32)
        yf = torch.from_numpy(_aos(base, nf)).cuda()
        s.level_apply(k, "prolong", dx, None, yf)
        torch.cuda.synchronize()
        agg = lv["aggregate"][:nf]
        want_p = np.concatenate([base[c * nf:(c + 1) * nf] + x[c * n + agg] for c in range(4)])
        assert np.array_equal(bits(_planes(yf.cpu().numpy(), nf)), bits(want_p)), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["coupled_tet6x5x4_tight", "coupled_hex12x10x8_closed"])
def test_graph_replay_changes_no_bits(cuda, name, monkeypatch):
    """Each BiCGStab iteration replayed as a CUDA graph (the default) gives
    the directly launched iterations' solution and statistics bit for bit,
    over two solves (the second replays graphs captured in the first)."""
    meta, mesh, fields, _ = load(name)
    runs = []
    for graphs in ("1", "0"):
        monkeypatch.setenv("KUTTA_B200_COUPLED_GRAPHS", graphs)
        s, st, d = _solver(meta, mesh, fields)
        rel, abs_, max_iter = meta["control"]
        st2 = s.solve(d, L.SolveControl(rel, abs_, max_iter))
        runs.append((st, st2, s.copy("x")))
    (a1, a2, ax), (b1, b2, bx) = runs
    assert (a1.iterations, a1.final_residual) == (b1.iterations, b1.final_residual)
    assert (a2.iterations, a2.final_residual) == (b2.iterations, b2.final_residual)
    assert np.array_equal(bits(ax), bits(bx))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["coupled_tet6x5x4_tight", "coupled_hex12x10x8_closed",
                                  "coupled_hex10x8x6_v22_net"])
def test_one_block_tail_changes_no_bits(cuda, name, monkeypatch):
    """The small coarse levels' V-cycle in one launch (the default on these
    sizes) gives the separate launches' solution and statistics bit for bit."""
    meta, mesh, fields, _ = load(name)
    runs = []
    for tail in ("1", "0"):
        monkeypatch.setenv("KUTTA_B200_COUPLED_TAIL", tail)
        s, st, d = _solver(meta, mesh, fields)
        rel, abs_, max_iter = meta["control"]
        st2 = s.solve(d, L.SolveControl(rel, abs_, max_iter))
        runs.append((st, st2, s.copy("x")))
    (a1, a2, ax), (b1, b2, bx) = runs
    assert (a1.iterations, a1.final_residual) == (b1.iterations, b1.final_residual)
    assert (a2.iterations, a2.final_residual) == (b2.iterations, b2.final_residual)
    assert np.array_equal(bits(ax), bits(bx))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["coupled_tet6x5x4_tight", "coupled_hex10x8x6_v22_net"])
@pytest.mark.parametrize("tail", ["1", "0"], ids=["tail", "separate"])
def test_warp_rows_change_no_bits(cuda, name, tail, monkeypatch):
    """Every separately launched coarse level with a warp per row (the levels
    of the one-block tail keep a thread per row, and with the tail off every
    level is launched separately) gives the thread-per-row solution and
    statistics bit for bit, over two solves."""
    meta, mesh, fields, _ = load(name)
    monkeypatch.setenv("KUTTA_B200_COUPLED_TAIL", tail)
    runs = []
    for wide in ("1", "0"):
        monkeypatch.setenv("KUTTA_B200_COUPLED_WIDE_ROWS", wide)
        s, st, d = _solver(meta, mesh, fields)
        rel, abs_, max_iter = meta["control"]
        st2 = s.solve(d, L.SolveControl(rel, abs_, max_iter))
        runs.append((st, st2, s.copy("x")))
    (a1, a2, ax), (b1, b2, bx) = runs
    assert (a1.iterations, a1.final_residual) == (b1.iterations, b1.final_residual)
    assert (a2.iterations, a2.final_residual) == (b2.iterations, b2.final_residual)
    assert np.array_equal(bits(ax), bits(bx))


@pytest.mark.gpu
@pytest.mark.parametrize("tet,dims,kinds,reference", [
    (False, (32, 32, 32), (1, 2, 0, 0, 3, 3), -1),
    (True, (16, 14, 12), (1, 4, 0, 3, 0, 0), -1),
    (False, (24, 20, 16), (0, 0, 0, 0, 0, 0), 7),
], ids=["hex32_open", "tet16x14x12_open", "hex24x20x16_closed"])
def test_coupled_matches_reference_at_scale(cuda, tet, dims, kinds, reference):
    """Larger meshes than the fixtures (16K to 32K cells, 4 to 5 levels, the
    one-block tail on the small ones), against the reference's CoupledSolver
    run here when oracle/_ref is present: the right-hand side, the cell data
    and every coarse level bit for bit, the same iterations, the solution to
    1e-4."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from kutta_b200 import coupled_harness as H
    case = ref.CoupledCase(tet, *dims, patch_kinds=kinds)
    fields = H.flow_fields(case.arrays, 21, reference=reference)
    want = case.solve(fields, ref.coupled_options(), rel_tol=1e-3, max_iter=60)
    meta = {"reference": reference, "options": {}, "control": (1e-3, 1e-12, 60),
            "density": fields["density"], "velocity_scale": fields["velocity_scale"]}
    s, st, _ = _solver(meta, case.arrays, fields)
    assert s.describe() == want["describe"]
    n = int(case.arrays["sizes"][0])
    assert np.array_equal(bits(s.copy("rhs")), bits(want["rhs"]))
    assert np.array_equal(bits(s.copy("cell")), bits(want["cell"][: 27 * n]))
    sizes, levels = ref_levels({"describe": want["describe"]}, want)
    for k, lv in enumerate(levels, start=1):
        got = s.level(k)
        for key in ("rows", "cols", "diag", "a", "c", "g", "h", "d"):
            assert np.array_equal(bits(got[key]), bits(lv[key][: len(got[key])])), (k, key)
    assert st.iterations == want["iterations"]
    assert st.converged == want["converged"]
    assert st.final_residual == pytest.approx(want["final_residual"], rel=1e-2)
    x = s.copy("x")
    err = np.linalg.norm(x.astype(np.float64) - want["x"]) / np.linalg.norm(want["x"])
    assert err <= 1e-4, err



def _paired_oracle(hi, lo, x, n, au, ap, vs, ps, wc, reference):
    """The reference's paired update restated (coupled_paired_update and, for
    a closed domain, the paired pick and gauge), planes u | v | w | p."""
    out = []
    for k in range(3):
        out.append(O.pair_add(hi[k * n:(k + 1) * n], lo[k * n:(k + 1) * n],
                              np.float32(au) * x[k * n:(k + 1) * n], vs))
    ph, pl = O.pair_add(hi[3 * n:], lo[3 * n:], np.float32(ap * float(wc)) * x[3 * n:], ps)
    if reference >= 0:
        shift = -(np.float32(ph[reference]) + np.float32(pl[reference]))
        ph, pl = O.pair_add(ph, pl, np.full(n, shift, np.float32), ps)
    out.append((ph, pl))
    return out


def test_oracle_pair_update_reproduces_reference():
    """The oracle's paired update on the reference's own solution and hi/lo
    fields gives the reference's paired update bit for bit (kpair_add,
    prelude.h:139-149)."""
    meta, mesh, _, refs = load("coupled_tet5x4x3_loworder_paired")
    n = int(mesh["sizes"][0])
    au, ap, vs, ps = meta["pairs"]
    want = _paired_oracle(refs["pair_hi"], refs["pair_lo"], refs["x"], n, au, ap, vs, ps,
                          wc_of(meta), meta["reference"])
    for k, c in enumerate("uvwp"):
        assert np.array_equal(bits(want[k][0]), bits(refs[f"paired_{c}"])), c
        assert np.array_equal(bits(want[k][1]), bits(refs[f"paired_{c}_lo"])), c


@pytest.mark.gpu
def test_coupled_paired_update_on_low_order_mesh(cuda):
    """On a mesh with low-order pressure cells: the solve takes the
    reference's iterations, and the device's paired update equals the
    oracle's (pinned to the reference above) on the device's solution, and the
    reference's own result bit for bit when the two solutions agree bit for
    bit."""
    import torch
    name = "coupled_tet5x4x3_loworder_paired"
    meta, mesh, fields, refs = load(name)
    assert "low_order" in mesh
    s, st, _ = _solver(meta, mesh, fields)
    assert st.iterations == meta["iterations"]
    n = int(mesh["sizes"][0])
    au, ap, vs, ps = meta["pairs"]
    hi = [torch.from_numpy(refs["pair_hi"][k * n:(k + 1) * n].copy()).cuda() for k in range(4)]
    lo = [torch.from_numpy(refs["pair_lo"][k * n:(k + 1) * n].copy()).cuda() for k in range(4)]
    s.paired_update(*hi, *lo, au, ap, vs, ps)
    torch.cuda.synchronize()
    x = s.copy("x")
    want = _paired_oracle(refs["pair_hi"], refs["pair_lo"], x, n, au, ap, vs, ps, wc_of(meta),
                          meta["reference"])
    same_x = np.array_equal(bits(x), bits(refs["x"]))
    for k, c in enumerate("uvwp"):
        assert np.array_equal(bits(hi[k].cpu().numpy()), bits(want[k][0])), c
        assert np.array_equal(bits(lo[k].cpu().numpy()), bits(want[k][1])), c
        if same_x:
            assert np.array_equal(bits(hi[k].cpu().numpy()), bits(refs[f"paired_{c}"])), c


@pytest.mark.parametrize("tet,dims,lo,hi,kinds", [
    (False, (3, 2, 2), (0, 0, 0), (3, 2, 2), None),
    (False, (7, 5, 4), (0, 0, 0), (1, 1, 1), None),
    (False, (6, 4, 5), (-1, 0.5, 0), (2, 1, 0.25), None),
    (True, (3, 2, 2), (0, 0, 0), (3, 2, 2), None),
    (True, (5, 4, 3), (0, 0, 0), (1, 1, 1), "normal"),
    (True, (4, 3, 5), (-1, 0.5, 0), (2, 1, 0.25), None)])
def test_box_matches_reference_arrays(tet, dims, lo, hi, kinds):
    """coupled_harness.box_hex / box_tet (the bench's meshes, built without
    the reference) give the reference's arrays for the same box, bit for bit
    but for the least-squares inverse (to double round-off). On the tets the
    pressure fit observes walls and symmetry planes at the normal foot, which
    differs from the face centroid."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from kutta_b200 import coupled_harness as H
    kw = {}
    if kinds == "normal":
        kw["patch_kinds"] = (H.INLET, H.OUTLET_NORMAL, H.WALL, H.SYMMETRY, H.WALL, H.WALL)
    want = ref.CoupledCase(tet, *dims, lo=lo, hi=hi, **kw).arrays
    got = (H.box_tet if tet else H.box_hex)(*dims, lo=lo, hi=hi, **kw)
    assert set(got) <= set(want)
    for k, v in got.items():
        w = want[k]
        assert v.shape == w.shape, k
        if k != "lsq_inverse":
            # The geometry restates the reference's double operations in their
            # order, so every array but the fit's inverse (a Jacobi eigensolve
            # there) is the same bits.
            assert np.array_equal(v, w), k
        else:
            assert np.allclose(v.astype(np.float64), w.astype(np.float64), rtol=1e-6, atol=1e-12), k


@pytest.mark.parametrize("tet,side", [(False, 24), (True, 20), (True, 40)])
def test_box_hierarchy_matches_reference(tet, side):
    """On the generated boxes the host setup forms the reference's aggregation
    hierarchy and pressure-force sensitivities: the aggregation ties of the
    regular boxes fall the same way only when the geometry's doubles are the
    reference's. The 40^3 x 6 tet box (384,000 cells) has the hub aggregates
    of tet hierarchies: rows of 41 and 83 entries on its two smallest levels."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from kutta_b200 import coupled_harness as H
    from kutta_b200 import linalg as L
    want = L.build_coupled_setup(ref.CoupledCase(tet, side, side, side).arrays,
                                 L.CoupledOptions())
    got = L.build_coupled_setup((H.box_tet if tet else H.box_hex)(side, side, side),
                                L.CoupledOptions())
    assert [lv["n"] for lv in got["levels"]] == [lv["n"] for lv in want["levels"]]
    for g, w in zip(got["levels"], want["levels"]):
        for k, v in w.items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(g[k], v), k
    assert np.max(np.abs(got["cell"] - want["cell"])) <= 1e-6 * np.max(np.abs(want["cell"]))
