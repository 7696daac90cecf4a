"""The learned preconditioner stage (no reference counterpart): the CUDA
forward, backward and Adam kernels against a plain PyTorch FP32 statement of
the same network and energy loss, training that lowers the loss, and the stage
attached to the mixed solve (which must still meet its FP64 tolerance, and
whose safeguarded step never raises the error's A-energy)."""
import numpy as np
import pytest

from kutta_b200 import harness
from kutta_b200 import linalg as L

HIDDEN = 32


def _layers(w):
    """(Ws, Wn, b) per layer and wo from the flat parameter vector."""
    out, k = [], 0
    for cin in (1, HIDDEN, HIDDEN):
        ws = w[k:k + HIDDEN * cin].reshape(HIDDEN, cin); k += HIDDEN * cin
        wn = w[k:k + HIDDEN * cin].reshape(HIDDEN, cin); k += HIDDEN * cin
        b = w[k:k + HIDDEN]; k += HIDDEN
        out.append((ws, wn, b))
    return out, w[k:k + HIDDEN]


def _torch_operators(s):
    """Edge-weight matrix W, node scales and A (FP32 CUDA tensors) of system s."""
    import torch
    n = s.n
    rows = np.repeat(np.arange(n), np.diff(s.row_ptr))
    vals = s.val.astype(np.float32)
    d = vals[s.diag]
    off = rows != s.col
    edge = np.zeros_like(vals)
    edge[off] = -vals[off] / np.sqrt(d[rows[off]] * d[s.col[off]])
    idx = np.vstack([rows, s.col])
    W = torch.sparse_coo_tensor(idx, torch.from_numpy(edge), (n, n)).cuda()
    A = torch.sparse_coo_tensor(idx, torch.from_numpy(vals), (n, n)).cuda()
    scale = torch.from_numpy(1.0 / np.sqrt(d)).cuda()
    return W, scale, A


def _torch_network(s):
    """The network in PyTorch FP32 for system s: returns f(w, r) -> z."""
    import torch
    W, scale, _ = _torch_operators(s)

    def f(w, r):
        layers, wo = _layers(w)
        h0 = scale * r
        rho = torch.sqrt((h0.double() ** 2).mean()).float()
        h = (h0 / rho)[:, None]
        for ws, wn, b in layers:
            m = torch.sparse.mm(W, h)
            h = torch.relu(h @ ws.T + m @ wn.T + b)
        return rho * scale * (h @ wo)
    return f


def _torch_network_bf16(s):
    """The tensor-core forward's arithmetic in PyTorch: layer 1 in FP32, the
    A-tile operands [H | W H] and the 32-wide weights rounded to BF16, FP32
    accumulation, the hidden rows stored in BF16."""
    import torch
    W, scale, _ = _torch_operators(s)

    def bf(x):
        return x.to(torch.bfloat16).float()

    def f(w, r):
        (l1, l2, l3), wo = _layers(w)
        h0 = scale * r
        rho = torch.sqrt((h0.double() ** 2).mean()).float()
        u = (h0 / rho)[:, None]
        v = torch.sparse.mm(W, u)
        h1 = torch.relu(u @ l1[0].T + v @ l1[1].T + l1[2])
        m1 = torch.sparse.mm(W, h1)
        h2 = bf(torch.relu(torch.cat([bf(h1), bf(m1)], 1) @ bf(torch.cat(l2[:2], 1)).T + l2[2]))
        m2 = torch.sparse.mm(W, h2)
        h3 = torch.relu(torch.cat([h2, bf(m2)], 1) @ bf(torch.cat(l3[:2], 1)).T + l3[2])
        return rho * scale * (h3 @ wo)
    return f


def _energy_loss(s, f, w, t, e):
    import torch
    _, _, A = _torch_operators(s)
    c = f(w, t)
    q = torch.sparse.mm(A, c[:, None])[:, 0]
    P, Q, E = (c * t).sum(), (c * q).sum(), (t.double() * e.double()).sum().float()
    return 1 - P * P / (Q * E)


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def _setup(seed=3, n_side=8):
    import torch
    s = harness.box_system(n_side, n_side, n_side, tet=True, seed=seed)
    a = L.upload(s)
    g = L.LearnedStage(seed=seed)
    g.bind(a)
    r = torch.from_numpy(np.random.default_rng(seed).normal(size=s.n).astype(np.float32)).cuda()
    return s, a, g, r


def _pair(s, a, solver):
    """(t, e) with A e = t: the error of one preconditioner application to b."""
    import scipy.sparse as sp
    import torch
    A = sp.csr_matrix((s.val.astype(np.float64), s.col, s.row_ptr), shape=(s.n, s.n))
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    b = torch.from_numpy(s.b).cuda()
    solver.solve(a, x, b, L.SolveControl(1e-10, 1e-30, 3000))
    z = torch.zeros(s.n, dtype=torch.float32, device="cuda")
    solver.precondition(a, b, z)
    zc = z.double().cpu().numpy()
    t = s.b.astype(np.float64) - A @ zc
    e = x.cpu().numpy() - zc
    return (torch.from_numpy(t.astype(np.float32)).cuda(),
            torch.from_numpy(e.astype(np.float32)).cuda(), A, x.cpu().numpy(), zc)


@pytest.mark.gpu
@pytest.mark.parametrize("n_side", [9, 40])
def test_forward_matches_torch(cuda, n_side):
    """The tensor-core forward (b2_gnn_apply) against its arithmetic in
    PyTorch and against the FP32 network; 9^3 tets end in a partial 128-row
    tile, 40^3 tets give every CTA several tiles."""
    import torch
    s, a, g, r = _setup(n_side=n_side)
    z = torch.zeros(s.n, device="cuda")
    g.apply(r, z)
    w = torch.from_numpy(g.weights()).cuda()
    emulated = _torch_network_bf16(s)(w, r)
    fp32 = _torch_network(s)(w, r)
    torch.cuda.synchronize()
    assert torch.isfinite(z).all()
    assert _rel(z, emulated) < 2e-3
    assert _rel(z, fp32) < 3e-2
    # beta = 1 adds to z.
    z2 = z.clone()
    g.apply(r, z2, beta=1.0)
    assert torch.equal(z2, 2 * z)
    # Positive homogeneity: G(lambda r) = lambda G(r) (the input is normalised).
    z3 = torch.zeros_like(z)
    g.apply(1e-3 * r, z3)
    assert _rel(z3, 1e-3 * z) < 1e-2


@pytest.mark.gpu
def test_given_up_wait_reports_timeout_and_the_stage_recovers(cuda):
    """The forward's bounded wait for each tile's MMA: with the first wait's
    poll limit at 0 every tile gives up at once while its MMA is healthy.
    Each block records the fault, waits for its MMA again with the full
    bound, frees its tensor memory and returns, and the call raises
    DeviceTimeout (B2_TIMEOUT). With the bound restored, the next call on the
    same stage succeeds and gives the same result as before."""
    import torch
    s, a, g, r = _setup(n_side=9)
    want = torch.zeros(s.n, device="cuda")
    g.apply(r, want)
    g.set_wait_limit(0)
    z = torch.zeros(s.n, device="cuda")
    with pytest.raises(L.DeviceTimeout):
        g.apply(r, z)
    g.set_wait_limit(-1)
    again = torch.zeros(s.n, device="cuda")
    g.apply(r, again)
    torch.cuda.synchronize()
    assert torch.equal(again, want)


@pytest.mark.gpu
def test_training_step_follows_torch_gradient(cuda):
    """One Adam step from zero moments moves every weight by about
    -lr sign(gradient): the signs of the CUDA step must be those of PyTorch's
    autograd gradient of the energy loss wherever that gradient is clearly
    nonzero, and the losses must agree."""
    import torch
    s, a, g, _ = _setup(seed=4)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    t, e, *_ = _pair(s, a, solver)
    w0 = g.weights()
    wt = torch.from_numpy(w0).cuda().requires_grad_(True)
    loss_t = _energy_loss(s, _torch_network(s), wt, t, e)
    loss_t.backward()
    grad = wt.grad.cpu().numpy()
    loss = g.train_step(t, e, learning_rate=1e-4)
    assert 0.0 <= loss <= 1.0
    assert loss == pytest.approx(float(loss_t), rel=1e-3, abs=1e-5)
    step = g.weights() - w0
    # The step's backward runs its 32-wide layers on the tensor cores (BF16
    # operands): components within ~1 % of zero may take either sign.
    clear = np.abs(grad) > 1e-2 * np.abs(grad).max()
    assert clear.sum() > 100
    assert np.mean(np.sign(step[clear]) == -np.sign(grad[clear])) > 0.99


def _parameter_blocks():
    """(name, slice) of each weight block: per layer Ws, Wn, b; then wo."""
    out, k = [], 0
    for layer, cin in enumerate((1, HIDDEN, HIDDEN)):
        for name, size in (("ws", HIDDEN * cin), ("wn", HIDDEN * cin), ("b", HIDDEN)):
            out.append((f"{name}{layer}", slice(k, k + size)))
            k += size
    out.append(("wo", slice(k, k + HIDDEN)))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n_side", [9, 40])
def test_tensor_core_backward_matches_fp32_and_autograd(cuda, n_side):
    """The training backward with the 32-wide layers' products on the tensor
    cores ([dH | dM] = G [Ws | Wn] per 128-row tile, [H | M | 1]^T G summed in
    tensor memory; BF16 operands, FP32 accumulation) against the same
    backward in FP32 on CUDA cores and against PyTorch autograd, weight block
    by weight block. Tolerances: 1e-3 relative for FP32 against autograd, 3e-2
    for the tensor cores (BF16 operands carry 8 significant bits). 9^3 tets
    end in a partial tile; 40^3 tets give every CTA several tiles."""
    import torch
    s, a, g, _ = _setup(seed=4, n_side=n_side)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    t, e, *_ = _pair(s, a, solver)
    wt = torch.from_numpy(g.weights()).cuda().requires_grad_(True)
    loss_t = _energy_loss(s, _torch_network(s), wt, t, e)
    loss_t.backward()
    auto = wt.grad.cpu().numpy().astype(np.float64)
    tc, loss_tc = g.gradient(t, e, tensor_cores=True)
    fp, loss_fp = g.gradient(t, e, tensor_cores=False)
    assert loss_tc == pytest.approx(loss_fp, rel=1e-6, abs=1e-7)
    assert loss_fp == pytest.approx(float(loss_t), rel=1e-3, abs=1e-5)
    scale = np.linalg.norm(auto)
    for name, sl in _parameter_blocks():
        ref = auto[sl]
        denom = max(np.linalg.norm(ref), 1e-3 * scale)
        assert np.linalg.norm(fp[sl] - ref) / denom < 1e-3, name
        assert np.linalg.norm(tc[sl] - ref) / denom < 3e-2, name


@pytest.mark.gpu
def test_training_lowers_the_loss(cuda):
    """Fitting one (residual, error) pair of the mixed preconditioner."""
    s, a, g, _ = _setup(seed=5, n_side=10)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    t, e, *_ = _pair(s, a, solver)
    losses = [g.train_step(t, e, learning_rate=3e-3) for _ in range(300)]
    assert np.mean(losses[-20:]) < np.mean(losses[:5]) - 0.05


@pytest.mark.gpu
def test_precondition_step_never_raises_the_energy(cuda):
    """With the stage attached after the cycle, one preconditioner application
    z' = M(r) + alpha G(t) has an A-norm error no larger than M(r)'s: the
    step is the energy-optimal one along G(t), clipped at zero."""
    import torch
    s = harness.box_system(12, 12, 12, tet=True, seed=8)
    a = L.upload(s)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    t, e, A, x, zc = _pair(s, a, solver)
    g = L.LearnedStage(seed=8)
    solver.set_learned(g, L.LEARNED_CYCLE)
    z = torch.zeros(s.n, dtype=torch.float32, device="cuda")
    solver.precondition(a, torch.from_numpy(s.b).cuda(), z)
    zl = z.double().cpu().numpy()

    def energy(v):
        d = x - v
        return float(d @ (A @ d))
    assert energy(zl) <= energy(zc) * (1 + 1e-5)
    solver.set_learned(None)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [L.LEARNED_CYCLE, L.LEARNED_WARM_START,
                                  L.LEARNED_CYCLE | L.LEARNED_WARM_START])
def test_learned_stage_in_mixed_solve(cuda, mode):
    """With the stage attached (even untrained) the mixed solve still meets the
    FP64 tolerance relative to the caller's initial residual; detaching
    restores the plain mixed solve."""
    import scipy.sparse as sp
    import torch
    s = harness.box_system(16, 16, 16, tet=True, seed=6)
    a = L.upload(s)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    r0 = np.linalg.norm(s.b.astype(np.float64))
    for attached in (True, False):
        g = L.LearnedStage(seed=6)
        solver.set_learned(g if attached else None, mode)
        text = solver.describe()
        assert ("learned stage" in text) == (attached and bool(mode & L.LEARNED_CYCLE))
        assert ("learned warm start" in text) == (attached and bool(mode & L.LEARNED_WARM_START))
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
        torch.cuda.synchronize()
        true = np.linalg.norm(s.b.astype(np.float64) - A @ x.cpu().numpy())
        assert st.converged, st
        assert st.initial_residual == pytest.approx(r0, rel=1e-6)
        assert true <= 1e-8 * st.initial_residual * 1.0001
    solver.set_learned(None)


@pytest.mark.gpu
def test_warm_start_never_raises_the_residual(cuda):
    """The learned warm start's step along c = G(b - A x0) has the length that
    minimises the new residual, clipped at zero: with max_iter = 0 the solve
    returns right after the warm start, and its FP64 residual is no larger
    than the initial one (here on a white-noise right-hand side, where the
    energy-optimal length would raise it)."""
    import scipy.sparse as sp
    import torch
    from kutta_b200 import learn
    s = harness.box_system(16, 16, 16, tet=True, seed=9)
    a = L.upload(s)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    stage = learn.trained_stage()
    solver.set_learned(stage, L.LEARNED_WARM_START)
    b = torch.from_numpy(s.b).cuda()
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    st = solver.solve(a, x, b, L.SolveControl(1e-6, 1e-30, 0))
    torch.cuda.synchronize()
    solver.set_learned(None)
    assert st.iterations == 0
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    true = float(np.linalg.norm(s.b.astype(np.float64) - A @ x.cpu().numpy()))
    assert true == pytest.approx(st.final_residual, rel=1e-6)
    assert st.final_residual <= st.initial_residual
    assert np.any(x.cpu().numpy() != 0.0)  # a step was taken


@pytest.mark.gpu
def test_learned_mode_is_validated(cuda):
    s = harness.box_system(6, 6, 6, tet=True, seed=2)
    a = L.upload(s)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    g = L.LearnedStage(seed=2)
    for bad in (0, 4, -1):
        with pytest.raises(L.KuttaError):
            solver.set_learned(g, bad)


@pytest.mark.gpu
def test_nonfinite_network_output_leaves_the_solve_unchanged(cuda):
    """A stage whose output is not finite gets no step (alpha 0 and the
    update skipped, since 0 * NaN is NaN): the solve equals the solve without
    a stage, bit for bit, in both modes."""
    import torch
    s = harness.box_system(14, 14, 14, tet=True, seed=16)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    out = []
    for poisoned in (False, True):
        solver = L.make_mixed_solver(s)
        solver.refresh(a)
        if poisoned:
            g = L.LearnedStage(seed=2)
            w = g.weights()
            w[-L.LearnedStage.parameter_count() // 4:] = np.nan
            g.set_weights(w)
            solver.set_learned(g, L.LEARNED_CYCLE | L.LEARNED_WARM_START)
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
        assert st.converged and not st.learned_fallback
        out.append((st.iterations, st.final_residual, x.cpu().numpy()))
        if poisoned:
            solver.set_learned(None)
    assert out[0][:2] == out[1][:2]
    assert np.array_equal(out[0][2].view(np.uint64), out[1][2].view(np.uint64))


@pytest.mark.gpu
def test_stalled_refinement_falls_back_to_the_amg_cycle(cuda):
    """The plain AMG cycle is the learned stage's fallback: asked for a
    tolerance below the FP64 floor, the refinement must stall; the stage is
    then detached for the rest of the solve, re-attached afterwards, and a
    normal solve with it still meets its tolerance."""
    import torch
    s = harness.box_system(12, 12, 12, tet=True, seed=17)
    a = L.upload(s)
    b = torch.from_numpy(s.b).cuda()
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    g = L.LearnedStage(seed=3)
    solver.set_learned(g, L.LEARNED_CYCLE)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    st = solver.solve(a, x, b, L.SolveControl(1e-20, 0.0, 3000))
    assert st.learned_fallback and not st.converged
    assert "learned stage" in solver.describe()
    x.zero_()
    st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
    assert st.converged and not st.learned_fallback
    solver.set_learned(None)


def _gate_inputs(s):
    """Per entry: the ungated edge weight w, the geometry feature rho and the
    device geometry array (float32), as the stage computes them at bind."""
    import torch
    n = s.n
    rows = np.repeat(np.arange(n), np.diff(s.row_ptr))
    vals = s.val.astype(np.float32)
    d = vals[s.diag]
    off = rows != s.col
    w = np.zeros_like(vals)
    w[off] = -vals[off] / np.sqrt(d[rows[off]] * d[s.col[off]])
    g = s.geometry.astype(np.float32)
    G = np.add.reduceat(g.astype(np.float64), s.row_ptr[:-1]).astype(np.float32)
    gh = np.zeros_like(g)
    ok = off & (g > 0) & (w > 0)
    gh[ok] = g[ok] / np.sqrt(G[rows[ok]] * G[s.col[ok]])
    rho = np.zeros_like(g)
    rho[ok] = np.clip(np.log(gh[ok] / w[ok]), -20, 20)
    return rows, w, rho, torch.from_numpy(g).cuda()


def _torch_network_gated(s):
    """The network with the geometry gate E = w exp(theta_0 tanh(theta_1 rho))
    (the last two parameters), in PyTorch FP32, differentiable in theta."""
    import torch
    rows, w, rho, _ = _gate_inputs(s)
    idx = torch.from_numpy(np.vstack([rows, s.col])).cuda()
    w_t, rho_t = torch.from_numpy(w).cuda(), torch.from_numpy(rho).cuda()
    _, scale, _ = _torch_operators(s)

    def f(p, r):
        layers, wo = _layers(p)
        gamma = torch.exp(p[-2] * torch.tanh(p[-1] * rho_t))
        W = torch.sparse_coo_tensor(idx, w_t * gamma, (s.n, s.n))
        h0 = scale * r
        rms = torch.sqrt((h0.double() ** 2).mean()).float()
        h = (h0 / rms)[:, None]
        for ws, wn, b in layers:
            m = torch.sparse.mm(W, h)
            h = torch.relu(h @ ws.T + m @ wn.T + b)
        return rms * scale * (h @ wo)
    return f


@pytest.mark.gpu
def test_geometry_gate_is_off_at_zero_theta(cuda):
    """With theta = 0 the gate is exactly 1: binding the geometry changes no
    bit of the forward."""
    import torch
    s, a, g, r = _setup(seed=5, n_side=9)
    want = torch.zeros(s.n, device="cuda")
    g.apply(r, want)
    _, _, _, geometry = _gate_inputs(s)
    g.set_geometry(geometry)
    g.bind(a)
    z = torch.zeros(s.n, device="cuda")
    g.apply(r, z)
    torch.cuda.synchronize()
    assert torch.equal(z, want)


@pytest.mark.gpu
def test_geometry_gate_forward_and_gradient_match_torch(cuda):
    """theta = (0.4, 0.3): the tensor-core forward against PyTorch FP32 (3e-2,
    BF16 operands), and the FP32 backward's gradient, theta included, against
    autograd (1e-3)."""
    import torch
    s, a, g, r = _setup(seed=6, n_side=10)
    _, _, _, geometry = _gate_inputs(s)
    g.set_geometry(geometry)
    w = g.weights()
    w[-2:] = (0.4, 0.3)
    g.set_weights(w)
    g.bind(a)
    f = _torch_network_gated(s)
    z = torch.zeros(s.n, device="cuda")
    g.apply(r, z)
    want = f(torch.from_numpy(w).cuda(), r)
    assert _rel(z, want) < 3e-2
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    t, e, *_ = _pair(s, a, solver)
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    loss_t = _energy_loss(s, f, wt, t, e)
    loss_t.backward()
    auto = wt.grad.cpu().numpy().astype(np.float64)
    fp, loss_fp = g.gradient(t, e, tensor_cores=False)
    assert loss_fp == pytest.approx(float(loss_t), rel=1e-3, abs=1e-5)
    scale = np.linalg.norm(auto)
    for name, sl in _parameter_blocks() + [("theta", slice(-2, None))]:
        ref = auto[sl]
        denom = max(np.linalg.norm(ref), 1e-3 * scale)
        assert np.linalg.norm(fp[sl] - ref) / denom < 1e-3, name
    assert np.abs(auto[-2:]).max() > 0
