"""The learned preconditioner stage (no reference counterpart): the CUDA
forward, backward and Adam kernels against a plain PyTorch FP32 statement of
the same network, training that lowers the loss, and the stage attached to the
mixed solve (which must still meet its FP64 tolerance)."""
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


def _torch_network(s):
    """The network in PyTorch FP32 for system s: returns f(w, r) -> z."""
    import torch
    n = s.n
    rows = np.repeat(np.arange(n), np.diff(s.row_ptr))
    vals = s.val.astype(np.float32)
    d = vals[s.diag]
    off = rows != s.col
    edge = np.zeros_like(vals)
    edge[off] = -vals[off] / np.sqrt(d[rows[off]] * d[s.col[off]])
    W = torch.sparse_coo_tensor(np.vstack([rows, s.col]), torch.from_numpy(edge), (n, n)).cuda()
    scale = torch.from_numpy(1.0 / np.sqrt(d)).cuda()

    def f(w, r):
        layers, wo = _layers(w)
        h = (scale * r)[:, None]
        for ws, wn, b in layers:
            m = torch.sparse.mm(W, h)
            h = torch.relu(h @ ws.T + m @ wn.T + b)
        return scale * (h @ wo)
    return f


def _setup(seed=3, n_side=8):
    import torch
    s = harness.box_system(n_side, n_side, n_side, tet=True, seed=seed)
    a = L.upload(s)
    g = L.LearnedStage(seed=seed)
    g.bind(a)
    r = torch.from_numpy(np.random.default_rng(seed).normal(size=s.n).astype(np.float32)).cuda()
    return s, a, g, r


@pytest.mark.gpu
def test_forward_matches_torch(cuda):
    import torch
    s, a, g, r = _setup()
    z = torch.zeros(s.n, device="cuda")
    g.apply(r, z)
    w = torch.from_numpy(g.weights()).cuda()
    want = _torch_network(s)(w, r)
    torch.cuda.synchronize()
    assert torch.allclose(z, want, rtol=1e-4, atol=1e-5 * float(want.abs().max()))
    # beta = 1 adds to z.
    z2 = z.clone()
    g.apply(r, z2, beta=1.0)
    assert torch.allclose(z2, 2 * z, rtol=1e-5, atol=1e-6 * float(z.abs().max()))


@pytest.mark.gpu
def test_training_step_follows_torch_gradient(cuda):
    """One Adam step from zero moments moves every weight by about
    -lr sign(gradient): the signs of the CUDA step must be those of PyTorch's
    autograd gradient wherever that gradient is clearly nonzero."""
    import torch
    s, a, g, b = _setup(seed=4)
    x = torch.from_numpy(np.random.default_rng(7).normal(size=s.n).astype(np.float32)).cuda()
    w0 = g.weights()
    wt = torch.from_numpy(w0).cuda().requires_grad_(True)
    f = _torch_network(s)
    loss_t = ((f(wt, b) - x) ** 2).sum() / (x.double() ** 2).sum().float()
    loss_t.backward()
    grad = wt.grad.cpu().numpy()
    loss = g.train_step(b, x, learning_rate=1e-4)
    assert loss == pytest.approx(float(loss_t), rel=1e-4)
    step = g.weights() - w0
    clear = np.abs(grad) > 1e-3 * np.abs(grad).max()
    assert clear.sum() > 100
    assert np.mean(np.sign(step[clear]) == -np.sign(grad[clear])) > 0.99


@pytest.mark.gpu
def test_training_lowers_the_loss(cuda):
    """Fitting G(b) ~ x for the solver's own solution of A x = b."""
    import torch
    s, a, g, _ = _setup(seed=5, n_side=10)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    x64 = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    solver.solve(a, x64, b, L.SolveControl(1e-8, 1e-30, 2000))
    x = x64.float()
    losses = [g.train_step(b, x, learning_rate=3e-3) for _ in range(300)]
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5])


@pytest.mark.gpu
def test_learned_stage_in_mixed_solve(cuda):
    """With the stage attached (even untrained) the flexible inner PCG still
    meets the FP64 tolerance; detaching restores the plain mixed solve."""
    import scipy.sparse as sp
    import torch
    s = harness.box_system(16, 16, 16, tet=True, seed=6)
    a = L.upload(s)
    solver = L.make_mixed_solver(s)
    solver.refresh(a)
    b = torch.from_numpy(s.b).cuda()
    A = sp.csr_matrix((s.val, s.col, s.row_ptr), shape=(s.n, s.n))
    stats = {}
    for attached in (True, False):
        g = L.LearnedStage(seed=6)
        solver.set_learned(g if attached else None)
        assert ("learned stage" in solver.describe()) == attached
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        st = solver.solve(a, x, b, L.SolveControl(1e-8, 1e-30, 3000))
        torch.cuda.synchronize()
        true = np.linalg.norm(s.b.astype(np.float64) - A @ x.cpu().numpy())
        assert st.converged, st
        assert true <= 1e-8 * st.initial_residual * 1.0001
        stats[attached] = st
    solver.set_learned(None)
