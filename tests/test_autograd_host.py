"""Host logic of the torch.autograd wrapper (parflow_b200/autograd.py) on CPU.

The GPU handle is replaced by a linear stand-in whose adjoint is known in
closed form: observed pressures p = A [lnK; alpha; n] + p0, and the stand-in's
adjoint_gradient returns, like pfgpu_adjoint_gradient, the misfit
sum (p - obs)^2 and its gradient A^T 2 (p - obs).  The wrapper must turn that
into the exact vector-Jacobian product A^T w for any upstream gradient w,
including tiny w on large p (the scaling), and must re-solve a forward whose
trajectory the handle no longer holds.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from parflow_b200 import autograd as AG  # noqa: E402

SHAPE = (3, 4, 5)
NSTEPS, NCELLS = 2, 6


class _FakeGPU:
    def __init__(self, owner):
        self.owner = owner

    def adjoint_gradient(self, obs_steps, obs_cells, obs_values, tol=1e-10):
        p = self.owner.current
        r = p - np.asarray(obs_values).reshape(p.shape)
        g = self.owner.A.T @ (2.0 * r.ravel())
        n = int(np.prod(SHAPE))
        return float(np.sum(r * r)), g[:n].reshape(SHAPE), g[n:2 * n].reshape(SHAPE), \
            g[2 * n:].reshape(SHAPE)


class _LinearModel(AG.RichardsAdjointModel):
    def __init__(self, seed=0, offset=100.0):
        rng = np.random.default_rng(seed)
        n = int(np.prod(SHAPE))
        self.A = rng.standard_normal((NSTEPS * NCELLS, 3 * n))
        self.p0 = offset + rng.standard_normal(NSTEPS * NCELLS)
        self.gpu = _FakeGPU(self)
        self.obs_steps = np.arange(1, NSTEPS + 1, dtype=np.int32)
        self.obs_cells = np.arange(NCELLS, dtype=np.int64)
        self.prob = type("P", (), {"shape": SHAPE})()
        self.tol = 1e-12
        self._recorded = None
        self._tokens = 0
        self.forwards = 0

    def forward(self, lnk, alpha, vg_n):
        theta = np.concatenate([np.ravel(lnk), np.ravel(alpha), np.ravel(vg_n)])
        self.current = (self.A @ theta + self.p0).reshape(NSTEPS, NCELLS)
        self.forwards += 1
        self._tokens += 1
        self._recorded = self._tokens
        return self.current.copy(), self._recorded


def _fields(seed):
    rng = np.random.default_rng(seed)
    return [torch.tensor(rng.standard_normal(SHAPE), dtype=torch.float64, requires_grad=True)
            for _ in range(3)]


def _expected(model, w):
    g = model.A.T @ np.ravel(w)
    n = int(np.prod(SHAPE))
    return g[:n].reshape(SHAPE), g[n:2 * n].reshape(SHAPE), g[2 * n:].reshape(SHAPE)


def test_vjp_of_nonlinear_loss():
    m = _LinearModel()
    lnk, a, n = _fields(1)
    p = AG.observe(lnk, a, n, m)
    assert p.shape == (NSTEPS, NCELLS)
    c = torch.linspace(-1.0, 2.0, NSTEPS * NCELLS, dtype=torch.float64).reshape(NSTEPS, NCELLS)
    loss = (c * torch.sin(p / 50.0)).sum()
    loss.backward()
    w = (c * torch.cos(p / 50.0) / 50.0).detach().numpy()
    for got, want in zip((lnk.grad, a.grad, n.grad), _expected(m, w)):
        assert np.allclose(got.numpy(), want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_tiny_upstream_gradient_keeps_its_digits():
    """w ~ 1e-12 on p ~ 1e4: without scaling p - (p - w/2) would lose w."""
    m = _LinearModel(offset=1e4)
    lnk, a, n = _fields(2)
    p = AG.observe(lnk, a, n, m)
    w = 1e-12 * torch.arange(1, NSTEPS * NCELLS + 1, dtype=torch.float64).reshape(p.shape)
    (p * w).sum().backward()
    for got, want in zip((lnk.grad, a.grad, n.grad), _expected(m, w.numpy())):
        assert np.allclose(got.numpy(), want, rtol=1e-10, atol=1e-10 * np.abs(want).max())


def test_misfit_matches_quadratic_and_zero_gradient():
    m = _LinearModel()
    lnk, a, n = _fields(3)
    obs = np.random.default_rng(4).standard_normal((NSTEPS, NCELLS)) + 100.0
    j = AG.misfit(lnk, a, n, m, obs)
    sim = AG.observe(lnk, a, n, m).detach().numpy()
    jv = j.item()
    assert abs(jv - float(np.sum((sim - obs) ** 2))) <= 1e-9 * jv
    j.backward()
    for got, want in zip((lnk.grad, a.grad, n.grad), _expected(m, 2.0 * (sim - obs))):
        assert np.allclose(got.numpy(), want, rtol=1e-10, atol=1e-10 * np.abs(want).max())
    # zero upstream gradient: zero parameter gradients, no adjoint solve
    lnk2, a2, n2 = _fields(5)
    (0.0 * AG.observe(lnk2, a2, n2, m)).sum().backward()
    assert float(lnk2.grad.abs().max()) == 0.0


def test_backward_after_a_later_forward_resolves():
    m = _LinearModel()
    f1 = _fields(6)
    f2 = _fields(7)
    p1 = AG.observe(*f1, m)
    AG.observe(*f2, m)              # the handle now holds the second trajectory
    before = m.forwards
    w = torch.ones_like(p1)
    (p1 * w).sum().backward()
    assert m.forwards == before + 1  # the first forward was solved again
    for got, want in zip((t.grad for t in f1), _expected(m, w.numpy())):
        assert np.allclose(got.numpy(), want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_only_requested_gradients():
    m = _LinearModel()
    lnk, a, n = _fields(8)
    a.requires_grad_(False)
    AG.observe(lnk, a, n, m).sum().backward()
    assert lnk.grad is not None and n.grad is not None and a.grad is None
