"""torch.autograd over the discrete adjoint (parflow_b200/autograd.py) on the
GPU, through the C ABI.

Small box with config-0 physics, per-cell ln K, alpha and n, four steps with
observations at steps 2 and 4.  The wrapper's gradient of the squared misfit
must equal the library's own adjoint gradient; the gradient of a
non-quadratic loss of the observed heads must match central finite
differences of the oracle's forward solve (ResidualTol 1e-13) to 1e-5
relative; a backward pass after a later forward must still give the first
forward's gradient.
"""

import numpy as np
import pytest

from parflow_b200 import configs
from parflow_b200.problem import BC, BC_FLUX, SolverSettings

pytestmark = pytest.mark.gpu

NSTEPS = 4
OBS_STEPS = [2, 4]
H = 1e-5
TOL = 1e-5


def _problem(lnk, alpha, vg_n):
    s = SolverSettings(residual_tol=1e-13, step_tol=1e-30)
    p = configs.box(nx=10, ny=8, nz=7, nsteps=NSTEPS, dt=0.25, seed=21, solver=s)
    p.bc["z_upper"] = BC(BC_FLUX, (-0.2,))
    p.perm = np.exp(lnk)
    p.vg_alpha = alpha
    p.vg_n = vg_n
    return p


def _prior():
    rng = np.random.default_rng(18)
    base = configs.box(nx=10, ny=8, nz=7, nsteps=NSTEPS, seed=21)
    lnk = np.log(base.perm)
    alpha = 2.0 * (1.0 + 0.3 * (rng.random(base.shape) - 0.5))
    vg_n = 3.0 * (1.0 + 0.1 * (rng.random(base.shape) - 0.5))
    return lnk, alpha, vg_n


def _cells(shape):
    nz, ny, nx = shape
    rng = np.random.default_rng(19)
    return rng.choice(np.arange((nz - 3) * nx * ny, nz * nx * ny), size=20, replace=False)


@pytest.fixture(scope="module")
def setup():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200.autograd import RichardsAdjointModel

    lnk, alpha, vg_n = _prior()
    prob = _problem(lnk, alpha, vg_n)
    cells = _cells(prob.shape)
    model = RichardsAdjointModel(prob, OBS_STEPS, cells, device=0, tol=1e-12)
    yield dict(model=model, fields=(lnk, alpha, vg_n), cells=cells, torch=torch)
    model.close()


def _tensors(torch, fields):
    return [torch.tensor(f, dtype=torch.float64, device="cuda", requires_grad=True)
            for f in fields]


def _oracle_obs(fields, cells):
    from oracle.oracle import Oracle

    ps, st = Oracle(_problem(*fields)).run(NSTEPS)
    assert all(s.status in (1, 2) for s in st)
    return np.stack([ps[s - 1].ravel()[cells] for s in OBS_STEPS])


def test_quadratic_misfit_matches_library_adjoint(setup):
    from parflow_b200.autograd import misfit
    from parflow_b200.solver import RichardsGPU

    torch, model = setup["torch"], setup["model"]
    rng = np.random.default_rng(20)
    obs = 0.1 * rng.standard_normal((len(OBS_STEPS), len(setup["cells"])))
    t = _tensors(torch, setup["fields"])
    j = misfit(*t, model, obs)
    j.backward()
    # the library's own adjoint on a fresh handle with the same fields
    prob = _problem(*setup["fields"])
    g = RichardsGPU(prob, precision="fp64")
    g.set_pressure(prob.initial_pressure())
    g.adjoint_record(NSTEPS)
    for tt, dt in prob.time_plan()[:NSTEPS]:
        g.set_time(tt)
        g.advance(1, dt)
    m_ref, *grads = g.adjoint_gradient(OBS_STEPS, setup["cells"], obs, tol=1e-12)
    g.close()
    assert abs(j.item() - m_ref) <= 1e-10 * abs(m_ref)
    for got, want in zip(t, grads):
        got = got.grad.cpu().numpy()
        assert np.linalg.norm(got - want) <= 1e-8 * np.linalg.norm(want)


def test_nonquadratic_loss_vs_oracle_fd(setup):
    from parflow_b200.autograd import observe

    torch, model, cells = setup["torch"], setup["model"], setup["cells"]
    rng = np.random.default_rng(21)
    c = rng.standard_normal((len(OBS_STEPS), len(cells)))
    ct = torch.tensor(c, device="cuda")
    t = _tensors(torch, setup["fields"])
    p = observe(*t, model)
    ref = _oracle_obs(setup["fields"], cells)
    assert np.abs(p.detach().cpu().numpy() - ref).max() <= 1e-9 * np.abs(ref).max()
    loss = (ct * torch.tanh(p)).sum() + 0.5 * (p * p).sum()
    loss.backward()
    grads = [x.grad.cpu().numpy() for x in t]

    def loss_np(fields):
        q = _oracle_obs(fields, cells)
        return float(np.sum(c * np.tanh(q)) + 0.5 * np.sum(q * q))

    d = [rng.standard_normal(f.shape) for f in setup["fields"]]
    ad = sum(float(np.sum(g * dd)) for g, dd in zip(grads, d))
    plus = [f + H * dd for f, dd in zip(setup["fields"], d)]
    minus = [f - H * dd for f, dd in zip(setup["fields"], d)]
    fd = (loss_np(plus) - loss_np(minus)) / (2 * H)
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


def test_backward_after_later_forward(setup):
    from parflow_b200.autograd import observe

    torch, model = setup["torch"], setup["model"]
    t1 = _tensors(torch, setup["fields"])
    p1 = observe(*t1, model)
    lnk, alpha, vg_n = setup["fields"]
    t2 = _tensors(torch, (lnk + 0.2, alpha, vg_n))
    observe(*t2, model)
    p1.sum().backward()
    t3 = _tensors(torch, setup["fields"])
    observe(*t3, model).sum().backward()
    for a, b in zip(t1, t3):
        assert torch.equal(a.grad, b.grad)
