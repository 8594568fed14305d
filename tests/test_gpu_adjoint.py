"""Discrete adjoint (pfgpu_adjoint_record / pfgpu_adjoint_gradient) against
central finite differences of the oracle's forward model.

Box with config-0 physics, per-cell ln K, van Genuchten alpha and n, a
Dirichlet bottom (so the boundary-face gradient terms are exercised) and
observations at two of four steps.  Forward solves for the differences use
ResidualTol 1e-13 (the FD noise is tol / h); the gradient must agree to
1e-5 relative for single cells of each parameter field and for random
directions.
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
    rng = np.random.default_rng(8)
    base = configs.box(nx=10, ny=8, nz=7, nsteps=NSTEPS, seed=21)
    lnk = np.log(base.perm)
    alpha = 2.0 * (1.0 + 0.3 * (rng.random(base.shape) - 0.5))
    vg_n = 3.0 * (1.0 + 0.1 * (rng.random(base.shape) - 0.5))
    return lnk, alpha, vg_n


def _obs(shape):
    rng = np.random.default_rng(9)
    nz, ny, nx = shape
    # observation wells in the upper three layers, where the wetting front passes
    upper = np.arange((nz - 3) * nx * ny, nz * nx * ny)
    cells = rng.choice(upper, size=24, replace=False)
    lnk, alpha, vg_n = _prior()
    truth = _problem(lnk + 0.4 * rng.standard_normal(shape), alpha, vg_n)
    from oracle.oracle import Oracle

    ps, _ = Oracle(truth).run(NSTEPS)
    vals = np.stack([ps[s - 1].ravel()[cells] for s in OBS_STEPS])
    return cells, vals + 1e-3 * rng.standard_normal(vals.shape)


def _misfit_oracle(prob, cells, vals):
    from oracle.oracle import Oracle

    ps, st = Oracle(prob).run(NSTEPS)
    assert all(s.status in (1, 2) for s in st)
    return sum(float(np.sum((ps[s - 1].ravel()[cells] - vals[k]) ** 2))
               for k, s in enumerate(OBS_STEPS))


@pytest.fixture(scope="module")
def adjoint():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200.solver import RichardsGPU

    lnk, alpha, vg_n = _prior()
    prob = _problem(lnk, alpha, vg_n)
    cells, vals = _obs(prob.shape)
    g = RichardsGPU(prob, precision="fp64")
    g.set_pressure(prob.initial_pressure())
    g.adjoint_record(NSTEPS)
    for t, dt in prob.time_plan()[:NSTEPS]:
        g.set_time(t)
        g.advance(1, dt)
    misfit, g_lnk, g_a, g_n = g.adjoint_gradient(OBS_STEPS, cells, vals, tol=1e-12)
    g.close()
    return dict(prob=prob, cells=cells, vals=vals, misfit=misfit,
                grads={"lnk": g_lnk, "alpha": g_a, "n": g_n}, fields=(lnk, alpha, vg_n))


def _perturbed(fields, which, delta):
    lnk, alpha, vg_n = (f.copy() for f in fields)
    {"lnk": lnk, "alpha": alpha, "n": vg_n}[which][...] += delta
    return _problem(lnk, alpha, vg_n)


def test_misfit_matches_oracle_forward(adjoint):
    m = _misfit_oracle(adjoint["prob"], adjoint["cells"], adjoint["vals"])
    assert abs(adjoint["misfit"] - m) <= 1e-9 * max(1.0, abs(m))


@pytest.mark.parametrize("which", ["lnk", "alpha", "n"])
def test_gradient_single_cells_vs_fd(adjoint, which):
    grad = adjoint["grads"][which]
    shape = grad.shape
    order = np.argsort(-np.abs(grad).ravel())
    rng = np.random.default_rng(3)
    picks = list(order[:2]) + list(rng.choice(order[:max(8, len(order) // 10)], 2, replace=False))
    for c in picks:
        e = np.zeros(shape)
        e.ravel()[c] = H
        jp = _misfit_oracle(_perturbed(adjoint["fields"], which, e), adjoint["cells"], adjoint["vals"])
        jm = _misfit_oracle(_perturbed(adjoint["fields"], which, -e), adjoint["cells"], adjoint["vals"])
        fd = (jp - jm) / (2 * H)
        ad = grad.ravel()[c]
        assert abs(ad - fd) <= TOL * abs(fd), (which, int(c), ad, fd)


def test_gradient_random_directions_vs_fd(adjoint):
    rng = np.random.default_rng(4)
    g = adjoint["grads"]
    for _ in range(2):
        d = {k: rng.standard_normal(v.shape) for k, v in g.items()}
        ad = sum(float(np.sum(g[k] * d[k])) for k in g)
        lnk, alpha, vg_n = adjoint["fields"]
        plus = _problem(lnk + H * d["lnk"], alpha + H * d["alpha"], vg_n + H * d["n"])
        minus = _problem(lnk - H * d["lnk"], alpha - H * d["alpha"], vg_n - H * d["n"])
        fd = (_misfit_oracle(plus, adjoint["cells"], adjoint["vals"]) -
              _misfit_oracle(minus, adjoint["cells"], adjoint["vals"])) / (2 * H)
        assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)
