"""The kernels that run the middle multigrid levels as one team.

PFGPU_MID_CELLS hands the grid levels at or below that many cells (above the
single-block tail) to one cluster kernel, which walks their phases with
cluster barriers between them and runs the tail in its first block;
PFGPU_GRID_CELLS hands them to two cooperative kernels over the whole GPU
(down leg, up leg) with grid barriers between the phases, the tail running in
its own kernel in between.  Every per-cell operation is the one the per-level
grid kernels perform, in the same order, so the preconditioner output must be
bitwise identical to the default configuration, with fewer launches, for both
smoothers, every precision, the shared-memory and global-memory tails and any
cluster size.
"""

import numpy as np
import pytest

from parflow_b200 import configs
from parflow_b200.problem import SolverSettings

pytestmark = pytest.mark.gpu

ENV = ("PFGPU_MID_CELLS", "PFGPU_MID_CLUSTER", "PFGPU_TAIL_SMEM", "PFGPU_TAIL_CELLS",
       "PFGPU_GRID_CELLS", "PFGPU_GRID_PER_SM")


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _problems(smoother="RedBlackGSPoint"):
    s = SolverSettings(mg_smoother=smoother)
    return {
        "box_64": configs.box(nsteps=1, solver=s),
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=1, solver=s),
        "hetero_odd": configs.hetero(nx=123, ny=77, nz=19, nsteps=1, solver=s),
    }


def _pc(solver, prob, precision, monkeypatch, env):
    for k in ENV:
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    s = solver.RichardsGPU(prob, precision=precision)
    rng = np.random.default_rng(5)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    s.pc_setup(p, prob.dt)
    n0 = s.kernel_launches()
    z1 = s.pc_apply(r)
    z2 = s.pc_apply(z1)
    launches = s.kernel_launches() - n0
    s.close()
    return np.concatenate([z1.ravel(), z2.ravel()]), launches


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed16"])
@pytest.mark.parametrize("name", ["box_64", "hetero_96", "hetero_odd"])
def test_mid_levels_bitwise_equal(solver, monkeypatch, name, precision):
    prob = _problems()[name]
    z_ref, n_ref = _pc(solver, prob, precision, monkeypatch, {})
    assert np.isfinite(z_ref).all() and np.abs(z_ref).max() > 0
    for env in ({"PFGPU_MID_CELLS": "20000"},
                {"PFGPU_MID_CELLS": "1000000000"},
                {"PFGPU_MID_CELLS": "1000000000", "PFGPU_TAIL_SMEM": "0"},
                {"PFGPU_MID_CELLS": "1000000000", "PFGPU_MID_CLUSTER": "2"},
                {"PFGPU_MID_CELLS": "1000000000", "PFGPU_TAIL_CELLS": "1"},
                {"PFGPU_GRID_CELLS": "20000"},
                {"PFGPU_GRID_CELLS": "1000000000"},
                {"PFGPU_GRID_CELLS": "1000000000", "PFGPU_GRID_PER_SM": "2"},
                {"PFGPU_GRID_CELLS": "1000000000", "PFGPU_TAIL_SMEM": "0"}):
        z, n = _pc(solver, prob, precision, monkeypatch, env)
        assert np.array_equal(z, z_ref), env
        assert n < n_ref, ("the team kernel did not run", env)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mid_levels_weighted_jacobi(solver, monkeypatch, precision):
    prob = _problems("WJacobi")["hetero_96"]
    z_ref, n_ref = _pc(solver, prob, precision, monkeypatch, {})
    assert np.isfinite(z_ref).all()
    for env in ({"PFGPU_MID_CELLS": "1000000000"}, {"PFGPU_GRID_CELLS": "1000000000"}):
        z, n = _pc(solver, prob, precision, monkeypatch, env)
        assert np.array_equal(z, z_ref), env
        assert n < n_ref, env


def test_mid_levels_newton_solve_identical(solver, monkeypatch):
    """Two timesteps of the headline form: identical pressures and iteration
    counts with and without the cluster kernel."""
    prob = configs.hetero(nx=96, ny=80, nz=20, nsteps=2)
    out = []
    for env in ({}, {"PFGPU_MID_CELLS": "100000"}, {"PFGPU_GRID_CELLS": "100000"}):
        for k in ENV:
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        s = solver.RichardsGPU(prob, precision="mixed16")
        s.set_pressure(prob.initial_pressure())
        st = s.advance(2, prob.dt)
        out.append((s.get_pressure(), [(x.nonlin_iters, x.lin_iters) for x in st]))
        s.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0])
        assert out[0][1] == o[1]
