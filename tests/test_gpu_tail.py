"""The single-block V-cycle tail: shared-memory and global-memory variants
and the choice of the first tail level.

The tail runs the coarse levels of every V-cycle in one block.  By default it
starts at the largest level whose tail fits in shared memory and works there;
PFGPU_TAIL_SMEM=0 runs the same levels from global memory and
PFGPU_TAIL_CELLS moves the first tail level down, handing the levels above it
to the per-level grid kernels.  Every variant performs the same per-cell
arithmetic in the same order, so the preconditioner output must be bitwise
identical across them.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _problems():
    return {
        "box_small": cases.box_small(),
        "box_64": configs.box(nsteps=1),
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=1),
    }


def _pc(solver, prob, precision, monkeypatch, env):
    for k in ("PFGPU_TAIL_SMEM", "PFGPU_TAIL_CELLS"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    s = solver.RichardsGPU(prob, precision=precision)
    rng = np.random.default_rng(5)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    s.pc_setup(p, prob.dt)
    n0 = s.kernel_launches()
    z = s.pc_apply(r)
    launches = s.kernel_launches() - n0
    s.close()
    return z, launches


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed16"])
@pytest.mark.parametrize("name", ["box_small", "box_64", "hetero_96"])
def test_tail_variants_bitwise_equal(solver, monkeypatch, name, precision):
    prob = _problems()[name]
    z_smem, n_smem = _pc(solver, prob, precision, monkeypatch, {})
    z_glob, n_glob = _pc(solver, prob, precision, monkeypatch, {"PFGPU_TAIL_SMEM": "0"})
    z_grid, n_grid = _pc(solver, prob, precision, monkeypatch, {"PFGPU_TAIL_CELLS": "1"})
    assert np.isfinite(z_smem).all() and np.abs(z_smem).max() > 0
    assert np.array_equal(z_smem, z_glob)
    assert np.array_equal(z_smem, z_grid)
    assert n_smem == n_glob
    assert n_grid >= n_smem
