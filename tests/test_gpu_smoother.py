"""The TMA-pipelined fused red/black/red smoother (k_rbr_tma) against the
per-colour sweep kernels and the reference.

PFGPU_RBR_FUSED_CELLS selects, at handle creation, the grid levels the fused
kernel smooths: 0 = every level whose row pitch TMA can address, a huge
value = none (the default); it reads the natural (PFGPU_SPLIT=0) layout.  PFGPU_TAIL_CELLS = 16 keeps all but the last few levels on grid
kernels, so that the small fixtures exercise the fused kernel too.  Both
smoothers perform the same per-cell arithmetic, so the V-cycle output must be
bitwise identical; against the reference's preconditioner output the usual
1e-12 normwise bound applies.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs

pytestmark = pytest.mark.gpu

ALL, NONE = "0", str(1 << 62)


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _problems():
    return {
        "box_small": cases.box_small(),             # 12 x 10 x 8
        "box_64": configs.box(nsteps=1),             # 64 x 64 x 32
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=1),
    }


def _pc(solver, prob, precision, monkeypatch, cells):
    monkeypatch.setenv("PFGPU_RBR_FUSED_CELLS", cells)
    monkeypatch.setenv("PFGPU_TAIL_CELLS", "16")
    monkeypatch.setenv("PFGPU_SPLIT", "0")  # the fused kernel reads the natural layout
    s = solver.RichardsGPU(prob, precision=precision)
    rng = np.random.default_rng(3)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    s.pc_setup(p, prob.dt)
    n0 = s.kernel_launches()
    z = s.pc_apply(r)
    launches = s.kernel_launches() - n0
    z2 = s.pc_apply(r)
    s.close()
    assert np.array_equal(z, z2)
    return z, launches


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["box_small", "box_64", "hetero_96"])
def test_fused_smoother_bitwise_equals_colour_sweeps(solver, monkeypatch, name, precision):
    prob = _problems()[name]
    z_fused, n_fused = _pc(solver, prob, precision, monkeypatch, ALL)
    z_ref, n_ref = _pc(solver, prob, precision, monkeypatch, NONE)
    assert n_fused < n_ref, "the fused smoother did not run"
    assert np.all(np.isfinite(z_fused))
    assert np.array_equal(z_fused, z_ref)


@pytest.mark.parametrize("name", cases.GOLDEN)
def test_fused_preconditioner_vs_reference(solver, monkeypatch, golden, name):
    monkeypatch.setenv("PFGPU_RBR_FUSED_CELLS", ALL)
    monkeypatch.setenv("PFGPU_TAIL_CELLS", "16")
    monkeypatch.setenv("PFGPU_SPLIT", "0")  # the fused kernel reads the natural layout
    g = golden(name)
    s = solver.RichardsGPU(cases.get(name))
    for i in range(min(len(g["pc_in"]), len(g["mv_p"]))):
        s.set_time(g["mv_time"][i])
        s.pc_setup(g["mv_p"][i], g["mv_dt"][i], g["mv_pold"][i] if "mv_pold" in g else None)
        z = s.pc_apply(g["pc_in"][i])
        err = np.linalg.norm(z - g["pc_out"][i]) / np.linalg.norm(g["pc_out"][i])
        assert err <= 1e-12, (name, i, err)
    s.close()


def test_fused_timesteps_vs_oracle(solver, monkeypatch):
    """64 x 64 x 32, two steps, every eligible level on the fused smoother."""
    from oracle.oracle import Oracle

    monkeypatch.setenv("PFGPU_RBR_FUSED_CELLS", ALL)
    monkeypatch.setenv("PFGPU_SPLIT", "0")
    prob = configs.box(nsteps=2)
    ps_o, st_o = Oracle(prob).run()
    s = solver.RichardsGPU(prob)
    ps_g, st_g = s.run()
    s.close()
    for t in range(2):
        err = np.abs(ps_g[t] - ps_o[t]).max() / np.abs(ps_o[t]).max()
        assert err <= 1e-9, (t, err)
        assert st_g[t].nonlin_iters == st_o[t].nni and st_g[t].lin_iters == st_o[t].nli
