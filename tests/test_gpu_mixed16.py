"""The scaled FP16 multigrid operator (precision "mixed16",
PFGPU_PREC_MIXED_H16) on the configurations the benchmark runs.

The V-cycle works on S x, S^-1 b and S^-1 A S^-1 with S = sqrt(diag A); in
exact arithmetic it is the FP32/FP64 MGSemi V-cycle, so the Newton solution
must match the FP64 solver to the mixed-precision tolerance (1e-8 relative in
pressure) with the same Newton iteration counts, and the preconditioner
output must stay close to the FP32 one.
"""

import numpy as np
import pytest

from parflow_b200 import configs

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
        "box_64": configs.box(nsteps=3),
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=3),
        "overland_48": configs.overland(nx=48, ny=40, nz=10, nsteps=4, rain_steps=2,
                                        dry_steps=2),
    }


def _advance(solver, prob, precision):
    s = solver.RichardsGPU(prob, precision=precision)
    s.set_pressure(prob.initial_pressure())
    out, stats = [], []
    for t, dt in prob.time_plan()[:prob.nsteps]:
        s.set_time(t)
        stats += s.advance(1, dt)
        out.append(s.get_pressure())
    s.close()
    return out, stats


@pytest.mark.parametrize("name", ["box_64", "hetero_96", "overland_48"])
def test_mixed16_newton_matches_fp64(solver, name):
    prob = _problems()[name]
    p64, st64 = _advance(solver, prob, "fp64")
    p16, st16 = _advance(solver, prob, "mixed16")
    for t in range(prob.nsteps):
        err = np.abs(p16[t] - p64[t]).max() / np.abs(p64[t]).max()
        assert err <= 1e-8, (name, t, err)
        assert st16[t].kinsol_status in (1, 2)
        assert st16[t].nonlin_iters == st64[t].nonlin_iters, (name, t)


@pytest.mark.parametrize("name", ["box_64", "hetero_96"])
def test_mixed16_preconditioner_close_to_fp32(solver, name):
    prob = _problems()[name]
    rng = np.random.default_rng(11)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    z = {}
    for prec in ("mixed", "mixed16"):
        s = solver.RichardsGPU(prob, precision=prec)
        s.pc_setup(p, prob.dt)
        z[prec] = s.pc_apply(r)
        s.close()
    err = np.linalg.norm(z["mixed16"] - z["mixed"]) / np.linalg.norm(z["mixed"])
    assert err <= 5e-3, err


def test_unknown_precision_rejected(solver):
    with pytest.raises(ValueError):
        solver.RichardsGPU(configs.box(nx=8, ny=8, nz=4, nsteps=1), precision="half")
