"""Cell fields re-uploaded on a live handle (parameter studies, finite
differences): the solution must equal that of a fresh handle built from the
same problem, whatever was uploaded before.  A per-cell van Genuchten array
left by an earlier upload must not survive a later uniform field, and a
uniform field that differs from the descriptor scalar must reach the device.
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


def _problem():
    p = configs.box(nx=16, ny=12, nz=8, nsteps=2, dt=0.1, seed=3)
    p.vg_alpha = np.full(p.shape, 2.0)
    p.vg_n = np.full(p.shape, 3.0)
    return p


def _run(s, prob):
    s.update_fields()
    s.set_pressure(prob.initial_pressure())
    for t, dt in prob.time_plan()[:prob.nsteps]:
        s.set_time(t)
        s.advance(1, dt)
    return s.get_pressure()


def _fresh(solver, prob):
    s = solver.RichardsGPU(prob)
    p = _run(s, prob)
    s.close()
    return p


def test_uniform_field_after_per_cell_field(solver):
    prob = _problem()
    ref = _fresh(solver, prob)
    s = solver.RichardsGPU(prob)
    pert = prob.vg_alpha.copy()
    pert[prob.nz // 2:] *= 1.5  # the unsaturated upper half
    prob.vg_alpha = pert
    p_pert = _run(s, prob)
    assert not np.array_equal(p_pert, ref)
    prob.vg_alpha = np.full(prob.shape, 2.0)
    assert np.array_equal(_run(s, prob), ref)
    s.close()


def test_uniform_field_different_from_descriptor(solver):
    prob = _problem()
    s = solver.RichardsGPU(prob)
    prob.vg_n = np.full(prob.shape, 2.5)
    p = _run(s, prob)
    s.close()
    ref = _fresh(solver, prob)
    # per-cell array on one handle, descriptor scalar on the other: the same
    # values through the same arithmetic
    np.testing.assert_allclose(p, ref, rtol=1e-13, atol=0)
