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


def test_newton_solve_sat_equals_solve_then_saturation(solver):
    prob = _problem()
    p0 = prob.initial_pressure()
    a = solver.RichardsGPU(prob)
    s_old = a.saturation(p0)
    p_a, rc_a, _ = a.newton_solve(p0, p0, s_old, prob.dt)
    s_a = a.saturation(p_a)
    a.close()
    b = solver.RichardsGPU(prob)
    p_b, s_b, rc_b = b.newton_solve_sat(p0, p0, s_old, prob.dt)
    b.close()
    assert rc_a == rc_b == 0
    assert np.array_equal(p_a, p_b) and np.array_equal(s_a, s_b)


def test_newton_solve_sat_aliased_buffers(solver):
    """p passed in the p_old buffer and s in the s_old buffer (the caller's
    state at the start of a step): same result as separate buffers."""
    import ctypes as C

    from parflow_b200 import lib as L
    from parflow_b200.solver import pad, unpad

    prob = _problem()
    p0 = prob.initial_pressure()
    a = solver.RichardsGPU(prob)
    s0 = a.saturation(p0)
    p_ref, s_ref, _ = a.newton_solve_sat(p0, p0, s0, prob.dt)
    a.close()
    b = solver.RichardsGPU(prob)
    pb, sb = pad(p0), pad(s0)
    pp, sp = pb.ctypes.data_as(C.c_void_p), sb.ctypes.data_as(C.c_void_p)
    st = L.Stats()
    rc = b.lib.pfgpu_newton_solve_sat(b.h, pp, sp, prob.dt, pp, sp, C.byref(st))
    b.close()
    assert rc == 0
    assert np.array_equal(unpad(pb), p_ref) and np.array_equal(unpad(sb), s_ref)
