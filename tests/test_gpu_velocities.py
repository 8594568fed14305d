"""Face velocities and overland fluxes through the C ABI
(pfgpu_face_velocities) against the reference's own velx / vely / velz and
qx_overland / qy_overland outputs (golden fixtures), and after a device
solve against the oracle at the GPU's own solution.

Tolerance: max |v - v_ref| <= 1e-12 of the scale of the terms v is formed
from (same inputs; the kernels differ from the reference only by FMA
contraction, reciprocal products and the last bit of pow).  That scale is
max |v_ref|, except for the top-face z velocity of an overland patch: it
carries the ponding and routing term q_overlnd / dt (nl_function_eval.c:
1681-1687), a near-cancelling sum of the columns' surface fluxes
(ke - kw) / dx + (kn - ks) / dy, so its scale includes max |q| / dx.
"""

import numpy as np
import pytest

from parflow_b200 import cases

pytestmark = pytest.mark.gpu

VEL_CASES = [n for n in cases.GOLDEN if n.startswith("vel_")]
KEYS = ("velx", "vely", "velz", "qx_overland", "qy_overland")


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _close(mine, ref, what, extra_scale=0.0):
    scale = max(float(np.abs(ref).max()), extra_scale, 1e-300)
    err = float(np.abs(mine - ref).max()) / scale
    assert err <= 1e-12, (what, err)


def _qscale(prob, qx, qy):
    """max |q| / min(dx, dy): the size of the surface-flux terms of the
    overland top-face velocity."""
    return max(float(np.abs(qx).max()), float(np.abs(qy).max())) / min(prob.dx, prob.dy)


@pytest.mark.parametrize("name", VEL_CASES)
def test_velocities_vs_reference(name, golden, solver):
    g = golden(name)
    prob = cases.get(name)
    s = solver.RichardsGPU(prob)
    plan = prob.time_plan()
    for n in range(1, prob.nsteps + 1):
        t, dt = plan[n - 1]
        s.set_time(t)
        p_old, p = g["press"][n - 1], g["press"][n]
        out = s.face_velocities(dt, p=p, p_old=p_old, s_old=s.saturation(p_old))
        qs = _qscale(prob, g["qx_overland"][n - 1], g["qy_overland"][n - 1]) \
            if "qx_overland" in g else 0.0
        for key, mine in zip(KEYS, out):
            if key in g:
                _close(mine, g[key][n - 1].reshape(mine.shape), (name, n, key),
                       qs if key == "velz" else 0.0)
    s.close()


@pytest.mark.parametrize("name", VEL_CASES)
def test_velocities_after_device_step(name, solver):
    """After pfgpu_advance the call with no inputs uses the handle's solution
    and the step's old state; compared with the oracle evaluated at the
    same (GPU) solution."""
    from oracle.oracle import Oracle

    prob = cases.get(name)
    s = solver.RichardsGPU(prob)
    orc = Oracle(prob)
    p0 = prob.initial_pressure()
    t, dt = prob.time_plan()[0]
    s.set_pressure(p0)
    s.set_time(t)
    s.advance(1, dt)
    p1 = s.get_pressure()
    out = s.face_velocities(dt)
    orc.set_time(t)
    ref = orc.residual_velocities(p1, p0, orc.saturation(p0), dt)[1:]
    qs = _qscale(prob, ref[3], ref[4])
    for key, mine, r in zip(KEYS, out, ref):
        _close(mine, r, (name, key), qs if key == "velz" else 0.0)
    s.close()


def test_evap_trans_enters_residual(solver):
    """The sink/source changes F by -vol z_mult dt et, as the oracle's."""
    from oracle.oracle import Oracle

    prob = cases.get("vel_small")
    s = solver.RichardsGPU(prob)
    orc = Oracle(prob)
    t, dt = prob.time_plan()[0]
    s.set_time(t)
    orc.set_time(t)
    p_old = prob.initial_pressure()
    p = p_old + 0.01
    so = orc.saturation(p_old)
    f_gpu = s.nl_function_eval(p, p_old, so, dt)
    f_orc = orc.residual(p, p_old, so, dt)
    _close(f_gpu, f_orc, "F with evap_trans")
    s.set_evap_trans(None)
    f0 = s.nl_function_eval(p, p_old, so, dt)
    vol = prob.dx * prob.dy * prob.dz
    et = prob.field3d(prob.evap_trans)
    zm = prob.zmult()[:, None, None]
    np.testing.assert_allclose(f_gpu - f0, -vol * zm * dt * et, rtol=1e-9,
                               atol=1e-12 * float(np.abs(f0).max()))
    s.close()
