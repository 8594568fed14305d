"""The native time loop (pfgpu_run) against the reference and the host loop.

pfgpu_run keeps every boundary time cycle on the device (pfgpu_set_bc_cycle),
selects dt as SelectTimeStep does (constant, or growth of the running dt
clamped to [min, max], cut to the next cycle transition), snaps dt to dump
times, cuts it to the stop time and halves it on a failed solve, as
AdvanceRichards does.  On the reference's time-loop fixtures (growth with
cycle transitions; a forced dt-halving retry with dump snapping) it must take
the reference's steps with its counts and end on its pressures; on the other
fixtures it must take the steps of the host loop (RichardsGPU.run, which
follows time_plan) and end on the same pressure bitwise.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs
from parflow_b200.problem import BC, BC_FLUX

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


@pytest.mark.parametrize("name", cases.TIME_LOOP)
def test_run_device_vs_reference_time_loop(solver, golden, name):
    g = golden(name)
    prob = cases.get(name)
    dump = prob.dt * cases.DUMP.get(name, 1) if cases.DUMP.get(name, 1) > 0 else 0.0
    s = solver.RichardsGPU(prob)
    p, times, dts, st = s.run_device(dump_interval=dump, growth=prob.growth)
    s.close()
    at = g["attempt_times"]
    ok = [i for i in range(len(at)) if i == len(at) - 1 or at[i + 1] > at[i]]
    assert np.allclose(times, at[ok], rtol=0, atol=5e-7), (times, at[ok])
    assert [(x.nonlin_iters, x.lin_iters) for x in st] == [tuple(r) for r in g["counts"][ok, :2]]
    ref = g["press"][-1]
    assert np.abs(p - ref).max() / np.abs(ref).max() <= 1e-9


@pytest.mark.parametrize("name", [c for c in cases.GOLDEN if c not in cases.TIME_LOOP])
def test_run_device_equals_host_loop(solver, name):
    prob = cases.get(name)
    s = solver.RichardsGPU(prob)
    ps, sts = s.run()
    plan = prob.time_plan()
    s.close()
    s = solver.RichardsGPU(prob)
    p, times, dts, st = s.run_device()
    s.close()
    assert times == [t for t, _ in plan] and dts == [dt for _, dt in plan]
    assert [x.nonlin_iters for x in st] == [x.nonlin_iters for x in sts]
    assert np.array_equal(p, ps[-1])


def test_growth_steps_and_cycle_transitions(solver):
    """Growth steps cut at cycle transitions on a larger box: pfgpu_run
    against the host stepping the same steps one by one (the step rule is
    pinned to the reference by the time-loop fixtures above)."""
    prob = configs.box(nx=24, ny=20, nz=10, nsteps=6, dt=0.1, seed=7)
    prob.bc["z_upper"] = BC(BC_FLUX, (-0.05, 0.0), lengths=(2, 3), repeat=-1)
    prob.growth = (0.04, 1.7, 0.01, 0.15)
    s = solver.RichardsGPU(prob)
    p_dev, times, dts, _ = s.run_device(dump_interval=0.0, growth=prob.growth)
    s.close()
    # host restatement of SelectTimeStep growth on the running dt
    # (select_time_step.c:97-115; the initial step before the loop), the
    # transition cut and the stop cut
    init, factor, lo, hi = prob.growth
    stop = prob.stop_time()
    s = solver.RichardsGPU(prob)
    s.set_pressure(prob.initial_pressure())
    t, dt, want_t, want_dt = prob.start_time, init, [], []
    while t < stop:
        dt = min(max(dt * factor, lo), hi)
        bc_dt = prob.next_transition(t)
        if bc_dt > 0 and dt > bc_dt:
            dt = bc_dt
        if t + dt >= stop:
            dt = stop - t
        t += dt
        s.set_time(t)
        s.advance(1, dt)
        want_t.append(t)
        want_dt.append(dt)
    p_host = s.get_pressure()
    s.close()
    assert times == want_t and dts == want_dt
    assert any(d < hi for d in dts[1:-1])  # some step was cut to a transition
    assert np.array_equal(p_dev, p_host)


def test_run_reports_failure(solver):
    from parflow_b200 import lib as L
    from parflow_b200.problem import SolverSettings

    prob = configs.box(nx=16, ny=12, nz=8, nsteps=2, dt=0.5, seed=1,
                       solver=SolverSettings(max_iter=1, residual_tol=1e-14))
    s = solver.RichardsGPU(prob)
    with pytest.raises(L.PfgpuError):
        s.run_device()
    s.close()
