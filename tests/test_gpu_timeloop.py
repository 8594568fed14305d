"""The native time loop (pfgpu_run) against the per-step host loop.

pfgpu_run keeps every boundary time cycle on the device (pfgpu_set_bc_cycle),
selects dt as SelectTimeStep does (constant, or growth clamped to [min, max],
cut to the next cycle transition), snaps dt to dump times and cuts it to the
stop time, as AdvanceRichards does.  On the reference's fixtures it must take
the steps of the host loop (RichardsGPU.run, which follows time_plan) and end
on the same pressure bitwise; with growth steps it must follow a host
restatement of the same rules.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs
from parflow_b200.problem import BC, BC_FLUX, pfround

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


@pytest.mark.parametrize("name", cases.GOLDEN)
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


def _next_transition(bc, t, base, start):
    """TimeCycleDataComputeNextTransition (time_cycle_data.c:206-297) for one
    face cycle repeating for ever."""
    lengths = list(bc.lengths)
    if len(lengths) <= 1:
        return -1.0
    clen = sum(lengths)
    sub = 1000
    dtime = pfround(t / (base / sub)) // sub
    dstart = pfround(start / (base / sub)) // sub
    n = (dtime - dstart) // clen
    done = int(np.fmod(dtime - dstart - 1, clen))
    q, total = 0, lengths[0]
    while done >= total:
        q += 1
        total += lengths[q]
    if (q + 1) % len(lengths) == 0:
        tt = start + (n + 1) * clen * base
    else:
        tt = start + (n * clen + total) * base
    return tt - t


def test_growth_steps_and_cycle_transitions(solver):
    prob = configs.box(nx=24, ny=20, nz=10, nsteps=6, dt=0.1, seed=7)
    prob.bc["z_upper"] = BC(BC_FLUX, (-0.05, 0.0), lengths=(2, 3), repeat=-1)
    growth = (0.04, 1.7, 0.01, 0.15)
    s = solver.RichardsGPU(prob)
    p_dev, times, dts, _ = s.run_device(dump_interval=0.0, growth=growth)
    s.close()
    # host restatement: SelectTimeStep growth, transition cut, stop cut
    init, factor, lo, hi = growth
    base, start, stop = prob.dt, prob.start_time, prob.stop_time()
    s = solver.RichardsGPU(prob)
    s.set_pressure(prob.initial_pressure())
    t, last, want_t, want_dt = start, 0.0, [], []
    while t < stop:
        dt = init if last == 0.0 else min(max(last * factor, lo), hi)
        bc_dt = _next_transition(prob.bc["z_upper"], t, base, start)
        if bc_dt > 0 and dt > bc_dt:
            dt = bc_dt
        if t + dt >= stop:
            dt = stop - t
        t += dt
        s.set_time(t)
        s.advance(1, dt)
        last = dt
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
