"""The Newton solve as one CUDA graph (device-side control, the default)
against the host-driven solve.

In graph mode every KINSOL and SPGMR decision (GMRES stop test and restarts,
line-search backtracking and refinement, the forcing term, KINStop) is taken
by control kernels on the device that steer the graph's conditional nodes;
the host reads the counters once per solve.  The control kernels restate the
host's arithmetic without contracted multiply-adds, so the two forms must
take the same steps bit for bit: identical pressures after every step and
identical counters, on every golden case (analytic and difference-quotient
J v, GMRES restarts, overland and seepage faces, the relative-permeability
tables, the PFMG-keyed and WJacobi smoothers), in FP64 and in the mixed16
form, through the per-step entry point and through the native time loop
(growth, forced dt halving).
"""

import numpy as np
import pytest

from parflow_b200 import cases

pytestmark = pytest.mark.gpu

STEP_CASES = [c for c in cases.GOLDEN if c not in cases.TIME_LOOP]
FIELDS = ("kinsol_status", "nonlin_iters", "lin_iters", "fevals", "pc_setups", "pc_solves",
          "lin_conv_fails", "beta_cond_fails", "backtracks", "fnorm")


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver

    return solver


def _check_graph(s, mode):
    used = s.solve_graph(-1)
    if mode == 1 and used != 1:
        from parflow_b200 import lib

        pytest.fail("the solve did not run as a graph: " + lib.last_error())
    assert used == mode


def _run(gpu, prob, precision, mode):
    s = gpu.RichardsGPU(prob, precision=precision)
    s.solve_graph(mode)
    ps, sts = s.run()
    _check_graph(s, mode)
    s.close()
    return ps, sts


def _same_stats(a, b, where):
    for f in FIELDS:
        assert getattr(a, f) == getattr(b, f), (where, f, getattr(a, f), getattr(b, f))


# FP64 and the headline mixed form; FullJacobian runs on the FP64 and FP32
# multigrids only, so its reduced-precision pass is the FP32 one
PAIRS = [(c, p) for c in STEP_CASES
         for p in ("fp64", "mixed" if cases.get(c).solver.pc_matrix_code() else "mixed16")]


@pytest.mark.parametrize("name,precision", PAIRS)
def test_graph_solve_equals_host_driven(gpu, name, precision):
    prob = cases.get(name)
    pg, sg = _run(gpu, prob, precision, 1)
    ph, sh = _run(gpu, prob, precision, 0)
    assert len(pg) == len(ph)
    for t, (a, b) in enumerate(zip(pg, ph)):
        assert np.array_equal(a, b), (name, t, np.abs(a - b).max())
    for t, (a, b) in enumerate(zip(sg, sh)):
        _same_stats(a, b, (name, t))


@pytest.mark.parametrize("name", cases.TIME_LOOP)
def test_graph_time_loop_equals_host_driven(gpu, name):
    """pfgpu_run with growth, cycle transitions, failed attempts and dt
    halving: the graph solve reports the same failures, so the loop takes the
    same attempts."""
    prob = cases.get(name)
    dump = prob.dt * cases.DUMP.get(name, 1) if cases.DUMP.get(name, 1) > 0 else 0.0
    out = []
    for mode in (1, 0):
        s = gpu.RichardsGPU(prob)
        s.solve_graph(mode)
        out.append(s.run_device(dump_interval=dump, growth=prob.growth))
        _check_graph(s, mode)
        s.close()
    (pa, ta, da, sa), (pb, tb, db, sb) = out
    assert ta == tb and da == db
    assert np.array_equal(pa, pb)
    for t, (a, b) in enumerate(zip(sa, sb)):
        _same_stats(a, b, (name, t))


def test_graph_recaptured_when_the_problem_changes(gpu):
    """A Jacobian-mode change after the first solves gives a new graph: the
    results equal a host-driven solve of the changed problem."""
    prob = cases.get("box_small")
    res = []
    for mode in (1, 0):
        s = gpu.RichardsGPU(prob)
        s.solve_graph(mode)
        ps1, _ = s.run()
        assert s.lib.pfgpu_set_jacobian_mode(s.h, 0, 1e-7) == 0
        ps2, st2 = s.run()
        _check_graph(s, mode)
        res.append((ps1, ps2, st2))
        s.close()
    for a, b in zip(res[0][1], res[1][1]):
        assert np.array_equal(a, b)
    for a, b in zip(res[0][2], res[1][2]):
        _same_stats(a, b, "dq")


def test_graph_solve_large_krylov_dimension(gpu):
    """Krylov dimension 50 (the reference's tilted-V tests) with a one-level
    multigrid, so that GMRES cycles run past 30 iterations (27 on average in
    the second step): the graph's nested GMRES iteration bodies are 50 deep.
    Graph and host-driven solves bitwise equal, counts equal the oracle's."""
    from oracle.oracle import Oracle
    from parflow_b200 import configs
    from parflow_b200.problem import SolverSettings

    prob = configs.hetero(nx=16, ny=14, nz=10, nsteps=2, dt=5.0, seed=29,
                          solver=SolverSettings(krylov_dim=50, eta_value=1e-10,
                                                mg_max_levels=1))
    pg, sg = _run(gpu, prob, "fp64", 1)
    ph, sh = _run(gpu, prob, "fp64", 0)
    _, so = Oracle(prob).run()
    for t, (a, b) in enumerate(zip(pg, ph)):
        assert np.array_equal(a, b), (t, np.abs(a - b).max())
    for t, (a, b) in enumerate(zip(sg, sh)):
        _same_stats(a, b, ("krylov50", t))
    assert [(x.nonlin_iters, x.lin_iters) for x in sg] == [(x.nni, x.nli) for x in so]
