"""The oracle (CPU restatement in oracle/pforacle.c) against golden fixtures
produced by the unmodified reference build (tests/golden/make_golden.py).

The restatement follows the reference's operation order, so the bar here is
bitwise equality for F(p), J x, M^-1 r and every timestep's pressure, and
identical KINSOL / GMRES iteration counts.
"""

import numpy as np
import pytest

from oracle.oracle import Oracle
from parflow_b200 import cases

CASES = cases.GOLDEN


@pytest.mark.parametrize("name", CASES)
def test_inputs_regenerate(name, golden):
    """Seeded inputs rebuild bit-identically on this machine."""
    g = golden(name)
    p = cases.get(name)
    assert np.array_equal(p.field3d(p.perm), g["perm"])
    assert np.array_equal(p.field3d(p.vg_alpha), g["alpha"])
    assert np.array_equal(p.initial_pressure(), g["press"][0])


@pytest.mark.parametrize("name", CASES)
def test_residual_bitexact(name, golden):
    g = golden(name)
    orc = Oracle(cases.get(name))
    for i in range(len(g["fe_p"])):
        orc.set_time(g["fe_time"][i])
        f = orc.residual(g["fe_p"][i], g["fe_pold"][i], g["fe_sold"][i], g["fe_dt"][i])
        assert np.array_equal(f, g["fe_f"][i]), (name, i, np.abs(f - g["fe_f"][i]).max())


@pytest.mark.parametrize("name", CASES)
def test_jacobian_and_pc_bitexact(name, golden):
    g = golden(name)
    orc = Oracle(cases.get(name))
    for i in range(len(g["mv_x"])):
        orc.set_time(g["mv_time"][i])
        # the old pressure (read only by the diffusive overland terms) was
        # dumped with the later fixtures
        p_old = g["mv_pold"][i] if "mv_pold" in g else None
        J = orc.jacobian(g["mv_p"][i], g["mv_dt"][i], 0, p_old)
        y = orc.matvec(J, g["mv_x"][i])
        assert np.array_equal(y, g["mv_y"][i]), (name, i)
        mg = orc.mg()
        if cases.get(name).solver.pc_matrix_code():
            mg.setup_full(J)
        else:
            mg.setup(orc.jacobian(g["mv_p"][i], g["mv_dt"][i], 2, p_old))
        z = mg.apply(g["pc_in"][i])
        assert np.array_equal(z, g["pc_out"][i]), (name, i)


@pytest.mark.parametrize("name", CASES)
def test_first_pc_bitexact(name, golden):
    """The first preconditioner application of a run is set up at the
    initial pressure of the first step (the first function evaluation's
    input), also where J v is a difference quotient and no J v dump exists;
    with UseJacobian False the reference builds that matrix without the
    overland surface terms."""
    g = golden(name)
    if not len(g["pc_in"]):
        pytest.skip("no preconditioner dump")
    prob = cases.get(name)
    orc = Oracle(prob)
    orc.set_time(g["fe_time"][0])
    fd = not prob.solver.use_jacobian
    mg = orc.mg()
    if prob.solver.pc_matrix_code():
        mg.setup_full(orc.jacobian(g["fe_p"][0], g["fe_dt"][0], 0, g["fe_pold"][0], fd=fd))
    else:
        mg.setup(orc.jacobian(g["fe_p"][0], g["fe_dt"][0], 2, g["fe_pold"][0], fd=fd))
    assert np.array_equal(mg.apply(g["pc_in"][0]), g["pc_out"][0]), name


def successful_attempts(times):
    """Indices of the solves that succeeded in a kinsol.log's sequence of
    target times: a failed solve is retried at an earlier time."""
    return [i for i in range(len(times)) if i == len(times) - 1 or times[i + 1] > times[i]]


@pytest.mark.parametrize("name", cases.TIME_LOOP)
def test_time_loop_bitexact(name, golden):
    """AdvanceRichards's step selection (growth from the running dt, cuts
    at cycle transitions, dump snapping, stop cut) and dt-halving retry:
    the oracle's loop takes the reference's steps, with its counts and
    pressures bit for bit."""
    g = golden(name)
    prob = cases.get(name)
    dump = prob.dt * cases.DUMP.get(name, 1) if cases.DUMP.get(name, 1) > 0 else 0.0
    ps, times, dts, sts = Oracle(prob).run_time_loop(dump_interval=dump)
    ok = successful_attempts(g["attempt_times"])
    assert np.allclose(times, g["attempt_times"][ok], rtol=0, atol=5e-7)
    assert [(s.nni, s.nli) for s in sts] == [tuple(r) for r in g["counts"][ok, :2]]
    if cases.DUMP.get(name, 1) < 0:  # every step written
        for n, p in enumerate(ps):
            assert np.array_equal(p, g["press"][n + 1]), (name, n)
    assert np.array_equal(ps[-1], g["press"][-1])


@pytest.mark.parametrize("name", [c for c in CASES if c not in cases.TIME_LOOP])
def test_timesteps_bitexact(name, golden):
    g = golden(name)
    prob = cases.get(name)
    orc = Oracle(prob)
    ps, sts = orc.run()
    for t, (p, st) in enumerate(zip(ps, sts)):
        assert np.array_equal(p, g["press"][t + 1]), (name, t, np.abs(p - g["press"][t + 1]).max())
        assert st.nni == g["counts"][t, 0] and st.nli == g["counts"][t, 1], (name, t)
        assert st.nfe == g["counts"][t, 2] and st.nps == g["counts"][t, 4], (name, t)
        assert st.status in (1, 2)


def test_hydrostatic_known_answer(golden):
    """Equilibrium: zero Newton iterations, pressure unchanged."""
    g = golden("hydrostatic")
    assert (g["counts"][:, 0] == 0).all()
    prob = cases.get("hydrostatic")
    ps, sts = Oracle(prob).run()
    for p, st in zip(ps, sts):
        assert st.nni == 0 and st.status == 2
        assert np.array_equal(p, prob.initial_pressure())


def test_mg_hierarchy_shape():
    """Coarsening order of mg_semi.c:858-923 for dx=dy=1, dz=0.5."""
    prob = cases.box_small()
    lv = Oracle(prob).mg().levels()
    assert lv[0] == (12, 10, 8, 2)
    assert lv[1] == (12, 10, 4, 0)
    assert lv[-1][:3] == (1, 1, 1) and lv[-1][3] == -1
    dirs = [d for *_, d in lv[:-1]]
    assert dirs[:4] == [2, 0, 1, 2]


VEL_CASES = [n for n in CASES if n.startswith("vel_")]


@pytest.mark.parametrize("name", VEL_CASES)
def test_face_velocities_bitexact(name, golden):
    """Face velocities (and overland fluxes) written by the residual at each
    step's solution equal the reference's velx / vely / velz (qx_overland,
    qy_overland) outputs bit for bit: interior faces, Dirichlet, flux and
    seepage faces, the overland top face, with an evap_trans sink/source."""
    g = golden(name)
    prob = cases.get(name)
    orc = Oracle(prob)
    plan = prob.time_plan()
    for n in range(1, prob.nsteps + 1):
        t, dt = plan[n - 1]
        orc.set_time(t)
        p_old, p = g["press"][n - 1], g["press"][n]
        _, vx, vy, vz, qx, qy = orc.residual_velocities(p, p_old, orc.saturation(p_old), dt)
        for key, mine in (("velx", vx), ("vely", vy), ("velz", vz),
                          ("qx_overland", qx), ("qy_overland", qy)):
            if key in g:
                ref = g[key][n - 1].reshape(mine.shape)
                assert np.array_equal(mine, ref), (name, n, key, np.abs(mine - ref).max())
