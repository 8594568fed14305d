"""Named small problems used as parity cases (and their golden fixtures).

Each is a scaled-down, seeded instance of a benchmark workload so that the
reference CPU build and the oracle finish in seconds.
"""

from __future__ import annotations

import numpy as np

from . import configs
from .problem import (BC, BC_DIRICHLET, BC_FLUX, BC_OVERLAND, BC_OVERLAND_DIFF, BC_SEEPAGE,
                      RichardsProblem,
                      SolverSettings)


def box_small() -> RichardsProblem:
    """Config-0 physics on 12x10x8, 2 steps."""
    return configs.box(nx=12, ny=10, nz=8, nsteps=2)


def box_odd() -> RichardsProblem:
    """Odd sizes (ragged multigrid levels), 3 steps, another seed."""
    return configs.box(nx=17, ny=9, nz=11, nsteps=3, seed=7)


def hetero_small() -> RichardsProblem:
    """Config-2 physics (per-cell van Genuchten files) on 16x16x10, 2 steps."""
    return configs.hetero(nx=16, ny=16, nz=10, nsteps=2)


def walker2_small() -> RichardsProblem:
    """Default Walker2 forcing term and side Dirichlet faces."""
    p = configs.box(nx=14, ny=12, nz=9, nsteps=2, seed=11,
                    solver=SolverSettings(eta_choice="Walker2"))
    p.bc["x_lower"] = BC(BC_DIRICHLET, (1.5,), ref_patch="z_lower")
    p.bc["y_upper"] = BC(BC_DIRICHLET, (2.5,), ref_patch="z_lower")
    return p


def hydrostatic() -> RichardsProblem:
    """Known answer: a box in hydrostatic equilibrium with no-flow faces and a
    Dirichlet bottom needs zero Newton iterations and keeps its pressure."""
    p = configs.box(nx=10, ny=8, nz=12, nsteps=2, seed=3)
    p.bc["z_upper"] = BC(BC_FLUX, (0.0,))
    return p


def overland_small() -> RichardsProblem:
    """Config-1 physics on 12x10x6 with the surface ponded from the start, so
    that kinematic overland flow and its boundary outflow are active; rain for
    2 steps, then none."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=4, seed=13, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=2)


def overland_diff_small() -> RichardsProblem:
    """The overland case with diffusive-wave routing (OverlandDiffusive): the
    friction slope includes the ponded-depth gradient and its magnitude comes
    from the old pressure."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=4, seed=13, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=2,
                            kind=BC_OVERLAND_DIFF)


def overland_flow_small() -> RichardsProblem:
    """The overland case with the OverlandFlow patch type (overlandflow_eval.c:
    each column's flux along its own slope, upwinded between columns)."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=4, seed=13, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=2, kind=BC_OVERLAND)


def seepage_small() -> RichardsProblem:
    """Config-0 box with SeepageFace patches: the top face (water table 0.3 m
    above it, so the top layer is ponded and drains) and the x_upper face."""
    p = configs.box(nx=12, ny=10, nz=8, nsteps=3, seed=19)
    p.bc["z_upper"] = BC(BC_SEEPAGE, (-0.05,))
    p.bc["x_upper"] = BC(BC_SEEPAGE, (0.0,))
    p.ic = p.hydrostatic_ic(4.3, "z_lower")
    return p


def dq_small() -> RichardsProblem:
    """The reference's default Solver.Nonlinear.UseJacobian False: GMRES on
    KINSOL's difference-quotient J v (the preconditioner keeps the analytic
    symmetric part), config-0 physics with per-cell van Genuchten files."""
    p = configs.hetero(nx=14, ny=12, nz=9, nsteps=2, seed=23,
                       solver=SolverSettings(use_jacobian=False))
    return p


def krtable_spline_small() -> RichardsProblem:
    """Config-0 box whose relative permeability comes from the reference's
    lookup table, monotone spline (crater2D_vangtable_spline's keys)."""
    p = configs.box(nx=12, ny=10, nz=8, nsteps=2, seed=29)
    p.kr_table = ("Spline", 20000, -300.0)
    return p


def krtable_linear_small() -> RichardsProblem:
    """The same with linear interpolation in the table."""
    p = configs.box(nx=12, ny=10, nz=8, nsteps=2, seed=29)
    p.kr_table = ("Linear", 20000, -300.0)
    return p


def default_richards() -> RichardsProblem:
    """The reference's own regression case default_richards
    (test/python/default_richards.py): 18x15x8 box at origin (-10, 10, 1),
    K = 4, porosity 1, VG alpha 0.005, n 2, Sres 0.2, Ssat 0.99, hydrostatic
    start (3.0 at the bottom), DirEquilRefPatch 5.0 / 3.0 on the x faces,
    no-flow elsewhere, 50 steps of 0.001.  Its reference outputs were made
    with PFMG; MGSemi stands in here, so the comparison is at the test's own
    6 significant digits."""
    s = SolverSettings(residual_tol=1e-9, max_iter=10, krylov_dim=10, eta_value=1e-5)
    p = RichardsProblem(nx=18, ny=15, nz=8, dx=8.8888888888888893, dy=10.666666666666666,
                        dz=1.0, perm=4.0, porosity=1.0, specific_storage=1.0e-4,
                        vg_alpha=0.005, vg_n=2.0, s_res=0.2, s_sat=0.99, dt=0.001, nsteps=50,
                        solver=s, name="default_richards")
    p.x0, p.y0, p.z0 = -10.0, 10.0, 1.0
    p.bc = {
        "x_lower": BC(BC_DIRICHLET, (5.0,), ref_patch="z_lower"),
        "x_upper": BC(BC_DIRICHLET, (3.0,), ref_patch="z_lower"),
        "y_lower": BC(BC_FLUX, (0.0,)),
        "y_upper": BC(BC_FLUX, (0.0,)),
        "z_lower": BC(BC_FLUX, (0.0,)),
        "z_upper": BC(BC_FLUX, (0.0,)),
    }
    p.ic = p.hydrostatic_ic(3.0, "z_lower")
    return p


def tfg_small() -> RichardsProblem:
    """Terrain-following slopes in the subsurface fluxes without overland
    flow: config-1 layers and slopes, no-flow top, Dirichlet bottom."""
    p = configs.overland(nx=13, ny=11, nz=7, nsteps=2, seed=17, wt_depth=0.5)
    p.bc["z_upper"] = BC(BC_FLUX, (-0.01,))
    p.bc["z_lower"] = BC(BC_DIRICHLET, (0.3,), ref_patch="z_lower")
    return p


def wjacobi_small() -> RichardsProblem:
    """The multigrid with the weighted Jacobi smoother (MGSemi.Smoother
    WJacobi, Smoother.Weight 0.8) on config-2 physics (per-cell van
    Genuchten files)."""
    return configs.hetero(nx=15, ny=13, nz=9, nsteps=2, seed=31,
                          solver=SolverSettings(mg_smoother="WJacobi", wjacobi_weight=0.8))


def rbgs_nonsym_small() -> RichardsProblem:
    """Red/black Gauss-Seidel with Smoother.Symmetric False (red, black per
    smoothing) on config-0 physics."""
    return configs.box(nx=13, ny=11, nz=9, nsteps=2, seed=37,
                       solver=SolverSettings(mg_smoother_symmetric=False))


def vel_small() -> RichardsProblem:
    """Face velocities written by the residual (Solver.PrintVelocities) on
    config-2 physics with a Dirichlet x_lower face, a SeepageFace x_upper
    face, a flux top and a seeded land-surface sink/source (evap_trans)."""
    import numpy as np

    p = configs.hetero(nx=12, ny=10, nz=8, nsteps=2, seed=41)
    p.bc["x_lower"] = BC(BC_DIRICHLET, (1.8,), ref_patch="z_lower")
    p.bc["x_upper"] = BC(BC_SEEPAGE, (0.0,))
    rng = np.random.default_rng(41)
    p.evap_trans = 0.02 * (rng.random(p.shape) - 0.5)
    p.print_velocities = True
    return p


def vel_overland_small() -> RichardsProblem:
    """Face velocities and the overland fluxes q_overlnd_x / y of the
    ponded kinematic overland case (Solver.PrintQxOverland / PrintQyOverland)."""
    p = overland_small()
    p.nsteps = 3
    p.print_velocities = True
    return p


def growth_small() -> RichardsProblem:
    """The time loop with TimeStep.Type Growth (initial 0.04, factor 1.7,
    min 0.01, max 0.15) on a box whose top flux cycles between rain (2 base
    units of 0.1) and none (3 units): steps grow, are cut at the cycle's
    transitions and at the stop time; pressures written every step."""
    p = configs.box(nx=14, ny=12, nz=9, nsteps=7, dt=0.1, seed=47)
    p.bc["z_upper"] = BC(BC_FLUX, (-0.05, 0.0), lengths=(2, 3), repeat=-1)
    p.growth = (0.04, 1.7, 0.01, 0.15)
    return p


def halving_small() -> RichardsProblem:
    """The dt-halving retry of AdvanceRichards: steps of 1.0 with
    Solver.Nonlinear.MaxIter 4, too few for the first steps, so KINSol fails
    and the step is retried at dt / 2 and dt / 4 from the old state
    (Solver.MaxConvergenceFailures 3); dump times every 1.0 snap the
    following steps."""
    return configs.box(nx=12, ny=10, nz=8, nsteps=2, dt=1.0, seed=43,
                       solver=SolverSettings(max_iter=4))


def restart_small() -> RichardsProblem:
    """Restarted GMRES: Solver.Linear.KrylovDimension 2 with
    Solver.Linear.MaxRestarts 5 and a two-level multigrid on config-2 physics
    with steps of 5 h, so that most linear solves need several cycles
    (spgmr.c:390-409)."""
    return configs.hetero(nx=15, ny=13, nz=9, nsteps=2, dt=5.0, seed=53,
                          solver=SolverSettings(krylov_dim=2, max_restarts=5, mg_max_levels=2))


def picard_small() -> RichardsProblem:
    """PCMatrixType Picard (the reference builds the same symmetric
    preconditioner matrix as for PFSymmetric) on config-2 physics."""
    return configs.hetero(nx=13, ny=11, nz=8, nsteps=2, seed=59,
                          solver=SolverSettings(pc_matrix_type="Picard"))


def inexact_small() -> RichardsProblem:
    """Solver.Nonlinear.Globalization InexactNewton: the full Newton step,
    no line search (kinsol.c:1152-1208), on config-2 physics with steps of
    20 h, where the line search would backtrack (8 Newton iterations and 35
    residual evaluations in the first step against 5 and 6 here)."""
    return configs.hetero(nx=13, ny=12, nz=8, nsteps=3, dt=20.0, seed=61,
                          solver=SolverSettings(globalization="InexactNewton"))


def flow_barrier_small() -> RichardsProblem:
    """Flow barriers (Solver.Nonlinear.FlowBarrierX/Y/Z with PFB fields, as
    the reference's richards_FBx / FBy tests): a near-closed x barrier
    between columns 5 and 6, a partial y barrier and a z barrier layer, all
    on interior faces, on config-2 physics."""
    prob = configs.hetero(nx=12, ny=11, nz=9, nsteps=2, seed=67)
    fbx = np.ones(prob.shape)
    fbx[:, :, 5] = 0.001
    fby = np.ones(prob.shape)
    fby[:, 4, 2:9] = 0.1
    fbz = np.ones(prob.shape)
    fbz[3, :, :] = 0.5
    prob.fbx, prob.fby, prob.fbz = fbx, fby, fbz
    return prob


def fulljac_small() -> RichardsProblem:
    """PCMatrixType FullJacobian: the multigrid's finest operator is the full
    non-symmetric Jacobian, the coarse operators symmetric
    (mg_semi.c:1071-1072), on config-2 physics."""
    return configs.hetero(nx=13, ny=11, nz=8, nsteps=2, seed=71,
                          solver=SolverSettings(pc_matrix_type="FullJacobian"))


def fulljac_overland_small() -> RichardsProblem:
    """PCMatrixType FullJacobian with kinematic overland flow and
    KINSOL's difference-quotient J v, the combination of the reference's
    overland_tiltedV_MGSemiTest: the finest multigrid operator carries the
    surface terms' non-symmetric entries."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=3, seed=73, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=1,
                            solver=SolverSettings(pc_matrix_type="FullJacobian",
                                                  use_jacobian=False))


def fulljac_diff_small() -> RichardsProblem:
    """PCMatrixType FullJacobian with diffusive-wave overland routing, whose
    surface terms reach the W entries of the first column."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=3, dt=0.05, seed=79, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=1, kind=BC_OVERLAND_DIFF,
                            solver=SolverSettings(pc_matrix_type="FullJacobian"))


def dq_overland_flow_small() -> RichardsProblem:
    """The OverlandFlow patch with KINSOL's difference-quotient J v: the
    reference then builds the preconditioner without the surface terms and
    with the diagonal term of its "simple" case on ponded top cells
    (richards_jacobian_eval.c:1241-1254, 2476-2484)."""
    return configs.overland(nx=12, ny=10, nz=6, nsteps=3, seed=83, wt_depth=-0.02,
                            mannings=1e-3, rain_steps=2, dry_steps=1, kind=BC_OVERLAND,
                            solver=SolverSettings(use_jacobian=False))


def dirichlet_top_small() -> RichardsProblem:
    """A Dirichlet (constant head) top face: its Jacobian coefficient takes
    the mean of the top layer's z multiplier and the ghost one above, which
    keeps the 1 it was initialised with (richards_jacobian_eval.c:1168-1170,
    problem_dz_scale.c:92)."""
    p = configs.box(nx=10, ny=8, nz=6, nsteps=2, seed=5)
    p.bc["z_upper"] = BC(BC_DIRICHLET, (-0.3,))
    return p


def mg_maxiter_small() -> RichardsProblem:
    """MGSemi.MaxIter 2: two V-cycles per preconditioner application, the
    second starting with a smoothing of the first's result (mg_semi.c:
    198-365), on config-2 physics."""
    return configs.hetero(nx=13, ny=11, nz=8, nsteps=2, seed=89,
                          solver=SolverSettings(mg_max_iter=2))


def mg_minn_small() -> RichardsProblem:
    """MGSemi.MaxMinNX 3 and MaxMinNZ 3: x and z are coarsened only while
    they have at least 5 cells (mg_semi.c:869-872), which changes the
    hierarchy's coarsening directions and depth, on config-2 physics."""
    return configs.hetero(nx=13, ny=11, nz=8, nsteps=2, seed=97,
                          solver=SolverSettings(mg_max_min_n=(3, 1, 3)))


def spinup_small() -> RichardsProblem:
    """OverlandFlowSpinUp 1 with OverlandSpinupDampP1 / P2 on the OverlandFlow
    case: the ponded head drains in place of the routing, and the damping
    term acts on non-ponded top cells (nl_function_eval.c:1659-1673)."""
    p = configs.overland(nx=12, ny=10, nz=6, nsteps=3, dt=1.0, seed=101, wt_depth=0.02,
                         mannings=1e-3, rain_steps=2, dry_steps=1, kind=BC_OVERLAND,
                         solver=SolverSettings(max_iter=60))
    p.overland_spinup = 1
    p.spinup_damp = (10.0, 1e-4)
    return p


def spinup_damp_small() -> RichardsProblem:
    """OverlandSpinupDampP1 / P2 without spin-up: the damping term joins the
    ponding and routing term of the OverlandFlow patch (two rain steps; the
    dry step after them needs 74 GMRES iterations in 4 Newton iterations,
    where rounding alone moves the count by one)."""
    p = configs.overland(nx=12, ny=10, nz=6, nsteps=2, seed=103, wt_depth=0.02,
                         mannings=1e-3, rain_steps=2, dry_steps=1, kind=BC_OVERLAND)
    p.spinup_damp = (10.0, 1e-4)
    return p


# pressure output of the golden runs (to_reference's dump_interval):
# every step for the growth case, every 1.0 (one base dt) otherwise
DUMP = {"growth_small": -1}

GOLDEN = ["box_small", "box_odd", "hetero_small", "walker2_small", "hydrostatic",
          "overland_small", "tfg_small", "overland_diff_small",
          "overland_flow_small", "seepage_small", "dq_small", "krtable_spline_small",
          "krtable_linear_small", "wjacobi_small", "rbgs_nonsym_small", "vel_small",
          "vel_overland_small", "growth_small", "halving_small", "restart_small",
          "picard_small", "inexact_small", "flow_barrier_small", "fulljac_small",
          "fulljac_overland_small", "fulljac_diff_small", "dq_overland_flow_small",
          "dirichlet_top_small", "mg_maxiter_small", "mg_minn_small",
          "spinup_small", "spinup_damp_small"]
# cases whose steps are not the constant-dt plan of RichardsProblem.time_plan
TIME_LOOP = ["growth_small", "halving_small"]


def get(name: str) -> RichardsProblem:
    return globals()[name]()


__all__ = ["get", "GOLDEN", "TIME_LOOP", "DUMP"] + GOLDEN
