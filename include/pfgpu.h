/*
 * pfgpu.h -- C ABI of the B200 Richards Newton-Krylov library (libpfgpu.so).
 *
 * One handle owns one Richards problem resident in GPU memory: the grid, the
 * cell fields, the boundary-condition tables and the nonlinear-solver state.
 * Every function is plain C: pointers, sizes and status codes; no CUDA or
 * torch type appears in a signature.  All functions return 0 on success,
 * a positive code for a recoverable condition (e.g. a nonlinear solve that
 * did not converge, which ParFlow answers by halving dt) and a negative code
 * for an error; pfgpu_last_error() describes the last failure.
 *
 * Cell vectors crossing this ABI use ParFlow's Subvector layout with a
 * one-cell ghost frame: element (i,j,k), -1 <= i <= nx etc., lives at
 *   (i+1) + ((j+1) + (k+1)*(ny+2))*(nx+2)
 * which is SubvectorEltIndex (pfsimulator/parflow_lib/vector.h:133-138) for
 * a subvector with ix = iy = iz = -1, so ParFlow can pass SubvectorData()
 * pointers unchanged.  Ghost values are ignored on input and written as 0 on
 * output.  Pointers may be host or device (including managed) memory; the
 * library detects which.
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the ParFlow source tree).
 */
#ifndef PFGPU_H
#define PFGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFGPU_ABI_VERSION 2

/* status codes */
#define PFGPU_OK 0
#define PFGPU_NOT_CONVERGED 1      /* recoverable: retry the step with dt/2 */
#define PFGPU_ERR_ARG (-1)
#define PFGPU_ERR_CUDA (-2)
#define PFGPU_ERR_STATE (-3)
#define PFGPU_ERR_NOMEM (-4)

/* precision of the preconditioner and of the Jacobian matvec inside GMRES;
 * the residual, Newton update, Arnoldi process and all norms stay FP64 */
#define PFGPU_PREC_FP64 0
#define PFGPU_PREC_MIXED 1
/* as MIXED, with each multigrid level's operator stored symmetrically
 * diagonal-scaled in FP16: with S = sqrt(diag A) the V-cycle runs on S x,
 * S^-1 b and S^-1 A S^-1 (unit diagonal, off-diagonals A_ij / (S_i S_j) in
 * FP16), the scaling folded into the transfer weights.  In exact arithmetic
 * this is the same MGSemi V-cycle; it moves 6 instead of 16 operator bytes
 * per cell (8 on hierarchies where some diagonal is not positive, e.g. with
 * kinematic overland terms: S = sqrt(|diag A|) and the +-1 diagonal is then
 * read too).  No counterpart in the reference. */
#define PFGPU_PREC_MIXED_H16 2

/* boundary-condition types, one per box face
 * (pfsimulator/parflow_lib/bc_pressure.h:97 BC_TYPE_TABLE) */
#define PFGPU_BC_FLUX 0        /* FluxConst: volume flux per area, + = out of upper faces */
#define PFGPU_BC_DIRICHLET 1   /* DirEquilRefPatch: pressure head values on the face */
#define PFGPU_BC_OVERLAND_KIN 2 /* OverlandKinematic (z_upper only): rain flux values as
                                  * FluxConst plus kinematic-wave ponding and routing */
#define PFGPU_BC_OVERLAND_DIFF 3 /* OverlandDiffusive (z_upper only): the same with
                                   * diffusive-wave routing, whose friction slope
                                   * includes the ponded-depth gradient */
#define PFGPU_BC_OVERLAND 4      /* OverlandFlow (z_upper only): the same with each
                                   * column's kinematic flux along its own slope,
                                   * upwinded between columns (overlandflow_eval.c) */
#define PFGPU_BC_SEEPAGE 5       /* SeepageFace: flux values as FluxConst; on z_upper
                                   * the ponded water also drains, (vol/dz) dt max(p, 0)
                                   * (nl_function_eval.c:1692-1784) */

/* faces, ParFlow box patch order */
#define PFGPU_X_LOWER 0
#define PFGPU_X_UPPER 1
#define PFGPU_Y_LOWER 2
#define PFGPU_Y_UPPER 3
#define PFGPU_Z_LOWER 4
#define PFGPU_Z_UPPER 5

/* cell fields for pfgpu_set_field */
#define PFGPU_FIELD_PERM_X 0
#define PFGPU_FIELD_PERM_Y 1
#define PFGPU_FIELD_PERM_Z 2
#define PFGPU_FIELD_VG_ALPHA 3
#define PFGPU_FIELD_VG_N 4
#define PFGPU_FIELD_S_RES 5
#define PFGPU_FIELD_S_SAT 6
/* flow-barrier multipliers of the faces between a cell and its +x / +y / +z
 * neighbour (Solver.Nonlinear.FlowBarrierX/Y/Z, problem_FBx.c:60-120;
 * nl_function_eval.c:841-843, richards_jacobian_eval.c:662-728); NULL values
 * restore 1 everywhere.  The multipliers of the last cell along each
 * direction (the boundary faces) are not used: the boundary patches set
 * those fluxes. */
#define PFGPU_FIELD_FB_X 7
#define PFGPU_FIELD_FB_Y 8
#define PFGPU_FIELD_FB_Z 9

/* eta choice (pfsimulator/parflow_lib/kinsol_nonlin_solver.c:804-850) */
#define PFGPU_ETA_CONSTANT 0
#define PFGPU_ETA_WALKER1 1
#define PFGPU_ETA_WALKER2 2

/* smoothers (pfsimulator/parflow_lib/mg_semi.c:1251): RedBlackGSPoint with
 * Smoother.Symmetric True (red, black, red) or False (red, black;
 * rb_GS_point.c:452-470), WJacobi with Smoother.Weight (w_jacobi.c:392) */
#define PFGPU_SMOOTH_RBGS 0
#define PFGPU_SMOOTH_WJACOBI 1
#define PFGPU_SMOOTH_RBGS_NONSYM 2

typedef struct pfgpu_handle pfgpu_handle;

/* Grid, constant physics and solver keys of one problem.  Scalar fields
 * (uniform porosity, storage, van Genuchten parameters) live here; spatially
 * varying ones are uploaded with pfgpu_set_field. */
typedef struct {
  int abi_version;                  /* PFGPU_ABI_VERSION */
  int nx, ny, nz;
  double dx, dy, dz;
  double gravity, viscosity, density;
  double porosity, specific_storage;
  double vg_alpha, vg_n, s_res, s_sat; /* used where no per-cell field is set */
  int vg_from_file;                 /* Phase.Saturation.VanGenuchten.File */
  const double *z_mult;             /* nz dz multipliers, NULL = 1 */
  int precision;                    /* PFGPU_PREC_* */
  /* Solver.Nonlinear.* / Solver.Linear.* keys */
  double residual_tol, step_tol;
  int max_iter, krylov_dim, max_restarts;  /* krylov_dim: 1 .. 64 */
  int eta_choice;
  double eta_value, eta_alpha, eta_gamma;
  int mg_max_levels, mg_smoother;
  double wjacobi_weight;
  /* MGSemi.MaxMinNX / NY / NZ (mg_semi.c:1318-1325, default 1): a direction
   * is coarsened only while it has at least max(2 n - 1, 2) cells
   * (mg_semi.c:869-872); 0 counts as 1 */
  int mg_max_min_n[3];
} pfgpu_desc;

/* Counters of one nonlinear solve (the kinsol.log fields,
 * pfsimulator/parflow_lib/kinsol_nonlin_solver.c:239-264). */
typedef struct {
  int kinsol_status;   /* KINSOL return value (1 success, 2 initial guess ok, ...) */
  int nonlin_iters, lin_iters, fevals, pc_setups, pc_solves;
  int lin_conv_fails, beta_cond_fails, backtracks;
  double fnorm;
} pfgpu_stats;

/* Creates the problem on CUDA device `device`; replaces the instance setup of
 * KinsolNonlinSolverInitInstanceXtra (pfsimulator/parflow_lib/kinsol_nonlin_solver.c:456-680).
 * Returns NULL on error (see pfgpu_last_error). */
pfgpu_handle *pfgpu_create(const pfgpu_desc *desc, int device);

/* Frees every device allocation of the handle
 * (KinsolNonlinSolverFreeInstanceXtra, kinsol_nonlin_solver.c:690). */
void pfgpu_destroy(pfgpu_handle *h);

/* Message for the last failing call on this thread. */
const char *pfgpu_last_error(void);

/* Uploads a spatially varying cell field (ParFlow layout).  Replaces the
 * ProblemData fields read by the modules: permeability (subsrf_sim.c:684-810),
 * per-cell van Genuchten parameters (problem_saturation.c:943-950,
 * problem_phase_rel_perm.c:1930-1932), flow barriers (problem_FBx.c).
 * values == NULL on a van Genuchten field (PFGPU_FIELD_VG_ALPHA .. S_SAT)
 * drops its per-cell array, so that the descriptor's scalar serves every cell
 * again, and on a flow-barrier field restores 1; permeability needs values. */
int pfgpu_set_field(pfgpu_handle *h, int field, const double *values);

/* Time-cycled boundary data (TimeCycleData, time_cycle_data.c, and the
 * per-interval patch values BCPressure keeps): face `face` takes, during
 * interval q of its cycle, type types[q] and the face table
 * values + q * (face cells) (the layout of pfgpu_set_bc).  Interval q lasts
 * lengths[q] base time units; the cycle repeats `repeat` times (-1: for
 * ever), counted from start_time (ProblemBaseTimeUnit / ProblemStartTime).
 * Every table is uploaded once; pfgpu_run selects the interval of each step
 * on the device side.  pfgpu_set_bc on the face replaces the cycle. */
int pfgpu_set_bc_cycle(pfgpu_handle *h, int face, int nint, const int *types,
                       const double *values, const int *lengths, int repeat, double base_unit,
                       double start_time);

/* Time step selection (SelectTimeStep, select_time_step.c:58-155): type 0
 * constant `step`; type 1 growth: `step` on the first step, then the last
 * step times `factor`, clamped to [min_step, max_step]; either is then cut to
 * the next boundary-cycle transition.  max_failures: convergence failures
 * (each halves dt) before a step is given up (Solver.MaxConvergenceFailures). */
int pfgpu_set_time_step(pfgpu_handle *h, int type, double step, double factor,
                        double min_step, double max_step, int max_failures);

/* AdvanceRichards's time loop on the device state (solver_richards.c:
 * 2965-3406): from time t until stop_time (at most max_steps steps) select
 * dt, snap it to the next dump time (dump_interval > 0) and cut it to the
 * stop time, copy the old pressure and saturation on the device, evaluate the
 * boundary cycles at the new time, solve, and on failure halve dt and retry
 * from the old state.  times / dts / stats (each max_steps long, may be
 * null) receive the new time, dt and counters of every step; *nsteps the
 * number of steps taken.  No counterpart as one call in the reference. */
int pfgpu_run(pfgpu_handle *h, double t, double stop_time, double dump_interval, int max_steps,
              double *times, double *dts, pfgpu_stats *stats, int *nsteps);

/* ParFlow binary (PFB) files of the device state.  The format
 * (write_parflow_binary.c:74-205, read_parflow_binary.c:38-120): big-endian
 * origin x y z and spacings, nx ny nz, the number of subgrids, then per
 * subgrid its box and values, x fastest.
 *
 * pfgpu_write_pfb writes the current pressure (PFGPU_PFB_PRESSURE) or the
 * saturation at it (PFGPU_PFB_SATURATION) as one subgrid with the
 * descriptor's spacings and the given origin; the values are packed and
 * byte-swapped on the device and copied to the host once.
 * pfgpu_read_pfb reads a file of any subgrid layout for this grid and sets
 * the current pressure (PFGPU_PFB_PRESSURE) or a cell field
 * (PFGPU_FIELD_*, as pfgpu_set_field): each subgrid's raw values are copied
 * to the device once and scattered and byte-swapped there.  A file for
 * another grid size, or a subgrid outside the grid, is an argument error. */
#define PFGPU_PFB_PRESSURE 100
#define PFGPU_PFB_SATURATION 101
int pfgpu_write_pfb(pfgpu_handle *h, int what, const char *path, double x0, double y0,
                    double z0);
int pfgpu_read_pfb(pfgpu_handle *h, int what, const char *path);

/* Surface data of the top layer (ProblemData TSlopeX / TSlopeY / Mannings,
 * problem_toposlopes.c, problem_mannings.c): host arrays in ParFlow's 2-D
 * subvector layout, element (i,j) at (i+1) + (j+1)*(nx+2), ghosts ignored.
 * terrain_following (Solver.TerrainFollowingGrid, solver_richards.c:562-572)
 * puts the slopes into the subsurface x / y face gravity terms
 * (nl_function_eval.c:725-733, richards_jacobian_eval.c:620-660);
 * ov_epsilon is Solver.OverlandKinematic.Epsilon or
 * Solver.OverlandDiffusive.Epsilon (1e-5 by default).  Needed before a
 * PFGPU_BC_OVERLAND_KIN, PFGPU_BC_OVERLAND_DIFF or PFGPU_BC_OVERLAND face is
 * set. */
int pfgpu_set_surface(pfgpu_handle *h, const double *slope_x, const double *slope_y,
                      const double *mannings, int terrain_following, double ov_epsilon);

/* OverlandFlowSpinUp (0 or 1) and OverlandSpinupDampP1 / P2 (0 by default)
 * of a PFGPU_BC_OVERLAND face (NlFunctionEval, nl_function_eval.c:1659-1673;
 * RichardsJacobianEval, richards_jacobian_eval.c:1258-1287, 2044-2057):
 * with spin-up the ponded head drains at (vol/dz) dt max(p, 0) in place of
 * the ponding and routing term; the damping term (vol/dz) dt
 * exp(min(p, 0) P1) P2 joins either.  The Jacobian keeps the reference's
 * terms as they are.  Not available with pfgpu_adjoint_gradient. */
int pfgpu_set_overland_spinup(pfgpu_handle *h, int spinup, double damp_p1, double damp_p2);

/* Sets the boundary condition of one face at the current time: `values`
 * holds one value per boundary cell, x faces (nz, ny), y faces (nz, nx),
 * z faces (ny, nx), first index slowest.  Replaces the BCStruct built by
 * BCPressure (pfsimulator/parflow_lib/problem_bc_pressure.c:60).  An
 * OverlandKinematic face (z_upper) adds the kinematic-wave overland flow of
 * overlandflow_eval_Kin.c to the top layer (nl_function_eval.c:1786-2000,
 * richards_jacobian_eval.c:1863-1990); an OverlandDiffusive face the
 * diffusive-wave flow of overlandflow_eval_diffusive.c
 * (nl_function_eval.c:2028-2259, richards_jacobian_eval.c:1989-2026); an
 * OverlandFlow face that of overlandflow_eval.c (nl_function_eval.c:1437-1690,
 * richards_jacobian_eval.c:2028-2090). */
int pfgpu_set_bc(pfgpu_handle *h, int face, int type, const double *values);

/* Residual F(p) of one implicit step (NlFunctionEval,
 * pfsimulator/parflow_lib/nl_function_eval.c:167).  p, p_old, s_old, f in
 * ParFlow layout. */
int pfgpu_nl_function_eval(pfgpu_handle *h, const double *p, const double *p_old,
                           const double *s_old, double dt, double *f);

/* Land-surface sink/source per cell [1/h], the evap_trans vector the
 * residual subtracts as vol z_mult dt (source + evap_trans)
 * (nl_function_eval.c:533-541; read from Solver.EvapTrans.FileName or set by
 * CLM each step, solver_richards.c:1080-1090).  ParFlow layout, host or
 * device; NULL clears it (zero).  Kept until replaced; the Jacobian does not
 * depend on it.  The reference's ovrl_bc_flx argument is not read by the
 * residual (nl_function_eval.c:178), so it has no setter. */
int pfgpu_set_evap_trans(pfgpu_handle *h, const double *et);

/* Face velocities [m/h] and overland fluxes of the residual evaluated at p:
 * what NlFunctionEval writes into x_velocity, y_velocity, z_velocity (interior
 * faces flux / area, nl_function_eval.c:845-848; boundary faces as the patch
 * loops store them, :1227-1230, :1432, :1681-1687, :1775-1781) and
 * q_overlnd_x / q_overlnd_y (ke, kn of each column on an overland z_upper
 * face, :1648-1656; zero otherwise).  p = NULL takes the handle's pressure
 * state (the solution of the last pfgpu_newton_solve / pfgpu_advance step);
 * p_old / s_old = NULL keep the old pressure and saturation of the last
 * solve or evaluation, so after a solve pfgpu_face_velocities(h, NULL, NULL,
 * NULL, dt, ...) gives the velocities of the last residual evaluation of
 * that step, as the reference's state holds after KINSol returns.  Outputs
 * in the layouts of ParFlow's state vectors on the face grids (one cell
 * wider along their axis; solver_richards.c:1035-1045, 5110-5160), ghosts
 * written as 0: vx (nx+3)(ny+2)(nz+2) and vy (nx+2)(ny+3)(nz+2) with one
 * ghost layer, vz (nx+4)(ny+4)(nz+5) with two, qx / qy on the 2-D grid
 * (nx+2)(ny+2)*3 with one; host or device; any may be NULL. */
int pfgpu_face_velocities(pfgpu_handle *h, const double *p, const double *p_old,
                          const double *s_old, double dt, double *vx, double *vy, double *vz,
                          double *qx, double *qy);

/* y = J(p) x with the analytic 7-point Jacobian assembled at p
 * (KINSolMatVec + RichardsJacobianEval with symm_part = 0,
 * pfsimulator/parflow_lib/richards_jacobian_eval.c:165, :217; Matvec,
 * matvec.c:35).  Uses the handle's matvec precision. */
int pfgpu_jacobian_matvec(pfgpu_handle *h, const double *p, double dt,
                          const double *x, double *y);

/* Relative permeability from the reference's lookup table instead of the
 * closed form (Geom.domain.RelPerm.NumSamplePoints / MinPressureHead /
 * InterpolationMethod, problem_phase_rel_perm.c:1894-1916; VanGComputeTable
 * :116-262): kr and its derivative at num_sample_points + 1 evenly spaced
 * heads from 0 to |min_pressure_head|, interpolated by monotone cubic
 * Hermite splines or linearly; zero beyond the table.  Needs uniform van
 * Genuchten alpha and n (the descriptor scalars).  PFGPU_KRT_NONE restores
 * the closed form.  The adjoint is not available with a table. */
#define PFGPU_KRT_NONE 0
#define PFGPU_KRT_SPLINE 1
#define PFGPU_KRT_LINEAR 2
int pfgpu_set_relperm_table(pfgpu_handle *h, int method, int num_sample_points,
                            double min_pressure_head);

/* Solver.Nonlinear.UseJacobian and Solver.Nonlinear.DerivativeEpsilon
 * (kinsol_nonlin_solver.c:860-885): use_jacobian = 1 (the default of this
 * library) gives GMRES the analytic Jacobian; 0 the difference quotient
 * J v = (F(u + sigma v) - F(u)) / sigma of KINSpgmrAtimesDQ
 * (kinsol/kinspgmr.c:481-518) with sigma from sqrt(derivative_epsilon), one
 * residual evaluation per product (counted in fevals); the preconditioner
 * keeps the analytic symmetric part.  Not available with an overland face
 * (the solves return PFGPU_ERR_STATE). */
int pfgpu_set_jacobian_mode(pfgpu_handle *h, int use_jacobian, double derivative_epsilon);

/* Sets the old pressure (ParFlow layout) that the Jacobian of
 * pfgpu_jacobian_matvec and pfgpu_pc_setup reads: the old_pressure argument
 * of RichardsJacobianEval (richards_jacobian_eval.c:217), used only by the
 * diffusive overland terms.  pfgpu_nl_function_eval and the solves set it
 * too (their p_old). */
int pfgpu_set_old_pressure(pfgpu_handle *h, const double *p_old);

/* Assembles the preconditioner matrix (PCMatrixType PFSymmetric) at p and
 * builds the semicoarsening multigrid hierarchy
 * (KinsolPCInitInstanceXtra, kinsol_pc.c:85; MGSemiInitInstanceXtra,
 * mg_semi.c:766). */
int pfgpu_pc_setup(pfgpu_handle *h, const double *p, double dt);

/* z = M^{-1} r: one V-cycle with zero initial guess (KinsolPC,
 * kinsol_pc.c:58 -> MGSemi, mg_semi.c:93).  r and z may alias. */
int pfgpu_pc_apply(pfgpu_handle *h, const double *r, double *z);

/* Saturation S(p) (Saturation with CALCFCN, problem_saturation.c:108). */
int pfgpu_saturation(pfgpu_handle *h, const double *p, double *s);

/* One implicit step: solves F(p) = 0 by inexact Newton-Krylov with line
 * search, entirely on the GPU (KinsolNonlinSolver -> KINSol,
 * kinsol_nonlin_solver.c:297, pfsimulator/kinsol/kinsol.c:690).
 * p: in = initial guess (normally p_old), out = solution; p may be the
 * p_old buffer itself (it is then copied in once).  Returns
 * PFGPU_OK, or PFGPU_NOT_CONVERGED when KINSOL would fail. */
int pfgpu_newton_solve(pfgpu_handle *h, const double *p_old, const double *s_old,
                       double dt, double *p, pfgpu_stats *stats);

/* pfgpu_newton_solve followed by the saturation at the new pressure
 * (AdvanceRichards evaluates it right after the solve,
 * solver_richards.c:3408-3420): both results leave the device in one call, so
 * a host caller copies p in once and p and s out once.  s may be the s_old
 * buffer and p the p_old buffer (both are read before anything is written). */
int pfgpu_newton_solve_sat(pfgpu_handle *h, const double *p_old, const double *s_old,
                           double dt, double *p, double *s, pfgpu_stats *stats);

/* How every Newton solve of the handle runs.  mode 1 (the default; the
 * environment variable PFGPU_SOLVE_GRAPH=0 makes 0 the default): the whole
 * solve is one CUDA graph launch, captured at the first solve and again
 * whenever the problem's boundary tables, fields or Jacobian mode change;
 * control kernels on the device take KINSOL's and SPGMR's decisions and the
 * host reads the counters once per solve.  mode 0: the host drives the
 * iteration (one small device-to-host read per GMRES iteration and per
 * line-search evaluation).  Both take the same steps with the same
 * arithmetic.  mode -1 returns 1 if the handle's last solve ran as a graph,
 * 0 if it ran host-driven (phase timing on, or the graph could not be built:
 * pfgpu_last_error then says why).  No counterpart in the reference (its
 * KINSOL loop is host code). */
int pfgpu_solve_graph(pfgpu_handle *h, int mode);

/* Solver.Nonlinear.Globalization (kinsol_nonlin_solver.c:887-905):
 * PFGPU_GLOBAL_LINE_SEARCH (the default, KINLineSearch, kinsol.c:1228-1420)
 * or PFGPU_GLOBAL_INEXACT_NEWTON (KINInexactNewton, kinsol.c:1152-1208: the
 * full Newton step, shortened to the maximum step, no backtracking). */
#define PFGPU_GLOBAL_LINE_SEARCH 0
#define PFGPU_GLOBAL_INEXACT_NEWTON 1
int pfgpu_set_globalization(pfgpu_handle *h, int strategy);

/* Solver.Linear.Preconditioner.PCMatrixType (KinsolPCNewPublicXtra,
 * kinsol_pc.c:215-246): PFGPU_PCM_SYMMETRIC for PFSymmetric, SymmetricPart
 * and Picard (the reference builds the same symmetric matrix for the three:
 * richards_jacobian_eval.c:760, 781), PFGPU_PCM_FULL for FullJacobian, where
 * the multigrid's finest operator is the full non-symmetric Jacobian and its
 * coarse operators are symmetric (mg_semi.c:1071-1072).  FullJacobian needs
 * a red/black Gauss-Seidel smoother, at least two multigrid levels and the
 * FP64 or FP32 multigrid (not PFGPU_PREC_MIXED_H16).  With
 * pfgpu_set_jacobian_mode(h, 0, ...) the matrix is built as the reference
 * builds it under UseJacobian False: without the overland surface terms
 * (richards_jacobian_eval.c:1241-1254, 1863, 2476-2484). */
#define PFGPU_PCM_SYMMETRIC 0
#define PFGPU_PCM_FULL 1
int pfgpu_set_pc_matrix(pfgpu_handle *h, int type);

/* Solver.Linear.Preconditioner.MGSemi.MaxIter (MGSemiNewPublicXtra,
 * mg_semi.c:1312-1313; default 1): V-cycles per preconditioner application,
 * KinsolPC's tolerance 0 skipping every convergence test (kinsol_pc.c:65-72,
 * mg_semi.c:198-365).  0 makes the preconditioner the identity; a cycle
 * after the first begins with a smoothing of the finest level's current
 * iterate. */
int pfgpu_set_mg_max_iter(pfgpu_handle *h, int max_iter);

/* Device-resident time stepping: advances the handle's own pressure state by
 * nsteps steps of dt with the boundary tables already set, keeping every
 * vector on the GPU (the step body of AdvanceRichards,
 * pfsimulator/parflow_lib/solver_richards.c:2965-3406, without output).
 * stats (may be NULL) receives the per-step counters, nsteps entries. */
int pfgpu_set_pressure(pfgpu_handle *h, const double *p);
int pfgpu_get_pressure(pfgpu_handle *h, double *p);
int pfgpu_advance(pfgpu_handle *h, double dt, int nsteps, pfgpu_stats *stats);

/* Ensemble stepping: advances n independent problems (one handle each, same
 * semantics as pfgpu_advance, members[m] by dt[m]) concurrently.  By default
 * each timestep of all members is one CUDA graph launch holding every
 * member's whole Newton solve with its own device-side control (members
 * converge independently; a failed solve is retried with the halved dt for
 * that member alone).  Where that does not apply (PFGPU_ENSEMBLE_GRAPH=0,
 * host-driven solves, trajectory recording, members on several devices) the
 * members run on their own streams, driven by nthreads host threads (0 = one
 * per member).  stats (may be NULL) receives
 * n * nsteps entries, member-major; status[m] receives each member's
 * pfgpu_advance result.  Returns PFGPU_OK when every member succeeded,
 * otherwise the first error (or PFGPU_NOT_CONVERGED).  The members must be
 * distinct handles.  The reference runs ensemble members as separate runs;
 * no counterpart in its API. */
int pfgpu_ensemble_advance(pfgpu_handle *const *members, int n, const double *dt, int nsteps,
                           int nthreads, pfgpu_stats *stats, int *status);

/* Discrete adjoint of the implicit timesteps (no counterpart in the
 * reference).  pfgpu_adjoint_record starts a trajectory at the handle's
 * current pressure (p_0) with room for max_steps steps; every successful step
 * of pfgpu_advance after it appends p_n and the dt it used.
 * pfgpu_adjoint_gradient then returns, for the objective
 *   g = sum over observed steps n and observed cells c of (p_n[c] - obs)^2,
 * its value (*misfit) and its gradient with respect to the per-cell ln K
 * (every direction's permeability scaled together), van Genuchten alpha and
 * n (ParFlow layout, host or device; NULL skips one), by solving
 * J_n^T lambda_n = -dg/dp_n - (dF_{n+1}/dp_n)^T lambda_{n+1} backwards in n
 * with GMRES on the transposed analytic Jacobian (multigrid preconditioned)
 * to relative residual tol, and summing lambda_n^T dF_n/dtheta.
 * obs_steps (nobs_steps values in 1..recorded steps), obs_cells (nobs dense
 * interior indices i + nx*(j + ny*k)) and obs_values (nobs_steps x nobs,
 * step-major) are host arrays.  The boundary tables in effect are used for
 * every step (constant boundary conditions over the window).  Use an FP64
 * handle: the mixed form stores J in FP32.  Not available with a diffusive
 * overland face (PFGPU_ERR_STATE): its terms depend on the old pressure
 * through the slope magnitude, a coupling between steps with no adjoint
 * here. */
int pfgpu_adjoint_record(pfgpu_handle *h, int max_steps);
int pfgpu_adjoint_gradient(pfgpu_handle *h, int nobs_steps, const int *obs_steps, int nobs,
                           const long long *obs_cells, const double *obs_values, double tol,
                           double *misfit, double *grad_lnk, double *grad_alpha,
                           double *grad_n);

/* Number of multigrid levels and their sizes/coarsening directions
 * (mg_semi.c:858-923); dims has 4*levels ints (nx, ny, nz, dir). */
int pfgpu_mg_levels(pfgpu_handle *h, int *levels, int *dims, int max_levels);

/* Times one of the library's kernels on its own stream with CUDA events:
 * `reps` back-to-back launches on the handle's current state (after a solve
 * or pfgpu_pc_setup), average duration per launch in *ms, and the kernel's
 * algorithmic HBM bytes per launch (each distinct per-cell array it needs
 * counted once; uniform fields count zero) in *bytes.
 * kernel: 0 residual (with its van Genuchten pass), 1 Jacobian + PC matrix
 * assembly, 2 Jacobian matvec, 3 the symmetric red/black/red smoother on the
 * finest level as the V-cycle runs it (bytes: each array once, the one-pass
 * ideal), 4 one multigrid V-cycle (all levels), 5 multigrid setup, 6 one red
 * colour sweep on the finest level (a single k_rb_sweep launch).
 * Benchmark support; no counterpart in the reference. */
#define PFGPU_KERNEL_RESIDUAL 0
#define PFGPU_KERNEL_JACOBIAN 1
#define PFGPU_KERNEL_MATVEC 2
#define PFGPU_KERNEL_RB_SWEEP 3
#define PFGPU_KERNEL_VCYCLE 4
#define PFGPU_KERNEL_MG_SETUP 5
#define PFGPU_KERNEL_COLOUR_SWEEP 6
int pfgpu_time_kernel(pfgpu_handle *h, int kernel, int reps, double *ms, double *bytes);

/* Autotuner of the stencil launches (no counterpart in the reference):
 * times candidate thread-block shapes (bx, by) of the residual, Jacobian
 * and matvec kernels on this handle's grid, `reps` launches each on its
 * current state, and keeps the fastest (the built-in heuristic unless a
 * shape is clearly faster).  Choices are cached per grid size, precision
 * and kernel variant for the life of the process, so later handles of the
 * same size (ensemble members) take them without timing.  shapes (6 ints,
 * may be NULL) receives bx, by of the residual, Jacobian and matvec; 0, 0
 * means the heuristic.  Results are unchanged bit for bit (every cell's
 * arithmetic is independent of the block shape).  The timing overwrites
 * the assembled Jacobian and preconditioner, which the next solve or
 * pfgpu_pc_setup rebuilds. */
int pfgpu_autotune(pfgpu_handle *h, int reps, int *shapes);

/* Residual F(p) without any device allocation, for callers that may not call
 * the CUDA allocator (a host framework with a fixed device-memory budget
 * reserved at start-up, or a latency-critical loop where cudaMalloc/cudaFree
 * would synchronise the device).  No handle: the per-cell van Genuchten
 * scratch lives in a static device array of the library (2^18 cells and 1024
 * layers at most; larger grids return PFGPU_ERR_ARG).  All vectors are DEVICE
 * pointers in dense interior layout (no ghost frame, x fastest,
 * c = i + nx*(j + ny*k)); perm is the one permeability array used for x, y
 * and z; vg_alpha, vg_n, s_res, s_sat are per-cell arrays or NULL for desc's
 * scalars; bc_type[6] lives on the host and bc_values[6] are device tables
 * laid out as for pfgpu_set_bc; only FluxConst (PFGPU_BC_FLUX) and Dirichlet
 * (PFGPU_BC_DIRICHLET) faces are accepted (no overland, seepage or terrain-
 * following terms), others return PFGPU_ERR_ARG.  Every pointer must be
 * memory of the current device (or managed memory).  Runs on the current
 * device and is ordered on `stream` (a cudaStream_t, NULL = legacy default
 * stream): f is ready when the stream reaches this point.  The first call on
 * a device resolves the scratch address (cudaGetSymbolAddress) and should
 * come before any stream capture; a cudaDeviceReset invalidates that address,
 * so do not call this again on a device that was reset.  Calls on one device
 * share the scratch, so calls that may overlap on the GPU race.  Host cost per
 * call: up to 15 cudaPointerGetAttributes checks and one small kernel per 64
 * layers (the layer constants) besides the two residual kernels.  Same
 * arithmetic as pfgpu_nl_function_eval.  No counterpart in the reference. */
int pfgpu_residual_noalloc(const pfgpu_desc *desc, const double *perm,
                           const double *vg_alpha, const double *vg_n,
                           const double *s_res, const double *s_sat,
                           const int *bc_type, const double *const *bc_values,
                           const double *p, const double *p_old, const double *s_old,
                           double dt, double *f, void *stream);

/* CUDA stream the handle launches on (a cudaStream_t as an opaque pointer),
 * so callers can order their own work. */
void *pfgpu_stream(pfgpu_handle *h);

/* Number of kernels this handle has launched so far. */
long long pfgpu_kernel_launches(pfgpu_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* PFGPU_H */
