/* Test infrastructure: CPU restatement ("oracle") of ParFlow's Richards
 * Newton-Krylov inner loop for box domains.  Only tests/, the package's smoke
 * check and bench.py's CPU-baseline leg use it, as the checker; the product
 * path never calls it.
 *
 * Layout: interior-only, x fastest, idx = i + nx*(j + ny*k).  Boundary faces
 * are handled through the per-face boundary-condition tables, which is the
 * net effect of ParFlow's ghost-frame insertion / correction / reset sequence
 * (pfsimulator/parflow_lib/nl_function_eval.c:574-610, 979-1233, 2269-2311)
 * when the permeability ghost frame is zero, as it is for box domains.
 */
#ifndef PFORACLE_H
#define PFORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { PFO_BC_FLUX = 0, PFO_BC_DIRICHLET = 1, PFO_BC_OVERLAND_KIN = 2, PFO_BC_OVERLAND_DIFF = 3,
       PFO_BC_OVERLAND = 4, PFO_BC_SEEPAGE = 5 };

/* van Genuchten relative-permeability lookup table (VanGComputeTable,
 * problem_phase_rel_perm.c:116-262): kr and dkr/dhead at npts + 1 evenly
 * spaced heads 0 .. |min_head|, with monotone spline slopes (Fritsch and
 * Carlson) or linear slopes */
typedef struct {
  int method;                      /* InterpolationMethod: 0 Spline, 1 Linear */
  int npts;                        /* NumSamplePoints */
  double min_head, interval;
  double *x, *a, *d, *a_der, *d_der, *slope, *slope_der;
} pfo_vgtable;
pfo_vgtable *pfo_vgtable_create(int method, int npts, double min_head, double alpha, double n);
void pfo_vgtable_destroy(pfo_vgtable *t);

typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;
  double gravity, viscosity, density;
  const double *kx, *ky, *kz;      /* per cell */
  double porosity, sstorage;
  const double *alpha, *n;         /* per cell */
  const double *s_res, *s_sat;     /* per cell */
  int vg_from_file;                /* Saturation(p>=0): s_sat (1) or s_dif+s_res (0) */
  const double *z_mult;            /* per layer (nz) */
  int bc_type[6];                  /* x_lower x_upper y_lower y_upper z_lower z_upper */
  const double *bc_val[6];         /* face arrays: x:(nz,ny) y:(nz,nx) z:(ny,nx) */
  /* slopes (ny, nx): subsurface ones enter the x/y face gravity terms
   * (nl_function_eval.c:696-741; equal to the topographic ones under
   * Solver.TerrainFollowingGrid, solver_richards.c:562-572, else NULL = 0);
   * topographic ones and Manning's n drive the kinematic overland flow on an
   * OverlandKinematic z_upper patch (overlandflow_eval_Kin.c) */
  const double *sslope_x, *sslope_y;
  const double *tslope_x, *tslope_y;
  const double *mannings;
  double ov_epsilon;               /* Solver.Overland{Kinematic,Diffusive}.Epsilon */
  /* old pressure (interior layout) for the diffusive overland slope magnitude
   * in the Jacobian (overlandflow_eval_diffusive.c CALCDER); the residual
   * takes it as an argument */
  const double *ov_p_old;
  /* relative permeability from a lookup table instead of the closed form
   * (Geom.domain.RelPerm.NumSamplePoints > 0), or NULL */
  const pfo_vgtable *kr_table;
  /* land-surface sink/source per cell [1/h] (the evap_trans vector), or
   * NULL = 0 (nl_function_eval.c:533-541) */
  const double *evap_trans;
  /* flow-barrier multipliers of the faces between cell (i,j,k) and its +x /
   * +y / +z neighbour (Solver.Nonlinear.FlowBarrierX/Y/Z, problem_FBx.c), or
   * NULL = 1; nl_function_eval.c:841-843, richards_jacobian_eval.c:662-728 */
  const double *fbx, *fby, *fbz;
  /* OverlandFlowSpinUp (0 / 1) and OverlandSpinupDampP1 / P2 of an
   * OverlandFlow top patch (nl_function_eval.c:1659-1673,
   * richards_jacobian_eval.c:1258-1287, 2044-2057) */
  int ov_spinup;
  double ov_damp_p1, ov_damp_p2;
} pfo_problem;

typedef struct {
  double residual_tol, step_tol;
  int max_iter, krylov_dim, max_restarts;
  int eta_choice;                  /* 0 = constant, 1 = Walker1, 2 = Walker2 */
  double eta_value, eta_alpha, eta_gamma;
  int mg_max_levels;
  int mg_smoother;                 /* 0 = RBGS (symmetric), 1 = WJacobi */
  double wjacobi_weight;
  int use_jacobian;                /* Solver.Nonlinear.UseJacobian: 1 analytic J v,
                                    * 0 KINSOL's difference quotient */
  double derivative_epsilon;       /* Solver.Nonlinear.DerivativeEpsilon */
  int globalization;               /* Solver.Nonlinear.Globalization: 0 LineSearch,
                                    * 1 InexactNewton */
  int mg_max_iter;                 /* Solver.Linear.Preconditioner.MGSemi.MaxIter */
  int mg_max_min_n[3];             /* ...MGSemi.MaxMinNX / NY / NZ (0 counts as 1) */
  int pc_full;                     /* Solver.Linear.Preconditioner.PCMatrixType:
                                    * 1 FullJacobian, 0 the symmetric part
                                    * (PFSymmetric, SymmetricPart, Picard) */
} pfo_settings;

typedef struct {
  int status;                      /* KINSOL return: 1 ok, 0 initial guess ok, else failure */
  int nni, nli, nfe, nps, npe, nbcf, nbktrk, ncfl;
  double fnorm;
} pfo_stats;

/* van Genuchten (problem_saturation.c:221-415, problem_phase_rel_perm.c:567-1361) */
void pfo_saturation(const pfo_problem *pb, const double *p, double *s, int der);
void pfo_relperm(const pfo_problem *pb, const double *p, double *kr, int der);

/* face velocities and overland fluxes written by the residual evaluation
 * (nl_function_eval.c:846-848 interior faces, the BC loops' vel_vec for the
 * boundary faces, q_overlnd_x/y on an overland z_upper patch); dense, x
 * fastest: vx (nz, ny, nx+1) with face i between cells i-1 and i, vy
 * (nz, ny+1, nx), vz (nz+1, ny, nx), qx / qy (ny, nx).  Any may be NULL. */
typedef struct {
  double *vx, *vy, *vz, *qx, *qy;
} pfo_flux_out;
void pfo_residual_out(const pfo_problem *pb, double dt, const double *p,
                      const double *p_old, const double *s_old, double *f,
                      const pfo_flux_out *out);

/* residual F(p) at (dt, time-fixed BC tables) (nl_function_eval.c:167-2323) */
void pfo_residual(const pfo_problem *pb, double dt, const double *p,
                  const double *p_old, const double *s_old, double *f);

/* Jacobian: full 7 arrays C,W,E,S,N,L,U (symm=0) or the symmetric PC part
 * stored as C,E,N,U (symm=1), plus J[4] = the (ny*nz) W entries of the
 * i = 0 cells (symm=2) (richards_jacobian_eval.c:217-1420) */
void pfo_jacobian(const pfo_problem *pb, double dt, const double *p, int symm,
                  double *const *J);
/* the same; fd = 1 builds the matrix of Solver.Nonlinear.UseJacobian False
 * (no overland surface terms; richards_jacobian_eval.c:1241-1254, 1863,
 * 2476-2484) */
void pfo_jacobian_fd(const pfo_problem *pb, double dt, const double *p, int symm, int fd,
                     double *const *J);

/* y = J x for a full 7-array stencil matrix (matvec.c:35-330) */
void pfo_matvec7(const pfo_problem *pb, double *const *J, const double *x, double *y);

/* MGSemi preconditioner on a symmetric C,E,N,U level-0 matrix */
typedef struct pfo_mg pfo_mg;
pfo_mg *pfo_mg_create(const pfo_problem *pb, const pfo_settings *st);
void pfo_mg_setup(pfo_mg *mg, double *const *A4);
/* the same on the full non-symmetric C,W,E,S,N,L,U level-0 matrix
 * (PCMatrixType FullJacobian) */
void pfo_mg_setup_full(pfo_mg *mg, double *const *A7);
/* W entries (ny*nz) of the finest operator's i = 0 cells, or NULL for none;
 * read by the next pfo_mg_setup */
void pfo_mg_set_wghost(pfo_mg *mg, const double *wg);
void pfo_mg_apply(pfo_mg *mg, const double *b, double *x);
int pfo_mg_num_levels(const pfo_mg *mg);
void pfo_mg_level_info(const pfo_mg *mg, int l, int *nx, int *ny, int *nz, int *dir);
void pfo_mg_destroy(pfo_mg *mg);

/* One KINSOL solve (kinsol.c:690-910): p in = initial guess, p out = result. */
void pfo_newton_solve(const pfo_problem *pb, const pfo_settings *st, double dt,
                      const double *p_old, const double *s_old, double *p,
                      pfo_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
