/* ParFlow nonlinear-solver module on libpfgpu.
 *
 * This file is compiled against ParFlow's own headers and linked into an
 * unmodified ParFlow build (oracle/ref.mk, target parflow_gpu).  It replaces
 * the module behind Solver.NonlinearSolver KINSol (KinsolNonlinSolver,
 * pfsimulator/parflow_lib/kinsol_nonlin_solver.c:297-1030) when the input
 * database sets
 *
 *   Solver.Nonlinear.GPU            True            (default False)
 *   Solver.Nonlinear.GPU.Precision  FP64 | Mixed | Mixed16   (default FP64)
 *   Solver.Nonlinear.GPU.Device     CUDA device index (default 0)
 *
 * and otherwise hands every call to the reference's KINSol module.  The
 * solver registry (solver_richards.c:5490-5502) lists only KINSol, so the
 * hook is made at link time: the executable is linked with
 * --wrap=KinsolNonlinSolver{,InitInstanceXtra,FreeInstanceXtra,
 * NewPublicXtra,FreePublicXtra,SizeOfTempData}, which routes the PFModule
 * function pointers solver_richards.c takes to the __wrap_ functions below.
 *
 * Per timestep (NonlinSolverInvoke, parflow_proto.h:301) the module
 *   - builds the BCStruct of BCPressure at time t, as NlFunctionEval does
 *     (nl_function_eval.c:543), and hands each box face's type and values to
 *     pfgpu_set_bc;
 *   - uploads evap_trans (nl_function_eval.c:533-541);
 *   - solves with pfgpu_newton_solve (KINSol with line search, SPGMR and the
 *     semicoarsening multigrid preconditioner on the GPU, keyed MGSemi or
 *     PFMG): pressure in as the initial guess,
 *     out as the solution; old_pressure and old_saturation in;
 *   - writes the face velocities and q_overlnd_x / q_overlnd_y of the last
 *     residual evaluation (pfgpu_face_velocities) into the state vectors;
 *   - appends the step's counters to <run>.out.kinsol.log in KINSol's format
 *     (kinsol_nonlin_solver.c:266-290);
 *   - returns 0 on convergence, 1 otherwise (AdvanceRichards then halves dt,
 *     solver_richards.c:3390-3420).
 *
 * Supported problems are those of the library: one subgrid (one process), a
 * box domain whose six patches are x_lower x_upper y_lower y_upper z_lower
 * z_upper, constant density, porosity and specific storage, and van Genuchten
 * saturation and relative permeability with the same alpha and n (region
 * values or per-cell files) in one geometry.  Anything else stops the run
 * with a message, before any step. */
#include "parflow.h"
#include "pfgpu.h"

#include <math.h>
#include <string.h>

/* the reference's functions this file wraps */
int __real_KinsolNonlinSolver(Vector *pressure, Vector *density, Vector *old_density,
                              Vector *saturation, Vector *old_saturation, double t, double dt,
                              ProblemData *problem_data, Vector *old_pressure,
                              Vector *evap_trans, Vector *ovrl_bc_flx, Vector *x_velocity,
                              Vector *y_velocity, Vector *z_velocity, Vector *q_overlnd_x,
                              Vector *q_overlnd_y);
PFModule *__real_KinsolNonlinSolverInitInstanceXtra(Problem *problem, Grid *grid, Grid *grid2d,
                                                    ProblemData *problem_data,
                                                    double *temp_data);
void __real_KinsolNonlinSolverFreeInstanceXtra(void);
PFModule *__real_KinsolNonlinSolverNewPublicXtra(void);
void __real_KinsolNonlinSolverFreePublicXtra(void);
int __real_KinsolNonlinSolverSizeOfTempData(void);

typedef struct {
  int precision;   /* PFGPU_PREC_* */
  int device;
  pfgpu_desc desc; /* solver keys */
  int use_jacobian;
  double derivative_epsilon;
  int globalization; /* PFGPU_GLOBAL_* */
  int pc_matrix;     /* PFGPU_PCM_* */
  int mg_max_iter;   /* MGSemi.MaxIter */
} GpuPublicXtra;

typedef struct {
  Problem *problem;
  pfgpu_handle *h;
  FILE *log;
  int nx, ny, nz;
  double *face[6];  /* host face tables, (nz, ny) / (nz, nx) / (ny, nx) */
  double *zmult;
} GpuInstanceXtra;

/* the GPU module is chosen once per process, from the input database */
static int g_gpu = -1;

static int gpu_selected(void)
{
  if (g_gpu < 0)
  {
    NameArray na = NA_NewNameArray("False True");
    char *name = GetStringDefault("Solver.Nonlinear.GPU", "False");
    g_gpu = NA_NameToIndexExitOnError(na, name, "Solver.Nonlinear.GPU");
    NA_FreeNameArray(na);
  }
  return g_gpu == 1;
}

static void gpu_fail(const char *what)
{
  amps_Printf("Solver.Nonlinear.GPU: %s\n", what);
  PARFLOW_ERROR("Solver.Nonlinear.GPU: unsupported problem or library error");
}

/* the value of a uniform vector, or stop */
static double uniform_value(Vector *v, const char *what)
{
  Subvector *sv = VectorSubvector(v, 0);
  Subgrid *sg = GridSubgrid(VectorGrid(v), 0);
  int nx = SubgridNX(sg), ny = SubgridNY(sg), nz = SubgridNZ(sg);
  double *d = SubvectorData(sv);
  double v0 = d[SubvectorEltIndex(sv, SubgridIX(sg), SubgridIY(sg), SubgridIZ(sg))];
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (d[SubvectorEltIndex(sv, SubgridIX(sg) + i, SubgridIY(sg) + j, SubgridIZ(sg) + k)] != v0)
        {
          amps_Printf("Solver.Nonlinear.GPU: %s must be uniform\n", what);
          gpu_fail("non-uniform field");
        }
  return v0;
}

static int same_cells(Vector *a, Vector *b)
{
  Subvector *sa = VectorSubvector(a, 0), *sb = VectorSubvector(b, 0);
  Subgrid *sg = GridSubgrid(VectorGrid(a), 0);
  for (int k = 0; k < SubgridNZ(sg); k++)
    for (int j = 0; j < SubgridNY(sg); j++)
      for (int i = 0; i < SubgridNX(sg); i++)
      {
        int x = SubgridIX(sg) + i, y = SubgridIY(sg) + j, z = SubgridIZ(sg) + k;
        if (SubvectorData(sa)[SubvectorEltIndex(sa, x, y, z)] !=
            SubvectorData(sb)[SubvectorEltIndex(sb, x, y, z)])
          return 0;
      }
  return 1;
}

/* a per-cell van Genuchten field read the way problem_saturation.c:943-950
 * reads it, or NULL when the key names no file */
static Vector *read_cell_file(Grid *grid, const char *key)
{
  char *fname = GetStringDefault((char*)key, "");
  if (!fname[0])
    return NULL;
  Vector *v = NewVectorType(grid, 1, 1, vector_cell_centered);
  InitVectorAll(v, 0.0);
  ReadPFBinary(fname, v);
  return v;
}

/* ---- module functions ------------------------------------------------------ */

PFModule *__wrap_KinsolNonlinSolverNewPublicXtra(void)
{
  if (!gpu_selected())
    return __real_KinsolNonlinSolverNewPublicXtra();
  PFModule *this_module = ThisPFModule;
  GpuPublicXtra *px = ctalloc(GpuPublicXtra, 1);
  px->mg_max_iter = 1;
  pfgpu_desc *d = &px->desc;
  NameArray na;
  char *name;

  /* KinsolNonlinSolverNewPublicXtra's keys and defaults
   * (kinsol_nonlin_solver.c:766-930) */
  d->residual_tol = GetDoubleDefault("Solver.Nonlinear.ResidualTol", 1e-7);
  d->step_tol = GetDoubleDefault("Solver.Nonlinear.StepTol", 1e-7);
  d->max_iter = GetIntDefault("Solver.Nonlinear.MaxIter", 15);
  d->krylov_dim = GetIntDefault("Solver.Linear.KrylovDimension", 10);
  d->max_restarts = GetIntDefault("Solver.Linear.MaxRestarts", 0);
  na = NA_NewNameArray("EtaConstant Walker1 Walker2");
  name = GetStringDefault("Solver.Nonlinear.EtaChoice", "Walker2");
  d->eta_choice = NA_NameToIndexExitOnError(na, name, "Solver.Nonlinear.EtaChoice");
  NA_FreeNameArray(na);
  d->eta_value = GetDoubleDefault("Solver.Nonlinear.EtaValue", 1e-4);
  d->eta_alpha = GetDoubleDefault("Solver.Nonlinear.EtaAlpha", 2.0);
  d->eta_gamma = GetDoubleDefault("Solver.Nonlinear.EtaGamma", 0.9);
  na = NA_NewNameArray("False True");
  name = GetStringDefault("Solver.Nonlinear.UseJacobian", "False");
  px->use_jacobian = NA_NameToIndexExitOnError(na, name, "Solver.Nonlinear.UseJacobian");
  NA_FreeNameArray(na);
  px->derivative_epsilon = GetDoubleDefault("Solver.Nonlinear.DerivativeEpsilon", 1e-7);
  na = NA_NewNameArray("InexactNewton LineSearch");
  name = GetStringDefault("Solver.Nonlinear.Globalization", "LineSearch");
  px->globalization =
      NA_NameToIndexExitOnError(na, name, "Solver.Nonlinear.Globalization") == 0
          ? PFGPU_GLOBAL_INEXACT_NEWTON
          : PFGPU_GLOBAL_LINE_SEARCH;
  NA_FreeNameArray(na);
  na = NA_NewNameArray("NoPC MGSemi SMG PFMG PFMGOctree");
  name = GetStringDefault("Solver.Linear.Preconditioner", "MGSemi");
  const int pc = NA_NameToIndexExitOnError(na, name, "Solver.Linear.Preconditioner");
  NA_FreeNameArray(na);
  if (pc != 1 && pc != 3)
    gpu_fail("only Solver.Linear.Preconditioner MGSemi or PFMG is available");
  /* KinsolPC's matrix type (kinsol_pc.c:215-246) and MGSemi's keys
   * (mg_semi.c:1230-1310, rb_GS_point.c:440-470, w_jacobi.c:385-395) */
  /* PFSymmetric, SymmetricPart and Picard give the same matrix: the
   * Jacobian evaluation tests its symm_part argument only for zero
   * (richards_jacobian_eval.c:760, 781, 2246) */
  na = NA_NewNameArray("FullJacobian PFSymmetric SymmetricPart Picard");
  name = GetStringDefault("Solver.Linear.Preconditioner.PCMatrixType", "PFSymmetric");
  px->pc_matrix =
    NA_NameToIndexExitOnError(na, name, "Solver.Linear.Preconditioner.PCMatrixType") == 0
    ? PFGPU_PCM_FULL : PFGPU_PCM_SYMMETRIC;
  NA_FreeNameArray(na);
  if (pc == 3)
  {
    /* PFMG (pf_pfmg.c:285-330) on the semicoarsening multigrid: one pre-
     * and one post-relaxation of its smoother per cycle, MaxIter cycles
     * (KinsolPC's tolerance 0 stops hypre on the count alone) */
    px->mg_max_iter = GetIntDefault("Solver.Linear.Preconditioner.PFMG.MaxIter", 1);
    if (GetIntDefault("Solver.Linear.Preconditioner.PFMG.NumPreRelax", 1) != 1 ||
        GetIntDefault("Solver.Linear.Preconditioner.PFMG.NumPostRelax", 1) != 1)
      gpu_fail("PFMG with NumPreRelax and NumPostRelax 1 only");
    na = NA_NewNameArray("Jacobi WJacobi RBGaussSeidelSymmetric RBGaussSeidelNonSymmetric");
    name = GetStringDefault("Solver.Linear.Preconditioner.PFMG.Smoother",
                            "RBGaussSeidelNonSymmetric");
    const int sm = NA_NameToIndexExitOnError(na, name,
                                             "Solver.Linear.Preconditioner.PFMG.Smoother");
    NA_FreeNameArray(na);
    if (sm == 1)
      gpu_fail("PFMG smoother WJacobi is not available");
    d->mg_smoother = sm == 0 ? PFGPU_SMOOTH_WJACOBI : sm == 2 ? PFGPU_SMOOTH_RBGS
                     : PFGPU_SMOOTH_RBGS_NONSYM;
    d->wjacobi_weight = 1.0;
    d->mg_max_levels = 100;
  }
  else
  {
    px->mg_max_iter = GetIntDefault("Solver.Linear.Preconditioner.MGSemi.MaxIter", 1);
    d->mg_max_levels = GetIntDefault("Solver.Linear.Preconditioner.MGSemi.MaxLevels", 100);
    d->mg_max_min_n[0] = GetIntDefault("Solver.Linear.Preconditioner.MGSemi.MaxMinNX", 1);
    d->mg_max_min_n[1] = GetIntDefault("Solver.Linear.Preconditioner.MGSemi.MaxMinNY", 1);
    d->mg_max_min_n[2] = GetIntDefault("Solver.Linear.Preconditioner.MGSemi.MaxMinNZ", 1);
    na = NA_NewNameArray("RedBlackGSPoint WJacobi");
    name = GetStringDefault("Solver.Linear.Preconditioner.MGSemi.Smoother", "RedBlackGSPoint");
    const int smoother =
        NA_NameToIndexExitOnError(na, name, "Solver.Linear.Preconditioner.MGSemi.Smoother");
    NA_FreeNameArray(na);
    if (smoother == 0)
    {
      na = NA_NewNameArray("True False");
      name = GetStringDefault("Solver.Linear.Preconditioner.MGSemi.Smoother.Symmetric", "True");
      const int sym = NA_NameToIndexExitOnError(
          na, name, "Solver.Linear.Preconditioner.MGSemi.Smoother.Symmetric");
      NA_FreeNameArray(na);
      d->mg_smoother = sym == 0 ? PFGPU_SMOOTH_RBGS : PFGPU_SMOOTH_RBGS_NONSYM;
    }
    else
    {
      d->mg_smoother = PFGPU_SMOOTH_WJACOBI;
    }
    d->wjacobi_weight =
        GetDoubleDefault("Solver.Linear.Preconditioner.MGSemi.Smoother.Weight", 1.0);
    /* one smoothing iteration and the default coarse solve, one symmetric
     * red/black Gauss-Seidel iteration (rb_GS_point.c:449-470,
     * mg_semi.c:1281-1310) */
    if (GetIntDefault("Solver.Linear.Preconditioner.MGSemi.Smoother.MaxIter", 1) != 1)
      gpu_fail("only MGSemi.Smoother.MaxIter 1 is available");
    if (strcmp(GetStringDefault("Solver.Linear.Preconditioner.MGSemi.CoarseSolve",
                                "RedBlackGSPoint"), "RedBlackGSPoint") != 0 ||
        GetIntDefault("Solver.Linear.Preconditioner.MGSemi.CoarseSolve.MaxIter", 1) != 1 ||
        strcmp(GetStringDefault("Solver.Linear.Preconditioner.MGSemi.CoarseSolve.Symmetric",
                                "True"), "True") != 0)
      gpu_fail("only the default MGSemi.CoarseSolve (RedBlackGSPoint, MaxIter 1, "
               "Symmetric True) is available");
  }
  na = NA_NewNameArray("FP64 Mixed Mixed16");
  name = GetStringDefault("Solver.Nonlinear.GPU.Precision", "FP64");
  int prec = NA_NameToIndexExitOnError(na, name, "Solver.Nonlinear.GPU.Precision");
  NA_FreeNameArray(na);
  px->precision = prec == 0 ? PFGPU_PREC_FP64 : prec == 1 ? PFGPU_PREC_MIXED : PFGPU_PREC_MIXED_H16;
  px->device = GetIntDefault("Solver.Nonlinear.GPU.Device", 0);
  PFModulePublicXtra(this_module) = px;
  return this_module;
}

void __wrap_KinsolNonlinSolverFreePublicXtra(void)
{
  if (!gpu_selected())
  {
    __real_KinsolNonlinSolverFreePublicXtra();
    return;
  }
  GpuPublicXtra *px = (GpuPublicXtra*)PFModulePublicXtra(ThisPFModule);
  if (px)
    tfree(px);
}

int __wrap_KinsolNonlinSolverSizeOfTempData(void)
{
  if (!gpu_selected())
    return __real_KinsolNonlinSolverSizeOfTempData();
  return 0;
}

PFModule *__wrap_KinsolNonlinSolverInitInstanceXtra(Problem *problem, Grid *grid, Grid *grid2d,
                                                    ProblemData *problem_data,
                                                    double *temp_data)
{
  if (!gpu_selected())
    return __real_KinsolNonlinSolverInitInstanceXtra(problem, grid, grid2d, problem_data,
                                                     temp_data);
  PFModule *this_module = ThisPFModule;
  GpuInstanceXtra *ix = (GpuInstanceXtra*)PFModuleInstanceXtra(this_module);
  (void)grid2d;
  (void)problem_data;
  (void)temp_data;
  if (ix == NULL)
  {
    ix = ctalloc(GpuInstanceXtra, 1);
    char filename[2048];
    sprintf(filename, "%s.%s", GlobalsOutFileName, "kinsol.log");
    if (!amps_Rank(amps_CommWorld))
      ix->log = fopen(filename, "w");
  }
  if (problem != NULL)
    ix->problem = problem;
  if (grid != NULL && GridNumSubgrids(grid) != 1)
    gpu_fail("one subgrid (one process) per run");
  PFModuleInstanceXtra(this_module) = ix;
  return this_module;
}

void __wrap_KinsolNonlinSolverFreeInstanceXtra(void)
{
  if (!gpu_selected())
  {
    __real_KinsolNonlinSolverFreeInstanceXtra();
    return;
  }
  GpuInstanceXtra *ix = (GpuInstanceXtra*)PFModuleInstanceXtra(ThisPFModule);
  if (!ix)
    return;
  if (ix->h)
    pfgpu_destroy(ix->h);
  if (ix->log)
    fclose(ix->log);
  for (int f = 0; f < 6; f++)
    tfree(ix->face[f]);
  tfree(ix->zmult);
  tfree(ix);
}

/* the handle, made at the first solve: ProblemData is complete only then */
static void create_handle(GpuInstanceXtra *ix, GpuPublicXtra *px, Vector *pressure,
                          Vector *density, ProblemData *pd)
{
  Problem *problem = ix->problem;
  Grid *grid = VectorGrid(pressure);
  Subgrid *sg = GridSubgrid(grid, 0);
  pfgpu_desc d = px->desc;
  d.abi_version = PFGPU_ABI_VERSION;
  d.nx = SubgridNX(sg);
  d.ny = SubgridNY(sg);
  d.nz = SubgridNZ(sg);
  d.dx = SubgridDX(sg);
  d.dy = SubgridDY(sg);
  d.dz = SubgridDZ(sg);
  d.gravity = ProblemGravity(problem);
  d.viscosity = ProblemPhaseViscosity(problem, 0);
  d.density = uniform_value(density, "the phase density (Phase.<name>.Density.Type Constant)");
  d.porosity = uniform_value(ProblemDataPorosity(pd), "porosity");
  d.specific_storage = uniform_value(ProblemDataSpecificStorage(pd), "specific storage");
  d.precision = px->precision;
  ix->nx = d.nx;
  ix->ny = d.ny;
  ix->nz = d.nz;

  /* dz multipliers per layer: every column must carry the same ones */
  Vector *zm = ProblemDataZmult(pd);
  Subvector *zs = VectorSubvector(zm, 0);
  ix->zmult = ctalloc(double, d.nz);
  for (int k = 0; k < d.nz; k++)
  {
    double v = SubvectorData(zs)[SubvectorEltIndex(zs, SubgridIX(sg), SubgridIY(sg), SubgridIZ(sg) + k)];
    ix->zmult[k] = v;
    for (int j = 0; j < d.ny; j++)
      for (int i = 0; i < d.nx; i++)
        if (SubvectorData(zs)[SubvectorEltIndex(zs, SubgridIX(sg) + i, SubgridIY(sg) + j,
                                                SubgridIZ(sg) + k)] != v)
          gpu_fail("dz multipliers must be the same in every column");
  }
  d.z_mult = ix->zmult;

  /* van Genuchten keys (problem_saturation.c:900-1010,
   * problem_phase_rel_perm.c:1880-1960): one geometry, equal saturation
   * and relative-permeability parameters */
  if (strcmp(GetString("Phase.Saturation.Type"), "VanGenuchten") != 0 ||
      strcmp(GetString("Phase.RelPerm.Type"), "VanGenuchten") != 0)
    gpu_fail("Phase.Saturation.Type and Phase.RelPerm.Type VanGenuchten");
  char *gs = GetString("Phase.Saturation.GeomNames");
  char *gr = GetString("Phase.RelPerm.GeomNames");
  if (strchr(gs, ' ') || strcmp(gs, gr) != 0)
    gpu_fail("one geometry for the saturation and relative-permeability parameters");
  char key[IDB_MAX_KEY_LEN];
  int s_file = GetIntDefault("Phase.Saturation.VanGenuchten.File", 0);
  int r_file = GetIntDefault("Phase.RelPerm.VanGenuchten.File", 0);
  if (s_file != r_file)
    gpu_fail("Phase.Saturation and Phase.RelPerm VanGenuchten.File must agree");
  sprintf(key, "Geom.%s.Saturation.Alpha", gs);
  d.vg_alpha = GetDouble(key);
  sprintf(key, "Geom.%s.Saturation.N", gs);
  d.vg_n = GetDouble(key);
  sprintf(key, "Geom.%s.Saturation.SRes", gs);
  d.s_res = GetDouble(key);
  sprintf(key, "Geom.%s.Saturation.SSat", gs);
  d.s_sat = GetDouble(key);
  d.vg_from_file = s_file;
  if (!s_file)
  {
    double ra, rn;
    sprintf(key, "Geom.%s.RelPerm.Alpha", gs);
    ra = GetDouble(key);
    sprintf(key, "Geom.%s.RelPerm.N", gs);
    rn = GetDouble(key);
    if (ra != d.vg_alpha || rn != d.vg_n)
      gpu_fail("saturation and relative-permeability alpha and n must be equal");
  }

  ix->h = pfgpu_create(&d, px->device);
  if (!ix->h)
    gpu_fail(pfgpu_last_error());
  if (!px->use_jacobian &&
      pfgpu_set_jacobian_mode(ix->h, 0, px->derivative_epsilon) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());
  if (pfgpu_set_globalization(ix->h, px->globalization) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());
  if (pfgpu_set_pc_matrix(ix->h, px->pc_matrix) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());
  if (pfgpu_set_mg_max_iter(ix->h, px->mg_max_iter) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());

  /* permeability: x, and y / z where they differ from x */
  Vector *kx = ProblemDataPermeabilityX(pd), *ky = ProblemDataPermeabilityY(pd),
         *kz = ProblemDataPermeabilityZ(pd);
  if (pfgpu_set_field(ix->h, PFGPU_FIELD_PERM_X, SubvectorData(VectorSubvector(kx, 0))))
    gpu_fail(pfgpu_last_error());
  if (!same_cells(kx, ky) &&
      pfgpu_set_field(ix->h, PFGPU_FIELD_PERM_Y, SubvectorData(VectorSubvector(ky, 0))))
    gpu_fail(pfgpu_last_error());
  if (!same_cells(kx, kz) &&
      pfgpu_set_field(ix->h, PFGPU_FIELD_PERM_Z, SubvectorData(VectorSubvector(kz, 0))))
    gpu_fail(pfgpu_last_error());

  /* flow barriers (problem_FBx.c etc.: 1 everywhere unless the key is on) */
  {
    static const char *const fkey[3] = {"Solver.Nonlinear.FlowBarrierX",
                                        "Solver.Nonlinear.FlowBarrierY",
                                        "Solver.Nonlinear.FlowBarrierZ"};
    Vector *fb[3] = {ProblemDataFBx(pd), ProblemDataFBy(pd), ProblemDataFBz(pd)};
    for (int q = 0; q < 3; q++)
    {
      NameArray fna = NA_NewNameArray("False True");
      const int on = NA_NameToIndexExitOnError(fna, GetStringDefault(fkey[q], "False"), fkey[q]);
      NA_FreeNameArray(fna);
      if (on && pfgpu_set_field(ix->h, PFGPU_FIELD_FB_X + q,
                                SubvectorData(VectorSubvector(fb[q], 0))) != PFGPU_OK)
        gpu_fail(pfgpu_last_error());
    }
  }

  /* per-cell van Genuchten files */
  if (s_file)
  {
    static const char *const skey[4] = {"Alpha", "N", "SRes", "SSat"};
    static const int field[4] = {PFGPU_FIELD_VG_ALPHA, PFGPU_FIELD_VG_N, PFGPU_FIELD_S_RES,
                                 PFGPU_FIELD_S_SAT};
    Vector *sv[4];
    for (int q = 0; q < 4; q++)
    {
      sprintf(key, "Geom.%s.Saturation.%s.Filename", gs, skey[q]);
      sv[q] = read_cell_file(grid, key);
      if (!sv[q])
        gpu_fail("VanGenuchten.File needs every Saturation.*.Filename");
      if (pfgpu_set_field(ix->h, field[q], SubvectorData(VectorSubvector(sv[q], 0))))
        gpu_fail(pfgpu_last_error());
    }
    for (int q = 0; q < 2; q++)
    {
      sprintf(key, "Geom.%s.RelPerm.%s.Filename", gs, skey[q]);
      Vector *rv = read_cell_file(grid, key);
      if (!rv || !same_cells(rv, sv[q]))
        gpu_fail("relative-permeability alpha and n files must equal the saturation ones");
      FreeVector(rv);
    }
    for (int q = 0; q < 4; q++)
      FreeVector(sv[q]);
  }
  else
  {
    /* relative-permeability lookup table (problem_phase_rel_perm.c:1894-1916) */
    sprintf(key, "Geom.%s.RelPerm.NumSamplePoints", gs);
    int npts = GetIntDefault(key, 0);
    if (npts > 0)
    {
      sprintf(key, "Geom.%s.RelPerm.MinPressureHead", gs);
      double minh = GetDouble(key);
      sprintf(key, "Geom.%s.RelPerm.InterpolationMethod", gs);
      NameArray na = NA_NewNameArray("Spline Linear");
      int method = NA_NameToIndexExitOnError(na, GetStringDefault(key, "Spline"), key);
      NA_FreeNameArray(na);
      if (pfgpu_set_relperm_table(ix->h, method == 0 ? 1 : 2, npts, minh) != PFGPU_OK)
        gpu_fail(pfgpu_last_error());
    }
  }

  /* surface data for the overland patch types and the terrain-following
   * grid: the 2-D vectors' data plane (one ghost layer in z as well) */
  int tfg = 0;
  {
    NameArray na = NA_NewNameArray("False True");
    tfg = NA_NameToIndexExitOnError(na, GetStringDefault("Solver.TerrainFollowingGrid", "False"),
                                    "Solver.TerrainFollowingGrid");
    NA_FreeNameArray(na);
  }
  int overland = BCPressurePackageUsingOverlandFlow(problem);
  if (tfg || overland)
  {
    long plane = (long)(d.nx + 2) * (d.ny + 2);
    double *sx = SubvectorData(VectorSubvector(ProblemDataTSlopeX(pd), 0)) + plane;
    double *sy = SubvectorData(VectorSubvector(ProblemDataTSlopeY(pd), 0)) + plane;
    double *mn = SubvectorData(VectorSubvector(ProblemDataMannings(pd), 0)) + plane;
    double eps = GetDoubleDefault("Solver.OverlandKinematic.Epsilon", 1e-5);
    if (pfgpu_set_surface(ix->h, sx, sy, mn, tfg, eps) != PFGPU_OK)
      gpu_fail(pfgpu_last_error());
  }
  /* OverlandFlowSpinUp and its damping (nl_function_eval.c:313, 2474-2477) */
  if (pfgpu_set_overland_spinup(ix->h, GetIntDefault("OverlandFlowSpinUp", 0),
                                GetDoubleDefault("OverlandSpinupDampP1", 0.0),
                                GetDoubleDefault("OverlandSpinupDampP2", 0.0)) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());
  ix->face[0] = ctalloc(double, (long)d.nz * d.ny);
  ix->face[1] = ctalloc(double, (long)d.nz * d.ny);
  ix->face[2] = ctalloc(double, (long)d.nz * d.nx);
  ix->face[3] = ctalloc(double, (long)d.nz * d.nx);
  ix->face[4] = ctalloc(double, (long)d.ny * d.nx);
  ix->face[5] = ctalloc(double, (long)d.ny * d.nx);
}

/* BCPressure at time t (nl_function_eval.c:543-544) into the six face
 * tables; each patch cell lands on the face its direction names */
static void upload_bcs(GpuInstanceXtra *ix, Problem *problem, ProblemData *pd, Grid *grid,
                       double t)
{
  PFModule *bc_pressure =
    PFModuleNewInstanceType(BCPressurePackageInitInstanceXtraInvoke,
                            ProblemBCPressure(problem), (problem));
  BCStruct *bc = PFModuleInvokeType(BCPressureInvoke, bc_pressure,
                                    (pd, grid, ProblemDataGrDomain(pd), t));
  int type[6] = {-1, -1, -1, -1, -1, -1};
  int ipatch, is = 0, i, j, k, ival;
  int *fdir;
  ForBCStructNumPatches(ipatch, bc)
  {
    double *values = BCStructPatchValues(bc, ipatch, is);
    int t_lib;
    switch (BCStructBCType(bc, ipatch))
    {
      case DirichletBC: t_lib = PFGPU_BC_DIRICHLET; break;
      case FluxBC: t_lib = PFGPU_BC_FLUX; break;
      case OverlandBC: t_lib = PFGPU_BC_OVERLAND; break;
      case SeepageFaceBC: t_lib = PFGPU_BC_SEEPAGE; break;
      case OverlandKinematicBC: t_lib = PFGPU_BC_OVERLAND_KIN; break;
      case OverlandDiffusiveBC: t_lib = PFGPU_BC_OVERLAND_DIFF; break;
      default: gpu_fail("unknown boundary condition type"); t_lib = -1;
    }
    BCStructPatchLoop(i, j, k, fdir, ival, bc, ipatch, is,
    {
      int face = fdir[0] ? (fdir[0] < 0 ? 0 : 1)
                 : fdir[1] ? (fdir[1] < 0 ? 2 : 3) : (fdir[2] < 0 ? 4 : 5);
      if (type[face] >= 0 && type[face] != t_lib)
        gpu_fail("one boundary condition type per box face");
      type[face] = t_lib;
      long slot = face < 2 ? j + (long)ix->ny * k : face < 4 ? i + (long)ix->nx * k
                  : i + (long)ix->nx * j;
      ix->face[face][slot] = values[ival];
    });
  }
  for (int f = 0; f < 6; f++)
  {
    if (type[f] < 0)
      gpu_fail("every box face needs a boundary patch");
    if (pfgpu_set_bc(ix->h, f, type[f], ix->face[f]) != PFGPU_OK)
      gpu_fail(pfgpu_last_error());
  }
  FreeBCStruct(bc);
  PFModuleFreeInstance(bc_pressure);
}

int __wrap_KinsolNonlinSolver(Vector *pressure, Vector *density, Vector *old_density,
                              Vector *saturation, Vector *old_saturation, double t, double dt,
                              ProblemData *problem_data, Vector *old_pressure,
                              Vector *evap_trans, Vector *ovrl_bc_flx, Vector *x_velocity,
                              Vector *y_velocity, Vector *z_velocity, Vector *q_overlnd_x,
                              Vector *q_overlnd_y)
{
  if (!gpu_selected())
    return __real_KinsolNonlinSolver(pressure, density, old_density, saturation,
                                     old_saturation, t, dt, problem_data, old_pressure,
                                     evap_trans, ovrl_bc_flx, x_velocity, y_velocity,
                                     z_velocity, q_overlnd_x, q_overlnd_y);
  PFModule *this_module = ThisPFModule;
  GpuPublicXtra *px = (GpuPublicXtra*)PFModulePublicXtra(this_module);
  GpuInstanceXtra *ix = (GpuInstanceXtra*)PFModuleInstanceXtra(this_module);
  (void)old_density;
  (void)saturation;
  (void)ovrl_bc_flx;  /* not read by the residual (nl_function_eval.c:178) */
  if (!ix->h)
    create_handle(ix, px, pressure, density, problem_data);
  if (ix->log)
    fprintf(ix->log, "\nKINSOL starting step for time %f\n", t);
  upload_bcs(ix, ix->problem, problem_data, VectorGrid(pressure), t);
  if (pfgpu_set_evap_trans(ix->h, SubvectorData(VectorSubvector(evap_trans, 0))) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());
  /* the old pressure of the step also enters the diffusive overland terms */
  if (pfgpu_set_old_pressure(ix->h, SubvectorData(VectorSubvector(old_pressure, 0))) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());

  pfgpu_stats st;
  memset(&st, 0, sizeof(st));
  double *p = SubvectorData(VectorSubvector(pressure, 0));
  int rc = pfgpu_newton_solve(ix->h, SubvectorData(VectorSubvector(old_pressure, 0)),
                              SubvectorData(VectorSubvector(old_saturation, 0)), dt, p, &st);
  if (rc < 0)
    gpu_fail(pfgpu_last_error());

  /* the velocities of the last residual evaluation, as the state holds them */
  double *q[2] = {q_overlnd_x ? SubvectorData(VectorSubvector(q_overlnd_x, 0)) : NULL,
                  q_overlnd_y ? SubvectorData(VectorSubvector(q_overlnd_y, 0)) : NULL};
  if (pfgpu_face_velocities(ix->h, NULL, NULL, NULL, dt,
                            SubvectorData(VectorSubvector(x_velocity, 0)),
                            SubvectorData(VectorSubvector(y_velocity, 0)),
                            SubvectorData(VectorSubvector(z_velocity, 0)), q[0], q[1]) != PFGPU_OK)
    gpu_fail(pfgpu_last_error());

  if (ix->log)
  {
    /* PrintFinalStats (kinsol_nonlin_solver.c:266-290): this step and the
     * running totals */
    static long tot[8];
    long now[8] = {st.nonlin_iters, st.lin_iters, st.fevals, st.pc_setups, st.pc_solves,
                   st.lin_conv_fails, st.beta_cond_fails, st.backtracks};
    static const char *const label[8] = {"Nonlin. Its.:    ", "Lin. Its.:       ",
                                         "Func. Evals.:    ", "PC Evals.:       ",
                                         "PC Solves:       ", "Lin. Conv. Fails:",
                                         "Beta Cond. Fails:", "Backtracks:      "};
    fprintf(ix->log, "\n-------------------------------------------------- \n");
    fprintf(ix->log, "                    Iteration             Total\n");
    for (int q2 = 0; q2 < 8; q2++)
    {
      tot[q2] += now[q2];
      fprintf(ix->log, "%s       %5ld             %5ld\n", label[q2], now[q2], tot[q2]);
    }
    fprintf(ix->log, "-------------------------------------------------- \n");
    fflush(ix->log);
  }
  return rc == PFGPU_OK ? 0 : 1;
}
