/* Test infrastructure: link-time hooks for the reference build (oracle/ref.mk,
 * target parflow_hook; linked with ld --wrap, the reference sources are not
 * modified).  When the environment variable PFREF_DUMP_DIR names a directory,
 * each hooked call writes its operands there so that the C restatement in
 * oracle/ and the CUDA library can be checked against the reference function
 * by function on identical inputs:
 *
 *   fe_NNNNN.bin  KINSolFunctionEval (pfsimulator/parflow_lib/nl_function_eval.c:125)
 *                 p (before the call), f, saturation, density, old pressure,
 *                 old saturation, dt, time
 *   mv_NNNNN.bin  KINSolMatVec (pfsimulator/parflow_lib/richards_jacobian_eval.c:165)
 *                 x, y = J x, pressure, old pressure, recompute flag
 *   pc_NNNNN.bin  KinsolPC (pfsimulator/parflow_lib/kinsol_pc.c:58)
 *                 rhs before, rhs after (= M^-1 rhs)
 *   pj_NNNNN.bin  RichardsJacobianEval with symm_part set (the preconditioner
 *                 matrix, pfsimulator/parflow_lib/richards_jacobian_eval.c:217)
 *                 its stored coefficients C E N U (ghost frame included),
 *                 pressure, old pressure
 *
 * PFREF_DUMP_MAX (default 64) bounds the number of files per kind.
 *
 * File layout (little endian): char tag[8]; int32 nvec; double dt, time;
 * int32 recompute; then per vector: int32 nx, ny, nz (subvector extents with
 * the ghost frame), int32 ix, iy, iz (subvector origin), double data[nx*ny*nz].
 */
#include "parflow.h"
#include "kinsol_dependences.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void __real_KINSolFunctionEval(int size, N_Vector pressure, N_Vector fval,
                               void *current_state);
int __real_KINSolMatVec(void *current_state, N_Vector x, N_Vector y,
                        int *recompute, N_Vector pressure);
void __real_KinsolPC(Vector *rhs);
void __real_RichardsJacobianEval(Vector *pressure, Vector *old_pressure, Matrix **ptr_to_J,
                                 Matrix **ptr_to_JC, Vector *saturation, Vector *density,
                                 ProblemData *problem_data, double dt, double time,
                                 int symm_part);

static int counters[4];

static FILE *open_dump(int kind, const char *prefix)
{
  const char *dir = getenv("PFREF_DUMP_DIR");
  const char *mx = getenv("PFREF_DUMP_MAX");
  int limit = mx ? atoi(mx) : 64;
  char path[4096];

  if (!dir || counters[kind] >= limit)
    return NULL;
  snprintf(path, sizeof(path), "%s/%s_%05d.bin", dir, prefix, counters[kind]);
  counters[kind]++;
  return fopen(path, "wb");
}

static void put_header(FILE *fp, const char *tag, int nvec, double dt,
                       double time, int recompute)
{
  char t[8];

  memset(t, 0, sizeof(t));
  strncpy(t, tag, sizeof(t));
  fwrite(t, 1, sizeof(t), fp);
  fwrite(&nvec, sizeof(int), 1, fp);
  fwrite(&dt, sizeof(double), 1, fp);
  fwrite(&time, sizeof(double), 1, fp);
  fwrite(&recompute, sizeof(int), 1, fp);
}

static void put_vector(FILE *fp, Vector *v)
{
  Subvector *sv = VectorSubvector(v, 0);
  int hdr[6];

  hdr[0] = SubvectorNX(sv);
  hdr[1] = SubvectorNY(sv);
  hdr[2] = SubvectorNZ(sv);
  hdr[3] = SubvectorIX(sv);
  hdr[4] = SubvectorIY(sv);
  hdr[5] = SubvectorIZ(sv);
  fwrite(hdr, sizeof(int), 6, fp);
  fwrite(SubvectorData(sv), sizeof(double),
         (size_t)hdr[0] * hdr[1] * hdr[2], fp);
}

/* Copy of a vector's subvector data (ghost frame included). */
static double *snapshot(Vector *v, size_t *n)
{
  Subvector *sv = VectorSubvector(v, 0);
  size_t cnt = (size_t)SubvectorNX(sv) * SubvectorNY(sv) * SubvectorNZ(sv);
  double *buf = (double*)malloc(cnt * sizeof(double));

  memcpy(buf, SubvectorData(sv), cnt * sizeof(double));
  *n = cnt;
  return buf;
}

static void put_snapshot(FILE *fp, Vector *like, const double *buf, size_t n)
{
  Subvector *sv = VectorSubvector(like, 0);
  int hdr[6];

  hdr[0] = SubvectorNX(sv);
  hdr[1] = SubvectorNY(sv);
  hdr[2] = SubvectorNZ(sv);
  hdr[3] = SubvectorIX(sv);
  hdr[4] = SubvectorIY(sv);
  hdr[5] = SubvectorIZ(sv);
  fwrite(hdr, sizeof(int), 6, fp);
  fwrite(buf, sizeof(double), n, fp);
}

void __wrap_KINSolFunctionEval(int size, N_Vector pressure, N_Vector fval,
                               void *current_state)
{
  State *st = (State*)current_state;
  size_t n = 0;
  double *p_in = getenv("PFREF_DUMP_DIR") ? snapshot(pressure, &n) : NULL;

  __real_KINSolFunctionEval(size, pressure, fval, current_state);

  if (p_in)
  {
    FILE *fp = open_dump(0, "fe");
    if (fp)
    {
      put_header(fp, "FEVAL", 7, StateDt(st), StateTime(st), 0);
      put_snapshot(fp, pressure, p_in, n);
      put_vector(fp, fval);
      put_vector(fp, StateSaturation(st));
      put_vector(fp, StateDensity(st));
      put_vector(fp, StateOldPressure(st));
      put_vector(fp, StateOldSaturation(st));
      put_vector(fp, pressure);
      fclose(fp);
    }
    free(p_in);
  }
}

int __wrap_KINSolMatVec(void *current_state, N_Vector x, N_Vector y,
                        int *recompute, N_Vector pressure)
{
  State *st = (State*)current_state;
  int rc_in = *recompute;
  size_t n = 0;
  double *x_in = getenv("PFREF_DUMP_DIR") ? snapshot(x, &n) : NULL;
  int ret = __real_KINSolMatVec(current_state, x, y, recompute, pressure);

  if (x_in)
  {
    FILE *fp = open_dump(1, "mv");
    if (fp)
    {
      put_header(fp, "MATVEC", 4, StateDt(st), StateTime(st), rc_in);
      put_snapshot(fp, x, x_in, n);
      put_vector(fp, y);
      put_vector(fp, pressure);
      put_vector(fp, StateOldPressure(st));
      fclose(fp);
    }
    free(x_in);
  }
  return ret;
}

void __wrap_KinsolPC(Vector *rhs)
{
  size_t n = 0;
  double *r_in = getenv("PFREF_DUMP_DIR") ? snapshot(rhs, &n) : NULL;

  __real_KinsolPC(rhs);

  if (r_in)
  {
    FILE *fp = open_dump(2, "pc");
    if (fp)
    {
      put_header(fp, "PCAPPLY", 2, 0.0, 0.0, 0);
      put_snapshot(fp, rhs, r_in, n);
      put_vector(fp, rhs);
      fclose(fp);
    }
    free(r_in);
  }
}

/* One stencil coefficient of a matrix's only submatrix, as a dump vector. */
static void put_stencil(FILE *fp, Matrix *A, int s)
{
  Submatrix *sm = MatrixSubmatrix(A, 0);
  int hdr[6];

  hdr[0] = SubmatrixNX(sm);
  hdr[1] = SubmatrixNY(sm);
  hdr[2] = SubmatrixNZ(sm);
  hdr[3] = SubmatrixIX(sm);
  hdr[4] = SubmatrixIY(sm);
  hdr[5] = SubmatrixIZ(sm);
  fwrite(hdr, sizeof(int), 6, fp);
  fwrite(SubmatrixStencilData(sm, s), sizeof(double),
         (size_t)hdr[0] * hdr[1] * hdr[2], fp);
}

void __wrap_RichardsJacobianEval(Vector *pressure, Vector *old_pressure, Matrix **ptr_to_J,
                                 Matrix **ptr_to_JC, Vector *saturation, Vector *density,
                                 ProblemData *problem_data, double dt, double time,
                                 int symm_part)
{
  __real_RichardsJacobianEval(pressure, old_pressure, ptr_to_J, ptr_to_JC, saturation,
                              density, problem_data, dt, time, symm_part);
  if (symm_part && getenv("PFREF_DUMP_DIR"))
  {
    FILE *fp = open_dump(3, "pj");
    if (fp)
    {
      /* stencil order C W E S N L U; the stored (upper) ones are C E N U */
      static const int stored[4] = { 0, 2, 4, 6 };
      put_header(fp, "PCMAT", 6, dt, time, symm_part);
      for (int s = 0; s < 4; s++)
        put_stencil(fp, *ptr_to_J, stored[s]);
      put_vector(fp, pressure);
      put_vector(fp, old_pressure);
      fclose(fp);
    }
  }
}
