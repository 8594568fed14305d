/* Test infrastructure: CPU restatement of ParFlow's Richards Newton-Krylov
 * inner loop (box domains).  Used only as the checker by tests/, the smoke
 * check and bench.py's CPU-baseline leg.  Each function cites the reference
 * code it restates; paths are relative to the ParFlow source tree
 * (PL = pfsimulator/parflow_lib, KS = pfsimulator/kinsol).
 */
#include "pforacle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k) ((i) + nx * ((j) + ny * (k)))
#define HARMONIC(a, b) (((a) + (b)) ? (2.0 * (a) * (b)) / ((a) + (b)) : 0.0)      /* PL/solver.h:44 */
#define HARMONIC_DZ(a, b, c, d) ((((c) * (b)) + ((a) * (d))) ?                   \
                                 ((((c) + (d)) * (a) * (b)) / (((b) * (c)) + ((a) * (d)))) : 0.0) /* PL/solver.h:46 */
#define UPSTREAM(a, b, c, d) ((((a) - (b)) >= 0) ? (c) : (d))                    /* PL/solver.h:47 */
#define AMEAN(a, b) (0.5 * ((a) + (b)))                                          /* PL/solver.h:42 */

/* -------------------------------------------------------------------------
 * van Genuchten
 * ------------------------------------------------------------------------- */

/* PL/problem_saturation.c:221-415 */
static double vg_sat(double p, double rho, double g, double alpha, double n,
                     double s_res, double s_sat, int from_file)
{
  double m = 1.0e0 - (1.0e0 / n);
  double s_dif = s_sat - s_res;
  if (p >= 0.0)
    return from_file ? s_sat : s_dif + s_res;
  double head = fabs(p) / (rho * g);
  return s_dif / pow(1.0 + pow((alpha * head), n), m) + s_res;
}

static double vg_dsat(double p, double rho, double g, double alpha, double n,
                      double s_res, double s_sat)
{
  double m = 1.0e0 - (1.0e0 / n);
  double s_dif = s_sat - s_res;
  if (p >= 0.0)
    return 0.0;
  double head = fabs(p) / (rho * g);
  return (m * n * alpha * pow(alpha * head, (n - 1))) * s_dif
         / (pow(1.0 + pow(alpha * head, n), m + 1));
}

/* PL/problem_phase_rel_perm.c:788 (function) and :981 (derivative) */
static double vg_kr(double p, double rho, double g, double alpha, double n)
{
  if (p >= 0.0)
    return 1.0;
  double m = 1.0e0 - (1.0e0 / n);
  double head = fabs(p) / (rho * g);
  double opahn = 1.0 + pow(alpha * head, n);
  double ahnm1 = pow(alpha * head, n - 1);
  return pow(1.0 - ahnm1 / (pow(opahn, m)), 2) / pow(opahn, (m / 2));
}

static double vg_dkr(double p, double rho, double g, double alpha, double n)
{
  if (p >= 0.0)
    return 0.0;
  double m = 1.0e0 - (1.0e0 / n);
  double head = fabs(p) / (rho * g);
  double opahn = 1.0 + pow(alpha * head, n);
  double ahnm1 = pow(alpha * head, n - 1);
  double coeff = 1.0 - ahnm1 * pow(opahn, -m);
  return 2.0 * (coeff / (pow(opahn, (m / 2))))
         * ((n - 1) * pow(alpha * head, n - 2) * alpha * pow(opahn, -m)
            - ahnm1 * m * pow(opahn, -(m + 1)) * n * alpha * ahnm1)
         + pow(coeff, 2) * (m / 2) * pow(opahn, (-(m + 2) / 2)) * n * alpha * ahnm1;
}

void pfo_saturation(const pfo_problem *pb, const double *p, double *s, int der)
{
  long N = (long)pb->nx * pb->ny * pb->nz;
  for (long c = 0; c < N; c++)
    s[c] = der ? vg_dsat(p[c], pb->density, pb->gravity, pb->alpha[c], pb->n[c],
                         pb->s_res[c], pb->s_sat[c])
               : vg_sat(p[c], pb->density, pb->gravity, pb->alpha[c], pb->n[c],
                        pb->s_res[c], pb->s_sat[c], pb->vg_from_file);
}

/* VanGComputeTable (problem_phase_rel_perm.c:116-262) */
pfo_vgtable *pfo_vgtable_create(int method, int npts, double min_head, double alpha, double n)
{
  pfo_vgtable *t = (pfo_vgtable*)calloc(1, sizeof(pfo_vgtable));
  t->method = method;
  t->npts = npts;
  t->min_head = min_head;
  double **arr[] = { &t->x, &t->a, &t->d, &t->a_der, &t->d_der, &t->slope, &t->slope_der };
  for (int q = 0; q < 7; q++)
    *arr[q] = (double*)calloc(npts + 1, sizeof(double));
  double *x = t->x, *a = t->a, *d = t->d, *a_der = t->a_der, *d_der = t->d_der;
  double *del = (double*)calloc(npts + 1, sizeof(double));
  double *del_der = (double*)calloc(npts + 1, sizeof(double));
  double interval = min_head / (double)(npts - 1);
  t->interval = fabs(interval);
  double m = 1.0e0 - (1.0e0 / n);
  for (int i = 0; i <= npts; i++)
  {
    x[i] = fabs(i * interval);
    double opahn = 1.0 + pow(alpha * x[i], n);
    double ahnm1 = pow(alpha * x[i], n - 1);
    a[i] = pow(1.0 - ahnm1 / (pow(opahn, m)), 2) / pow(opahn, (m / 2));
    double coeff = 1.0 - ahnm1 * pow(opahn, -m);
    a_der[i] = 2.0 * (coeff / (pow(opahn, (m / 2))))
               * ((n - 1) * pow(alpha * x[i], n - 2) * alpha * pow(opahn, -m)
                  - ahnm1 * m * pow(opahn, -(m + 1)) * n * alpha * ahnm1)
               + pow(coeff, 2) * (m / 2) * pow(opahn, (-(m + 2) / 2)) * n * alpha * ahnm1;
    if ((n < 2) && (i == 0))
      a_der[i] = 0;
  }
  if (method == 1)
    for (int i = 0; i < npts; i++)
    {
      t->slope[i] = (a[i + 1] - a[i]) / t->interval;
      t->slope_der[i] = (a_der[i + 1] - a_der[i]) / t->interval;
    }
  /* monotone cubic Hermite slopes (Fritsch and Carlson 1980) */
  for (int i = 0; i < npts; i++)
  {
    double h = x[i + 1] - x[i];
    del[i] = (a[i + 1] - a[i]) / h;
    del_der[i] = (a_der[i + 1] - a_der[i]) / h;
  }
  d[0] = del[0];
  d[npts] = del[npts - 1];
  d_der[0] = del_der[0];
  d_der[npts] = del_der[npts - 1];
  for (int i = 1; i < npts; i++)
  {
    d[i] = (del[i - 1] + del[i]) / 2;
    d_der[i] = (del_der[i - 1] + del_der[i]) / 2;
  }
  for (int i = 0; i < npts; i++)
  {
    if (del[i] == 0.0)
    {
      d[i] = 0;
      d[i + 1] = 0;
    }
    else
    {
      double alph = d[i] / del[i], beta = d[i + 1] / del[i];
      double magn = pow(alph, 2) + pow(beta, 2);
      if (magn > 9.0)
      {
        d[i] = 3 * alph * del[i] / magn;
        d[i + 1] = 3 * beta * del[i] / magn;
      }
    }
    if (del_der[i] == 0.0)
    {
      d_der[i] = 0;
      d_der[i + 1] = 0;
    }
    else
    {
      double alph = d_der[i] / del_der[i], beta = d_der[i + 1] / del_der[i];
      double magn = pow(alph, 2) + pow(beta, 2);
      if (magn > 9.0)
      {
        d_der[i] = 3 * alph * del_der[i] / magn;
        d_der[i + 1] = 3 * beta * del_der[i] / magn;
      }
    }
  }
  free(del);
  free(del_der);
  return t;
}

void pfo_vgtable_destroy(pfo_vgtable *t)
{
  if (!t) return;
  free(t->x); free(t->a); free(t->d); free(t->a_der); free(t->d_der);
  free(t->slope); free(t->slope_der);
  free(t);
}

/* VanGLookupSpline (:265-355) and the linear lookup (:357-400, and inline in
 * PhaseRelPerm :718-758): kr (der = 0) or the table's derivative (der = 1)
 * at a pressure head >= 0 */
static double vgt_lookup(const pfo_vgtable *t, double head, int der)
{
  if (head >= fabs(t->min_head))
    return 0.0;
  int pt = (int)floor(head / t->interval);
  if (t->method == 1)
    return der ? t->a_der[pt] + t->slope_der[pt] * (head - t->x[pt])
               : t->a[pt] + t->slope[pt] * (head - t->x[pt]);
  int max = t->npts + 1;
  if (pt > max)
    pt = max - 1;
  const double *A = der ? t->a_der : t->a, *D = der ? t->d_der : t->d;
  double x = t->x[pt], x1 = t->x[pt + 1];
  double tt = (head - x) / (x1 - x);
  return (2.0 * pow(tt, 3) - 3.0 * pow(tt, 2) + 1.0) * A[pt]
         + (pow(tt, 3) - 2.0 * pow(tt, 2) + tt) * (x1 - x) * D[pt]
         + (-2.0 * pow(tt, 3) + 3.0 * pow(tt, 2)) * (A[pt + 1])
         + (pow(tt, 3) - pow(tt, 2)) * (x1 - x) * (D[pt + 1]);
}

/* rel. perm. (der = 0) or its derivative (der = 1) at pressure p of a cell
 * with VG parameters alpha, n: the table when one is set (:700-712,
 * 1064-1080, 1170-1184), else the closed form */
static double kr_at(const pfo_problem *pb, double p, double alpha, double n, int der)
{
  if (pb->kr_table)
  {
    if (p >= 0.0)
      return der ? 0.0 : 1.0;
    return vgt_lookup(pb->kr_table, fabs(p) / (pb->density * pb->gravity), der);
  }
  return der ? vg_dkr(p, pb->density, pb->gravity, alpha, n)
             : vg_kr(p, pb->density, pb->gravity, alpha, n);
}

void pfo_relperm(const pfo_problem *pb, const double *p, double *kr, int der)
{
  long N = (long)pb->nx * pb->ny * pb->nz;
  for (long c = 0; c < N; c++)
    kr[c] = kr_at(pb, p[c], pb->alpha[c], pb->n[c], der);
}

/* -------------------------------------------------------------------------
 * Boundary faces
 * ------------------------------------------------------------------------- */

/* Face f of cell (i,j,k) lies on the domain boundary; returns the index into
 * the face's value table. */
static int face_index(const pfo_problem *pb, int f, int i, int j, int k)
{
  int nx = pb->nx, ny = pb->ny;
  (void)nx;
  switch (f)
  {
    case 0: case 1: return j + ny * k;     /* (nz, ny) */
    case 2: case 3: return i + pb->nx * k; /* (nz, nx) */
    default: return i + pb->nx * j;        /* (ny, nx) */
  }
}

static int on_face(const pfo_problem *pb, int f, int i, int j, int k)
{
  switch (f)
  {
    case 0: return i == 0;
    case 1: return i == pb->nx - 1;
    case 2: return j == 0;
    case 3: return j == pb->ny - 1;
    case 4: return k == 0;
    default: return k == pb->nz - 1;
  }
}

/* -------------------------------------------------------------------------
 * Terrain-following face gravity terms (PL/nl_function_eval.c:725-733,
 * SlopeUpwindFormulation "Original"): the mean over the two columns of
 * g sin(atan S) and g cos(atan S); zero slopes give 0 and g.
 * ------------------------------------------------------------------------- */
static double slope_at(const double *s, int nx, int ny, int i, int j)
{
  /* beyond the last column or row: the slope vector's zero ghost frame */
  if (!s || i >= nx || j >= ny) return 0.0;
  return s[i + nx * j];
}

static void tfg_x(const pfo_problem *pb, int i, int j, double *g_s, double *g_c)
{
  const double g = pb->gravity;
  double a = slope_at(pb->sslope_x, pb->nx, pb->ny, i, j);
  double b = slope_at(pb->sslope_x, pb->nx, pb->ny, i + 1, j);
  *g_s = AMEAN(g * sin(atan(a)), g * sin(atan(b)));
  *g_c = AMEAN(g * cos(atan(a)), g * cos(atan(b)));
}

static void tfg_y(const pfo_problem *pb, int i, int j, double *g_s, double *g_c)
{
  const double g = pb->gravity;
  double a = slope_at(pb->sslope_y, pb->nx, pb->ny, i, j);
  double b = slope_at(pb->sslope_y, pb->nx, pb->ny, i, j + 1);
  *g_s = AMEAN(g * sin(atan(a)), g * sin(atan(b)));
  *g_c = AMEAN(g * cos(atan(a)), g * cos(atan(b)));
}

/* -------------------------------------------------------------------------
 * Kinematic overland flow on the top layer (PL/overlandflow_eval_Kin.c).
 * 2-D arrays carry ParFlow's one-cell ghost frame: io = (i+1) + (j+1)*(nx+2).
 * The domain top index is nz-1 in every column and -1 in the ghost frame
 * (compute_top_and_bottom.c:69); the patch-index vector is all zero, so the
 * internal patch-edge fixes never apply; the pressure beyond the upper x / y
 * edge is a ghost value that is never positive, so it enters as 0.
 * ------------------------------------------------------------------------- */
#define PFMAX(a, b) (((a) < (b)) ? (b) : (a))

static void ovl_common(const pfo_problem *pb, const double *p, int i, int j,
                       double *sfx, double *sfy, double *sqm, double *px, double *py)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz;
  const long top = (long)nx * ny * (nz - 1);
  double Sf_x = pb->tslope_x[i + nx * j], Sf_y = pb->tslope_y[i + nx * j];
  double Sf_mag = pow(Sf_x * Sf_x + Sf_y * Sf_y, 0.5);
  if (Sf_mag < pb->ov_epsilon) Sf_mag = pb->ov_epsilon;
  double pp_ip = p[top + i + nx * j];
  double pp_e = (i + 1 < nx) ? p[top + i + 1 + nx * j] : 0.0;
  double pp_n = (j + 1 < ny) ? p[top + i + nx * (j + 1)] : 0.0;
  *sfx = Sf_x;
  *sfy = Sf_y;
  *sqm = pow(fabs(Sf_mag), 0.5);
  *px = UPSTREAM(-Sf_x, 0.0, PFMAX(pp_ip, 0.0), PFMAX(pp_e, 0.0));
  *py = UPSTREAM(-Sf_y, 0.0, PFMAX(pp_ip, 0.0), PFMAX(pp_n, 0.0));
}

/* CALCFCN (:120-290): ke, kw, kn, ks per top cell, ghost-framed */
static void ovl_fcn(const pfo_problem *pb, const double *p, double *ke, double *kw,
                    double *kn, double *ks)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz, sy = nx + 2;
  const long n2 = (long)(nx + 2) * (ny + 2);
  const long top = (long)nx * ny * (nz - 1);
  double *qx = (double*)calloc(n2, sizeof(double));
  double *qy = (double*)calloc(n2, sizeof(double));
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      double n_man = pb->mannings[i + nx * j];
      double Sf_x, Sf_y, sq, Px, Py;
      ovl_common(pb, p, i, j, &Sf_x, &Sf_y, &sq, &Px, &Py);
      qx[io] = -(Sf_x / (sq * n_man)) * pow(Px, (5.0 / 3.0));
      qy[io] = -(Sf_y / (sq * n_man)) * pow(Py, (5.0 / 3.0));
      double pown = PFMAX(p[top + i + nx * j], 0.0);
      if (i == 0 && Sf_x > 0.0)   /* lower x boundary */
        qx[io - 1] = -(Sf_x / (sq * n_man)) * pow(pown, (5.0 / 3.0));
      if (j == 0 && Sf_y > 0.0)   /* lower y boundary */
        qy[io - sy] = -(Sf_y / (sq * n_man)) * pow(pown, (5.0 / 3.0));
    }
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      ke[io] = qx[io];
      kw[io] = qx[io - 1];
      kn[io] = qy[io];
      ks[io] = qy[io - sy];
    }
  free(qx);
  free(qy);
}

/* CALCDER (:293-460): derivative terms, written into neighbouring entries */
static void ovl_der(const pfo_problem *pb, const double *p, double *ke, double *kw,
                    double *kn, double *ks)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz, sy = nx + 2;
  const long top = (long)nx * ny * (nz - 1);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      double n_man = pb->mannings[i + nx * j];
      double Sf_x, Sf_y, sq, Px, Py;
      ovl_common(pb, p, i, j, &Sf_x, &Sf_y, &sq, &Px, &Py);
      double qx_temp = -(5.0 / 3.0) * (Sf_x / (sq * n_man)) * pow(Px, (2.0 / 3.0));
      double qy_temp = -(5.0 / 3.0) * (Sf_y / (sq * n_man)) * pow(Py, (2.0 / 3.0));
      ke[io] = PFMAX(qx_temp, 0);
      kw[io + 1] = -PFMAX(-qx_temp, 0);
      kn[io] = PFMAX(qy_temp, 0);
      ks[io + sy] = -PFMAX(-qy_temp, 0);
      double pown = PFMAX(p[top + i + nx * j], 0.0);
      if (i == 0 && Sf_x > 0.0)
      {
        qx_temp = -(5.0 / 3.0) * (Sf_x / (sq * n_man)) * pow(pown, (2.0 / 3.0));
        kw[io] = -PFMAX(-qx_temp, 0);
        ke[io - 1] = PFMAX(qx_temp, 0);
      }
      if (j == 0 && Sf_y > 0.0)
      {
        qy_temp = -(5.0 / 3.0) * (Sf_y / (sq * n_man)) * pow(pown, (2.0 / 3.0));
        ks[io] = -PFMAX(-qy_temp, 0);
        kn[io - sy] = PFMAX(qy_temp, 0);
      }
    }
}

/* -------------------------------------------------------------------------
 * Overland flow of the OverlandFlow patch type (PL/overlandflow_eval.c):
 * each column's kinematic flux q = dir(S) |S|^(1/2) / n max(p, 0)^(5/3)
 * along the sign of its own slope, upwinded between neighbouring columns;
 * columns outside the domain (top index -1) carry no flux.
 * ------------------------------------------------------------------------- */
static double ovf_dir(double s)
{
  return (s > 0.0) ? -1.0 : (s < 0.0) ? 1.0 : 0.0;
}

/* q of column (i, j) along x (ax = 1) or y (ax = 0); 0 outside the domain */
static double ovf_q(const pfo_problem *pb, const double *p, int i, int j, int ax)
{
  if (i < 0 || j < 0 || i >= pb->nx || j >= pb->ny)
    return 0.0;
  const long a = i + (long)pb->nx * j;
  const double s = ax ? pb->tslope_x[a] : pb->tslope_y[a];
  const double pt = p[(long)pb->nx * pb->ny * (pb->nz - 1) + a];
  return ovf_dir(s) * (pow(fabs(s), 0.5) / pb->mannings[a]) * pow(PFMAX(pt, 0.0), (5.0 / 3.0));
}

/* CALCFCN (:104-250): ke, kw, kn, ks of every top cell */
static void ovf_fcn(const pfo_problem *pb, const double *p, double *ke, double *kw, double *kn,
                    double *ks)
{
  const int nx = pb->nx, ny = pb->ny, sy = nx + 2;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      double q0 = ovf_q(pb, p, i - 1, j, 1), q1 = ovf_q(pb, p, i, j, 1),
             q2 = ovf_q(pb, p, i + 1, j, 1);
      kw[io] = PFMAX(q0, 0.0) - PFMAX(-q1, 0.0);
      ke[io] = PFMAX(q1, 0.0) - PFMAX(-q2, 0.0);
      q0 = ovf_q(pb, p, i, j - 1, 0);
      q1 = ovf_q(pb, p, i, j, 0);
      q2 = ovf_q(pb, p, i, j + 1, 0);
      ks[io] = PFMAX(q0, 0.0) - PFMAX(-q1, 0.0);
      kn[io] = PFMAX(q1, 0.0) - PFMAX(-q2, 0.0);
    }
}

/* CALCDER (:251-330): derivative terms of each column's own flux */
static void ovf_der(const pfo_problem *pb, const double *p, double *ke, double *kw, double *kn,
                    double *ks)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz, sy = nx + 2;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      long a = i + (long)nx * j;
      double pt = p[(long)nx * ny * (nz - 1) + a];
      double sx = pb->tslope_x[a], syv = pb->tslope_y[a], n = pb->mannings[a];
      double q_mid = ovf_dir(sx) * (5.0 / 3.0) * (pow(fabs(sx), 0.5) / n)
                     * pow(PFMAX(pt, 0.0), (2.0 / 3.0));
      kw[io] = -PFMAX(-q_mid, 0.0);
      ke[io] = PFMAX(q_mid, 0.0);
      q_mid = ovf_dir(syv) * (5.0 / 3.0) * (pow(fabs(syv), 0.5) / n)
              * pow(PFMAX(pt, 0.0), (2.0 / 3.0));
      ks[io] = -PFMAX(-q_mid, 0.0);
      kn[io] = PFMAX(q_mid, 0.0);
    }
}

/* -------------------------------------------------------------------------
 * Diffusive overland flow on the top layer (PL/overlandflow_eval_diffusive.c).
 * The friction slope adds the ponded-depth gradient to the topographic slope;
 * its magnitude comes from the old pressure.  Box conventions as for the
 * kinematic form: top = nz-1 in every column, -1 in the ghost frame, and the
 * (never positive) ghost pressure beyond the upper x / y edges enters as 0.
 * ------------------------------------------------------------------------- */
static double ptop0(const pfo_problem *pb, const double *p, int i, int j)
{
  if (i >= pb->nx || j >= pb->ny)
    return 0.0;
  return PFMAX(p[(long)pb->nx * pb->ny * (pb->nz - 1) + i + (long)pb->nx * j], 0.0);
}

/* CALCFCN (:125-250): q_x, q_y per column, then ke/kw/kn/ks gathered */
static void ovd_fcn(const pfo_problem *pb, const double *p, const double *op, double *ke,
                    double *kw, double *kn, double *ks)
{
  const int nx = pb->nx, ny = pb->ny, sy = nx + 2;
  const long n2 = (long)(nx + 2) * (ny + 2);
  const double dx = pb->dx, dy = pb->dy, eps = pb->ov_epsilon;
  double *qx = (double*)calloc(n2, sizeof(double));
  double *qy = (double*)calloc(n2, sizeof(double));
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      const double sxv = pb->tslope_x[i + nx * j], syv = pb->tslope_y[i + nx * j];
      const double n_man = pb->mannings[i + nx * j];
      double Pupx = ptop0(pb, p, i + 1, j), Pupy = ptop0(pb, p, i, j + 1);
      double Pupox = ptop0(pb, op, i + 1, j), Pupoy = ptop0(pb, op, i, j + 1);
      double Pdown = ptop0(pb, p, i, j), Pdowno = ptop0(pb, op, i, j);
      double Sf_x = sxv + (Pupx - Pdown) / dx;
      double Sf_y = syv + (Pupy - Pdown) / dy;
      double Sf_xo = sxv + (Pupox - Pdowno) / dx;
      double Sf_yo = syv + (Pupoy - Pdowno) / dy;
      double Sf_mag = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
      if (Sf_mag < eps) Sf_mag = eps;
      double Press_x = UPSTREAM(-Sf_x, 0.0, Pdown, Pupx);
      double Press_y = UPSTREAM(-Sf_y, 0.0, Pdown, Pupy);
      qx[io] = -(Sf_x / (pow(fabs(Sf_mag), 0.5) * n_man)) * pow(Press_x, (5.0 / 3.0));
      qy[io] = -(Sf_y / (pow(fabs(Sf_mag), 0.5) * n_man)) * pow(Press_y, (5.0 / 3.0));
      if (i == 0)   /* lower x boundary :179-195 */
      {
        Press_x = Pdown;
        Sf_x = sxv + (Press_x - 0.0) / dx;
        Pupox = Pdowno;
        Sf_xo = sxv + (Pupox - 0.0) / dx;
        double m = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
        if (m < eps) m = eps;
        if (Sf_x > 0.0)
          qx[io - 1] = -(Sf_x / (pow(fabs(m), 0.5) * n_man)) * pow(Press_x, (5.0 / 3.0));
      }
      if (j == 0)   /* lower y boundary :197-228 (its y differences divide by dx) */
      {
        Press_y = Pdown;
        Sf_y = syv + (Press_y - 0.0) / dx;
        Pupoy = Pdowno;
        Sf_yo = syv + (Pupoy - 0.0) / dx;
        double m = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
        if (m < eps) m = eps;
        if (Sf_y > 0.0)
          qy[io - sy] = -(Sf_y / (pow(fabs(m), 0.5) * n_man)) * pow(Press_y, (5.0 / 3.0));
        if (i == 0 && Sf_x > 0.0)   /* corner: q_x again with this magnitude */
          qx[io - 1] = -(Sf_x / (pow(fabs(m), 0.5) * n_man)) * pow(Press_x, (5.0 / 3.0));
      }
    }
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      ke[io] = qx[io];
      kw[io] = qx[io - 1];
      kn[io] = qy[io];
      ks[io] = qy[io - sy];
    }
  free(qx);
  free(qy);
}

/* CALCDER (:252-455): symmetric (ke kw kn ks) and non-symmetric (…ns)
 * derivative terms, written into this and neighbouring columns' entries */
static void ovd_der(const pfo_problem *pb, const double *p, const double *op, double *ke,
                    double *kw, double *kn, double *ks, double *kens, double *kwns,
                    double *knns, double *ksns)
{
  const int nx = pb->nx, ny = pb->ny, sy = nx + 2;
  const double dx = pb->dx, dy = pb->dy, eps = pb->ov_epsilon;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
    {
      long io = (i + 1) + (long)sy * (j + 1);
      const double sxv = pb->tslope_x[i + nx * j], syv = pb->tslope_y[i + nx * j];
      const double n_man = pb->mannings[i + nx * j];
      double Pupx = ptop0(pb, p, i + 1, j), Pupy = ptop0(pb, p, i, j + 1);
      double Pupox = ptop0(pb, op, i + 1, j), Pupoy = ptop0(pb, op, i, j + 1);
      double Pdown = ptop0(pb, p, i, j), Pdowno = ptop0(pb, op, i, j);
      double Sf_x = sxv + (Pupx - Pdown) / dx;
      double Sf_y = syv + (Pupy - Pdown) / dy;
      double Sf_xo = sxv + (Pupox - Pdowno) / dx;
      double Sf_yo = syv + (Pupoy - Pdowno) / dy;
      double Sf_mag = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
      if (Sf_mag < eps) Sf_mag = eps;
      double sq = pow(fabs(Sf_mag), 0.5);
      if (Sf_x < 0)
      {
        ke[io] = (5.0 / 3.0) * (-sxv - (Pupx / dx)) / (sq * n_man) * pow(Pdown, (2.0 / 3.0)) +
                 (8.0 / 3.0) * pow(Pdown, (5.0 / 3.0)) / (sq * n_man * dx);
        kw[io + 1] = -pow(Pdown, (5.0 / 3.0)) / (sq * n_man * dx);
        kens[io] = kw[io + 1];
        kwns[io + 1] = ke[io];
      }
      if (Sf_x >= 0)
      {
        ke[io] = pow(Pupx, (5.0 / 3.0)) / (sq * n_man * dx);
        kw[io + 1] = (5.0 / 3.0) * (-sxv + (Pdown / dx)) / (sq * n_man) * pow(Pupx, (2.0 / 3.0)) -
                     (8.0 / 3.0) * pow(Pupx, (5.0 / 3.0)) / (sq * n_man * dx);
        kens[io] = kw[io + 1];
        kwns[io + 1] = ke[io];
      }
      if (Sf_y < 0)
      {
        kn[io] = (5.0 / 3.0) * (-syv - (Pupy / dy)) / (sq * n_man) * pow(Pdown, (2.0 / 3.0)) +
                 (8.0 / 3.0) * pow(Pdown, (5.0 / 3.0)) / (sq * n_man * dy);
        ks[io + sy] = -pow(Pdown, (5.0 / 3.0)) / (sq * n_man * dy);
        knns[io] = ks[io + sy];
        ksns[io + sy] = kn[io];
      }
      if (Sf_y >= 0)
      {
        kn[io] = pow(Pupy, (5.0 / 3.0)) / (sq * n_man * dy);
        ks[io + sy] = (5.0 / 3.0) * (-syv + (Pdown / dy)) / (sq * n_man) * pow(Pupy, (2.0 / 3.0)) -
                      (8.0 / 3.0) * pow(Pupy, (5.0 / 3.0)) / (sq * n_man * dy);
        knns[io] = ks[io + sy];
        ksns[io + sy] = kn[io];
      }
      if (i == 0)   /* lower x boundary :343-372 */
      {
        Pupx = Pdown;
        Sf_x = sxv + (Pupx - 0.0) / dx;
        Pupox = Pdowno;
        Sf_xo = sxv + (Pupox - 0.0) / dx;
        double m = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
        if (m < eps) m = eps;
        double sm = pow(fabs(m), 0.5);
        if (Sf_x < 0)
        {
          ke[io - 1] = 0.0;
          kw[io] = 0.0;
          kwns[io] = 0.0;
          kens[io - 1] = 0.0;
        }
        if (Sf_x >= 0)
        {
          ke[io - 1] = pow(Pupx, (5.0 / 3.0)) / (sm * n_man * dx);
          kw[io] = (5.0 / 3.0) * (-sxv + 0.0) / (sm * n_man) * pow(Pupx, (2.0 / 3.0)) -
                   (8.0 / 3.0) * pow(Pupx, (5.0 / 3.0)) / (sm * n_man * dx);
          kens[io - 1] = kw[io];
          kwns[io] = ke[io - 1];
        }
      }
      if (j == 0)   /* lower y boundary :374-421 */
      {
        Pupy = Pdown;
        Sf_y = syv + (Pupy - 0.0) / dy;
        Pupoy = Pdowno;
        Sf_yo = syv + (Pupoy - 0.0) / dy;
        double m = pow(Sf_xo * Sf_xo + Sf_yo * Sf_yo, 0.5);
        if (m < eps) m = eps;
        double sm = pow(fabs(m), 0.5);
        if (Sf_y < 0)
        {
          kn[io - sy] = 0.0;
          ks[io] = 0.0;
          ksns[io] = 0.0;
          knns[io - sy] = 0.0;
        }
        if (Sf_y >= 0)
        {
          knns[io - sy] = pow(Pupy, (5.0 / 3.0)) / (sm * n_man * dy);
          ks[io] = (5.0 / 3.0) * (-syv + 0.0) / (sm * n_man) * pow(Pupy, (2.0 / 3.0)) -
                   (8.0 / 3.0) * pow(Pupy, (5.0 / 3.0)) / (sm * n_man * dy);
          knns[io - sy] = ks[io];
          ksns[io] = kn[io - sy];
        }
        if (i == 0)   /* corner (:404-420): the x terms again with this magnitude */
        {
          if (Sf_x < 0)
          {
            kn[io - sy] = 0.0;
            ks[io] = 0.0;
            ksns[io] = 0.0;
            knns[io - sy] = 0.0;
          }
          if (Sf_x >= 0)
          {
            ke[io - 1] = pow(Pupx, (5.0 / 3.0)) / (sm * n_man * dx);
            kw[io] = (5.0 / 3.0) * (-sxv + 0.0) / (sm * n_man) * pow(Pupx, (2.0 / 3.0)) -
                     (8.0 / 3.0) * pow(Pupx, (5.0 / 3.0)) / (sm * n_man * dx);
            kens[io - 1] = kw[io];
            kwns[io] = ke[io - 1];
          }
        }
      }
    }
}

/* -------------------------------------------------------------------------
 * Residual  (PL/nl_function_eval.c:167-2323)
 * ------------------------------------------------------------------------- */
void pfo_residual(const pfo_problem *pb, double dt, const double *p,
                  const double *p_old, const double *s_old, double *f)
{
  pfo_residual_out(pb, dt, p, p_old, s_old, f, NULL);
}

void pfo_residual_out(const pfo_problem *pb, double dt, const double *p,
                      const double *p_old, const double *s_old, double *f,
                      const pfo_flux_out *out)
{
  static const pfo_flux_out none = {NULL, NULL, NULL, NULL, NULL};
  if (!out)
    out = &none;
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz;
  const long N = (long)nx * ny * nz;
  const double dx = pb->dx, dy = pb->dy, dz = pb->dz;
  const double g = pb->gravity, visc = pb->viscosity, rho = pb->density;
  const double vol = dx * dy * dz;
  const double ffx = dy * dz, ffy = dx * dz, ffz = dx * dy;
  const double *zm = pb->z_mult;
  double *sat = (double*)malloc(N * sizeof(double));
  double *kr = (double*)malloc(N * sizeof(double));

  pfo_saturation(pb, p, sat, 0);
  pfo_relperm(pb, p, kr, 0);

  /* accumulation :394-405 and compressible storage :462-472 */
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        f[c] = (sat[c] * rho - s_old[c] * rho) * pb->porosity * vol * 1.0 * 1.0 * zm[k];
        f[c] += pb->sstorage * vol * 1.0 * 1.0 * zm[k]
                * (p[c] * sat[c] * rho - p_old[c] * s_old[c] * rho);
        /* sources: PhaseSources (0 here) plus the evap_trans sink (:533-541) */
        f[c] -= vol * 1.0 * 1.0 * zm[k] * dt * (0.0 + (pb->evap_trans ? pb->evap_trans[c] : 0.0));
      }

  /* interior faces :696-854, gravity terms from the subsurface slopes */
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        double u_right = 0.0, u_front = 0.0, u_upper = 0.0;
        double x_dir_g, x_dir_g_c, y_dir_g, y_dir_g_c;
        tfg_x(pb, i, j, &x_dir_g, &x_dir_g_c);
        tfg_y(pb, i, j, &y_dir_g, &y_dir_g_c);
        if (i + 1 < nx)
        {
          long e = c + 1;
          double diff_l = p[c] - p[e];
          double updir = (diff_l / dx) * x_dir_g_c - x_dir_g;
          double km = HARMONIC(pb->kx[c], pb->kx[e]);
          double up = UPSTREAM(updir, 0.0, kr[c] * rho, kr[e] * rho);
          u_right = zm[k] * ffx * 1.0 * km * (diff_l / (dx * 1.0)) * x_dir_g_c * up / visc;
          u_right += zm[k] * ffx * 1.0 * km * (-x_dir_g) * up / visc;
        }
        if (j + 1 < ny)
        {
          long n = c + nx;
          double diff_l = p[c] - p[n];
          double updir = (diff_l / dy) * y_dir_g_c - y_dir_g;
          double km = HARMONIC(pb->ky[c], pb->ky[n]);
          double up = UPSTREAM(updir, 0.0, kr[c] * rho, kr[n] * rho);
          u_front = zm[k] * ffy * 1.0 * km * (diff_l / (dy * 1.0)) * y_dir_g_c * up / visc;
          u_front += zm[k] * ffy * 1.0 * km * (-y_dir_g) * up / visc;
        }
        if (k + 1 < nz)
        {
          long u = c + (long)nx * ny;
          double zc = zm[k], zu = zm[k + 1];
          double sep = dz * AMEAN(zc, zu);
          double lower = p[c] / sep - (zc / (zc + zu)) * rho * g * 1.0;
          double upper = p[u] / sep + (zu / (zc + zu)) * rho * g * 1.0;
          double diff_l = lower - upper;
          u_upper = ffz * 1.0 * 1.0 * HARMONIC_DZ(pb->kz[c], pb->kz[u], zc, zu) * diff_l
                    * UPSTREAM(lower, upper, kr[c] * rho, kr[u] * rho) / visc;
        }
        /* flow barriers :841-843, then the face velocities :845-848; the
         * boundary faces are written by the patch loops below */
        if (pb->fbx) u_right = u_right * pb->fbx[c];
        if (pb->fby) u_front = u_front * pb->fby[c];
        if (pb->fbz) u_upper = u_upper * pb->fbz[c];
        if (out->vx && i + 1 < nx)
          out->vx[(i + 1) + (long)(nx + 1) * (j + (long)ny * k)] = u_right / (ffx * zm[k] * 1.0);
        if (out->vy && j + 1 < ny)
          out->vy[i + (long)nx * ((j + 1) + (long)(ny + 1) * k)] = u_front / (ffy * zm[k] * 1.0);
        if (out->vz && k + 1 < nz)
          out->vz[c + (long)nx * ny] = u_upper / (ffz * 1.0 * 1.0);
        f[c] += dt * (u_right + u_front + u_upper);
        if (i + 1 < nx) f[c + 1] += -dt * u_right;
        if (j + 1 < ny) f[c + nx] += -dt * u_front;
        if (k + 1 < nz) f[c + (long)nx * ny] += -dt * u_upper;
      }

  /* boundary patches :979-2060, in patch order */
  double *ke = NULL, *kw = NULL, *kn = NULL, *ks = NULL;
  for (int face = 0; face < 6; face++)
  {
    const double *vals = pb->bc_val[face];
    int type = pb->bc_type[face];
    if (type == PFO_BC_OVERLAND_KIN || type == PFO_BC_OVERLAND_DIFF || type == PFO_BC_OVERLAND)
    {
      /* OverlandBC :1437-1690 / OverlandKinematicBC :1786-2026 /
       * OverlandDiffusiveBC :2028-2259, z_upper only; they differ in the
       * face fluxes (and OverlandBC adds the spin-up damping term, zero
       * with OverlandSpinupDampP1/P2 at their defaults of 0) */
      long n2 = (long)(nx + 2) * (ny + 2);
      ke = (double*)calloc(n2, sizeof(double));
      kw = (double*)calloc(n2, sizeof(double));
      kn = (double*)calloc(n2, sizeof(double));
      ks = (double*)calloc(n2, sizeof(double));
      if (type == PFO_BC_OVERLAND_KIN)
        ovl_fcn(pb, p, ke, kw, kn, ks);
      else if (type == PFO_BC_OVERLAND_DIFF)
        ovd_fcn(pb, p, p_old, ke, kw, kn, ks);
      else
        ovf_fcn(pb, p, ke, kw, kn, ks);
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
        {
          long c = IDX(i, j, nz - 1);
          long io = (i + 1) + (long)(nx + 2) * (j + 1);
          double q_overlnd = vol * (PFMAX(p[c], 0.0) - PFMAX(p_old[c], 0.0)) / dz +
                             dt * vol * ((ke[io] - kw[io]) / dx + (kn[io] - ks[io]) / dy) / dz;
          if (type == PFO_BC_OVERLAND)
          {
            /* spin-up damping (OverlandSpinupDampP1 / P2), and with
             * OverlandFlowSpinUp the ponded head drained in place of the
             * ponding and routing term (:1659-1673) */
            const double pm = p[c] < 0.0 ? p[c] : 0.0;
            q_overlnd = q_overlnd + vol * dt / dz * (exp(pm * pb->ov_damp_p1) * pb->ov_damp_p2);
            if (pb->ov_spinup == 1)
              q_overlnd = (vol / dz) * dt
                          * ((PFMAX(p[c], 0.0) - 0.0) + exp(pm * pb->ov_damp_p1) * pb->ov_damp_p2);
          }
          f[c] += q_overlnd;
          double u_new = ffz * vals[i + nx * j];
          f[c] += dt * 1.0 * u_new;
          /* q_overlnd_x/y = ke, kn of the column; the top face velocity
           * carries the ponding and routing term (:1648-1687) */
          if (out->qx)
            out->qx[i + (long)nx * j] = ke[io];
          if (out->qy)
            out->qy[i + (long)nx * j] = kn[io];
          if (out->vz)
          {
            u_new += q_overlnd / dt;
            out->vz[c + (long)nx * ny] = u_new / ffz;
          }
        }
      continue;
    }
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
        {
          if (!on_face(pb, face, i, j, k))
            continue;
          long c = IDX(i, j, k);
          double value = vals[face_index(pb, face, i, j, k)];
          double dir = (face & 1) ? 1.0 : -1.0;
          double u_new, h_face = 0.0, vel;
          /* this face's entry of vx / vy / vz (the patch loops' vel_idx) */
          double *vslot = NULL;
          if (face < 2 && out->vx)
            vslot = out->vx + (i + (face & 1)) + (long)(nx + 1) * (j + (long)ny * k);
          else if (face >= 2 && face < 4 && out->vy)
            vslot = out->vy + i + (long)nx * ((j + (face & 1)) + (long)(ny + 1) * k);
          else if (face >= 4 && out->vz)
            vslot = out->vz + i + (long)nx * (j + (long)ny * (k + (face & 1)));
          if (type == PFO_BC_FLUX || type == PFO_BC_SEEPAGE)
          {
            /* FluxConst, or SeepageFace (:1692-1784): a flux face whose top
             * face also drains the ponded water, (vol / dz) dt max(p, 0) */
            double q_overlnd = 0.0;
            if (type == PFO_BC_SEEPAGE && face == 5)
            {
              q_overlnd = (vol / dz) * dt * (PFMAX(p[c], 0.0) - 0.0);
              f[c] += q_overlnd;
            }
            double h = (face < 2) ? ffx * zm[k] : (face < 4) ? ffy * zm[k] : ffz;
            u_new = h * value;
            /* FluxBC stores the patch value itself (:1432); SeepageFaceBC
             * (u_new + q_overlnd / dt) / h (:1775-1781) */
            vel = (type == PFO_BC_FLUX) ? value : (u_new + q_overlnd / dt) / h;
            if (vslot)
              *vslot = vel;
          }
          else
          {
            /* ghost cell holds the Dirichlet value; its rel. perm. uses the
             * interior cell's VG parameters (GrGeomSurfLoop, :615) */
            double krg = kr_at(pb, value, pb->alpha[c], pb->n[c], 0);
            if (face < 4)
            {
              double h = (face < 2) ? ffx * zm[k] : ffy * zm[k];
              double kk = (face < 2) ? pb->kx[c] : pb->ky[c];
              double dd = (face < 2) ? dx : dy;
              if (dir < 0)
              {
                double diff = value - p[c];
                u_new = UPSTREAM(value, p[c], krg * rho, kr[c] * rho);
                u_new = u_new * h * (kk / visc) * 2.0 * (diff / dd);
              }
              else
              {
                double diff = p[c] - value;
                u_new = UPSTREAM(p[c], value, kr[c] * rho, krg * rho);
                u_new = u_new * h * (kk / visc) * 2.0 * (diff / dd);
              }
            }
            else
            {
              double h = ffz;
              double sep = dz * zm[k];
              double lower, upper;
              if (dir < 0)
              {
                lower = value / sep - 0.25 * rho * g;
                upper = p[c] / sep + 0.25 * rho * g;
                u_new = UPSTREAM(lower, upper, krg * rho, kr[c] * rho);
              }
              else
              {
                lower = (p[c] / sep) - 0.25 * rho * g * 1.0;
                upper = (value / sep) + 0.25 * rho * g * 1.0;
                u_new = UPSTREAM(lower, upper, kr[c] * rho, krg * rho);
              }
              u_new = u_new * h * (pb->kz[c] / visc) * 2.0 * (lower - upper);
            }
            /* DirichletBC: u_new / h (:1227-1230) */
            h_face = (face < 2) ? ffx * zm[k] : (face < 4) ? ffy * zm[k] : ffz;
            if (vslot)
              *vslot = u_new / h_face;
          }
          f[c] += dt * dir * u_new;
        }
  }
  free(ke);
  free(kw);
  free(kn);
  free(ks);
  free(sat);
  free(kr);
}

/* -------------------------------------------------------------------------
 * Jacobian  (PL/richards_jacobian_eval.c:217-1420)
 *   J[0..6] = C W E S N L U (full) ; symm: J[0..3] = C E N U ; symm 2: also
 *   J[4] (ny*nz) = the W entries of the i = 0 cells, which the symmetric
 *   storage keeps in the x_lower ghost column of E (matrix.c:477-490) and
 *   MGSemi's setup reads (mg_semi.c:563, 671-682)
 * ------------------------------------------------------------------------- */
void pfo_jacobian_fd(const pfo_problem *pb, double dt, const double *p, int symm, int fd,
                     double *const *J);

void pfo_jacobian(const pfo_problem *pb, double dt, const double *p, int symm,
                  double *const *J)
{
  pfo_jacobian_fd(pb, dt, p, symm, 0, J);
}

/* fd = 1: the matrix the reference builds under Solver.Nonlinear.UseJacobian
 * False, where the Jacobian module's type is no_nonlinear_jacobian
 * (richards_jacobian_eval.c:2476-2484): the overland surface terms are left
 * out (they are added only with using_MGSemi, which that key clears, :1863),
 * and an OverlandFlow top cell with p > 0 gets the diagonal term of the
 * "simple" case it falls through to (:1241-1254) */
void pfo_jacobian_fd(const pfo_problem *pb, double dt, const double *p, int symm, int fd,
                     double *const *J)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz;
  const long N = (long)nx * ny * nz;
  const long sy = nx, sz = (long)nx * ny;
  const double dx = pb->dx, dy = pb->dy, dz = pb->dz;
  const double g = pb->gravity, visc = pb->viscosity, rho = pb->density;
  const double drho = 0.0;
  const double vol = dx * dy * dz;
  const double ffx = dy * dz, ffy = dx * dz, ffz = dx * dy;
  const double *zm = pb->z_mult;
  double *cp = J[0];
  double *wp = symm ? NULL : J[1], *ep = symm ? J[1] : J[2];
  double *sop = symm ? NULL : J[3], *np = symm ? J[2] : J[4];
  double *lp = symm ? NULL : J[5], *up = symm ? J[3] : J[6];
  int nst = symm ? 4 : 7;
  double *sat = (double*)malloc(N * sizeof(double));
  double *dsat = (double*)malloc(N * sizeof(double));
  double *kr = (double*)malloc(N * sizeof(double));
  double *dkr = (double*)malloc(N * sizeof(double));

  for (int s = 0; s < nst; s++)
    memset(J[s], 0, N * sizeof(double));
  double *wghost = (symm == 2) ? J[4] : NULL;
  if (wghost)
    memset(wghost, 0, (size_t)ny * nz * sizeof(double));
  pfo_saturation(pb, p, sat, 0);
  pfo_saturation(pb, p, dsat, 1);
  pfo_relperm(pb, p, kr, 0);
  pfo_relperm(pb, p, dkr, 1);

  /* storage diagonal :445-452 */
  for (int k = 0; k < nz; k++)
    for (long c = k * sz; c < (k + 1) * sz; c++)
    {
      double vol2 = vol * zm[k];
      cp[c] += (dsat[c] * rho + sat[c] * drho) * pb->porosity * vol2
               + pb->sstorage * vol2 * (dsat[c] * rho * p[c] + sat[c] * drho * p[c] + sat[c] * rho);
    }

  /* face terms :594-780, gravity terms from the subsurface slopes */
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        double x_dir_g, x_dir_g_c, y_dir_g, y_dir_g_c;
        tfg_x(pb, i, j, &x_dir_g, &x_dir_g_c);
        tfg_y(pb, i, j, &y_dir_g, &y_dir_g_c);
        double prod = kr[c] * rho;
        double prod_der = dkr[c] * rho + kr[c] * drho;
        double west_temp = 0.0, east_temp = 0.0, sym_east_temp = 0.0;
        double south_temp = 0.0, north_temp = 0.0, sym_north_temp = 0.0;
        double lower_temp = 0.0, upper_temp = 0.0, sym_upper_temp = 0.0;
        if (i + 1 < nx)
        {
          long e = c + 1;
          double prod_rt = kr[e] * rho;
          double prod_rt_der = dkr[e] * rho + kr[e] * drho;
          double diff = p[c] - p[e];
          double updir = (diff / dx) * x_dir_g_c - x_dir_g;
          double x_coeff = (pb->fbx ? pb->fbx[c] : 1.0) * dt * ffx * (1.0 / dx) * zm[k] *
                           HARMONIC(pb->kx[c], pb->kx[e]) / visc;
          double sym_west_temp = (-x_coeff * UPSTREAM(updir, 0.0, prod, prod_rt)) * x_dir_g_c;
          west_temp = (-x_coeff * diff * UPSTREAM(updir, 0.0, prod_der, 0.0)) * x_dir_g_c + sym_west_temp;
          west_temp += (x_coeff * dx * UPSTREAM(updir, 0.0, prod_der, 0.0)) * x_dir_g;
          sym_east_temp = (-x_coeff * UPSTREAM(updir, 0.0, prod, prod_rt)) * x_dir_g_c;
          east_temp = (x_coeff * diff * UPSTREAM(updir, 0.0, 0.0, prod_rt_der)) * x_dir_g_c + sym_east_temp;
          east_temp += -(x_coeff * dx * UPSTREAM(updir, 0.0, 0.0, prod_rt_der)) * x_dir_g;
        }
        if (j + 1 < ny)
        {
          long n = c + sy;
          double prod_no = kr[n] * rho;
          double prod_no_der = dkr[n] * rho + kr[n] * drho;
          double diff = p[c] - p[n];
          double updir = (diff / dy) * y_dir_g_c - y_dir_g;
          double y_coeff = (pb->fby ? pb->fby[c] : 1.0) * dt * ffy * (1.0 / dy) * zm[k] *
                           HARMONIC(pb->ky[c], pb->ky[n]) / visc;
          double sym_south_temp = -y_coeff * UPSTREAM(updir, 0.0, prod, prod_no) * y_dir_g_c;
          south_temp = -y_coeff * diff * UPSTREAM(updir, 0.0, prod_der, 0.0) * y_dir_g_c + sym_south_temp;
          south_temp += (y_coeff * dy * UPSTREAM(updir, 0.0, prod_der, 0.0)) * y_dir_g;
          sym_north_temp = y_coeff * -UPSTREAM(updir, 0.0, prod, prod_no) * y_dir_g_c;
          north_temp = y_coeff * diff * UPSTREAM(updir, 0.0, 0.0, prod_no_der) * y_dir_g_c + sym_north_temp;
          north_temp += -(y_coeff * dy * UPSTREAM(updir, 0.0, 0.0, prod_no_der)) * y_dir_g;
        }
        if (k + 1 < nz)
        {
          long u = c + sz;
          double prod_up = kr[u] * rho;
          double prod_up_der = dkr[u] * rho + kr[u] * drho;
          double zc = zm[k], zu = zm[k + 1];
          double sep = (dz * AMEAN(zc, zu));
          double lower_cond = p[c] / sep - (zc / (zc + zu)) * rho * g;
          double upper_cond = p[u] / sep + (zu / (zc + zu)) * rho * g;
          double diff = lower_cond - upper_cond;
          double z_coeff = (pb->fbz ? pb->fbz[c] : 1.0) * dt * ffz *
                           HARMONIC_DZ(pb->kz[c], pb->kz[u], zc, zu) / visc;
          double sym_lower_temp = -z_coeff * (1.0 / (dz * AMEAN(zc, zu)))
                                  * UPSTREAM(lower_cond, upper_cond, prod, prod_up);
          lower_temp = -z_coeff * (diff * UPSTREAM(lower_cond, upper_cond, prod_der, 0.0)
                                   + (-g * 0.5 * dz * (AMEAN(zc, zu)) * drho
                                      * UPSTREAM(lower_cond, upper_cond, prod, prod_up)))
                       + sym_lower_temp;
          sym_upper_temp = z_coeff * (1.0 / (dz * AMEAN(zc, zu)))
                           * -UPSTREAM(lower_cond, upper_cond, prod, prod_up);
          upper_temp = z_coeff * (diff * UPSTREAM(lower_cond, upper_cond, 0.0, prod_up_der)
                                  + (-g * 0.5 * dz * (AMEAN(zc, zu)) * drho
                                     * UPSTREAM(lower_cond, upper_cond, prod, prod_up)))
                       + sym_upper_temp;
        }
        cp[c] += -(west_temp + south_temp + lower_temp);
        if (i + 1 < nx) cp[c + 1] += -east_temp;
        if (j + 1 < ny) cp[c + sy] += -north_temp;
        if (k + 1 < nz) cp[c + sz] += -upper_temp;
        if (!symm)
        {
          if (i + 1 < nx) { ep[c] += east_temp; wp[c + 1] += west_temp; }
          if (j + 1 < ny) { np[c] += north_temp; sop[c + sy] += south_temp; }
          if (k + 1 < nz) { up[c] += upper_temp; lp[c + sz] += lower_temp; }
        }
        else
        {
          if (i + 1 < nx) ep[c] += sym_east_temp;
          if (j + 1 < ny) np[c] += sym_north_temp;
          if (k + 1 < nz) up[c] += sym_upper_temp;
        }
      }

  /* Dirichlet patches :1049-1200 (flux patches leave the row unchanged) */
  for (int face = 0; face < 6; face++)
  {
    if (pb->bc_type[face] != PFO_BC_DIRICHLET)
      continue;
    const double *vals = pb->bc_val[face];
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
        {
          if (!on_face(pb, face, i, j, k))
            continue;
          long c = IDX(i, j, k);
          double value = vals[face_index(pb, face, i, j, k)];
          double den_d = rho;
          double prod = kr[c] * rho;
          double prod_der = dkr[c] * rho + kr[c] * drho;
          double prod_val = kr_at(pb, value, pb->alpha[c], pb->n[c], 0) * den_d;
          double o_temp, coeff, diff;
          /* the z_mult ghost above the top layer keeps the 1 it was
           * initialised with (problem_dz_scale.c:92) */
          double zu = (k + 1 < nz) ? zm[k + 1] : 1.0;
          switch (face)
          {
            case 0:
              coeff = dt * ffx * zm[k] * (2.0 / dx) * pb->kx[c] / visc;
              diff = value - p[c];
              o_temp = coeff * (diff * UPSTREAM(value, p[c], 0.0, prod_der)
                                - UPSTREAM(value, p[c], prod_val, prod));
              break;
            case 1:
              coeff = dt * ffx * zm[k] * (2.0 / dx) * pb->kx[c] / visc;
              diff = p[c] - value;
              o_temp = -coeff * (diff * UPSTREAM(p[c], value, prod_der, 0.0)
                                 + UPSTREAM(p[c], value, prod, prod_val));
              break;
            case 2:
              coeff = dt * ffy * zm[k] * (2.0 / dy) * pb->ky[c] / visc;
              diff = value - p[c];
              o_temp = coeff * (diff * UPSTREAM(value, p[c], 0.0, prod_der)
                                - UPSTREAM(value, p[c], prod_val, prod));
              break;
            case 3:
              coeff = dt * ffy * zm[k] * (2.0 / dy) * pb->ky[c] / visc;
              diff = p[c] - value;
              o_temp = -coeff * (diff * UPSTREAM(p[c], value, prod_der, 0.0)
                                 + UPSTREAM(p[c], value, prod, prod_val));
              break;
            case 4:
            {
              coeff = dt * ffz * (2.0 / (dz * AMEAN(zm[k], zu))) * pb->kz[c] / visc;
              double lower_cond = (value) - 0.5 * dz * zm[k] * den_d * g;
              double upper_cond = (p[c]) + 0.5 * dz * zm[k] * rho * g;
              diff = lower_cond - upper_cond;
              o_temp = coeff * (diff * UPSTREAM(lower_cond, upper_cond, 0.0, prod_der)
                                + ((-1.0 - g * 0.5 * dz * zm[k] * drho)
                                   * UPSTREAM(lower_cond, upper_cond, prod_val, prod)));
              break;
            }
            default:
            {
              coeff = dt * ffz * (2.0 / (dz * AMEAN(zm[k], zu))) * pb->kz[c] / visc;
              double lower_cond = (p[c]) - 0.5 * dz * zm[k] * rho * g;
              double upper_cond = (value) + 0.5 * dz * zm[k] * den_d * g;
              diff = lower_cond - upper_cond;
              o_temp = -coeff * (diff * UPSTREAM(lower_cond, upper_cond, prod_der, 0.0)
                                 + ((1.0 - g * 0.5 * dz * zm[k] * drho)
                                    * UPSTREAM(lower_cond, upper_cond, prod, prod_val)));
              break;
            }
          }
          cp[c] -= o_temp;
        }
  }

  /* SeepageFace on the top face (:1319-1345), in patch order after the
   * Dirichlet corrections of the other faces */
  if (pb->bc_type[5] == PFO_BC_SEEPAGE)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        if (p[c] >= 0.0)
          cp[c] += (vol / dz) * dt * (1.0 + 0.0);
        else
          cp[c] += 0.0;
      }

  /* the "simple" diagonal term of an OverlandFlow patch in the
   * difference-quotient mode; the z_mult ghost above the top layer keeps
   * the 1 it was initialised with (problem_dz_scale.c:92) */
  if (fd && pb->bc_type[5] == PFO_BC_OVERLAND)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        if (p[c] > 0.0)
          cp[c] += (vol * zm[nz - 1]) / (dz * AMEAN(zm[nz - 1], 1.0)) * (dt + 1);
      }

  /* kinematic overland terms on the top layer, MGSemi form (:1863-1990),
   * after every other term.  In the symmetric storage a lower coefficient is
   * the neighbour's upper one (matrix.c:484-490): W(i) = E(i-1), S(j) = N(j-1). */
  if (!fd && pb->bc_type[5] == PFO_BC_OVERLAND_KIN)
  {
    const int sy2 = nx + 2;
    long n2 = (long)(nx + 2) * (ny + 2);
    double *ke = (double*)calloc(n2, sizeof(double));
    double *kw = (double*)calloc(n2, sizeof(double));
    double *kn = (double*)calloc(n2, sizeof(double));
    double *ks = (double*)calloc(n2, sizeof(double));
    ovl_der(pb, p, ke, kw, kn, ks);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        long io = (i + 1) + (long)sy2 * (j + 1);
        if (p[c] > 0.0)
          cp[c] += (vol / dz) + (vol / ffy) * dt * (ke[io] - kw[io])
                   + (vol / ffx) * dt * (kn[io] - ks[io]);
        double tw = (vol / ffy) * dt * (ke[io - 1]);
        double te = (vol / ffy) * dt * (kw[io + 1]);
        double ts = (vol / ffx) * dt * (kn[io - sy2]);
        double tn = (vol / ffx) * dt * (ks[io + sy2]);
        if (!symm)
        {
          wp[c] -= tw;
          ep[c] += te;
          sop[c] -= ts;
          np[c] += tn;
        }
        else
        {
          if (i > 0) ep[c - 1] -= tw;
          ep[c] += te;
          if (j > 0) np[c - sy] -= ts;
          np[c] += tn;
        }
      }
    free(ke);
    free(kw);
    free(kn);
    free(ks);
  }
  /* OverlandFlowSpinUp: the OverlandFlow patch's own diagonal term of a
   * top cell with p >= 0 (:1258-1268), in patch order */
  if (!fd && pb->bc_type[5] == PFO_BC_OVERLAND && pb->ov_spinup == 1)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        if (p[c] >= 0.0)
          cp[c] += (vol / dz) * dt * (1.0 + 0.0);
      }

  /* OverlandFlow terms on the top layer, MGSemi form (:2028-2090): the
   * derivative parts of each column's own flux (zero with
   * OverlandFlowSpinUp, which skips their evaluation, :1287) and the
   * derivative of the spin-up damping term of a non-ponded cell */
  if (!fd && pb->bc_type[5] == PFO_BC_OVERLAND)
  {
    const int sy2 = nx + 2;
    long n2 = (long)(nx + 2) * (ny + 2);
    double *buf = (double*)calloc(4 * n2, sizeof(double));
    double *ke = buf, *kw = buf + n2, *kn = buf + 2 * n2, *ks = buf + 3 * n2;
    if (pb->ov_spinup != 1)
      ovf_der(pb, p, ke, kw, kn, ks);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        long io = (i + 1) + (long)sy2 * (j + 1);
        if (p[c] > 0.0)
          cp[c] += (vol / dz) + (vol / ffy) * dt * (ke[io] - kw[io])
                   + (vol / ffx) * dt * (kn[io] - ks[io]);
        else
          cp[c] += 0.0 + dt * (vol / dz)
                         * (pb->ov_damp_p1 * exp((p[c] < 0.0 ? p[c] : 0.0) * pb->ov_damp_p1)
                            * pb->ov_damp_p2);
        double tw = (vol / ffy) * dt * (ke[io - 1]);
        double te = (vol / ffy) * dt * (kw[io + 1]);
        double ts = (vol / ffx) * dt * (kn[io - sy2]);
        double tn = (vol / ffx) * dt * (ks[io + sy2]);
        if (!symm)
        {
          wp[c] -= tw;
          ep[c] += te;
          sop[c] -= ts;
          np[c] += tn;
        }
        else
        {
          if (i > 0) ep[c - 1] -= tw;
          else if (wghost) wghost[j + (long)ny * (nz - 1)] -= tw;
          ep[c] += te;
          if (j > 0) np[c - sy] -= ts;
          np[c] += tn;
        }
      }
    free(buf);
  }
  /* diffusive overland terms on the top layer, MGSemi form (:1989-2026):
   * off-diagonals from the non-symmetric derivative parts of this column */
  if (!fd && pb->bc_type[5] == PFO_BC_OVERLAND_DIFF)
  {
    const int sy2 = nx + 2;
    long n2 = (long)(nx + 2) * (ny + 2);
    double *buf = (double*)calloc(8 * n2, sizeof(double));
    double *ke = buf, *kw = buf + n2, *kn = buf + 2 * n2, *ks = buf + 3 * n2;
    double *kens = buf + 4 * n2, *kwns = buf + 5 * n2, *knns = buf + 6 * n2, *ksns = buf + 7 * n2;
    ovd_der(pb, p, pb->ov_p_old, ke, kw, kn, ks, kens, kwns, knns, ksns);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, nz - 1);
        long io = (i + 1) + (long)sy2 * (j + 1);
        if (p[c] > 0.0)
          cp[c] += (vol / dz) + (vol / ffy) * dt * (ke[io] - kw[io])
                   + (vol / ffx) * dt * (kn[io] - ks[io]);
        double tw = (vol / ffy) * dt * (kwns[io]);
        double te = (vol / ffy) * dt * (kens[io]);
        double ts = (vol / ffx) * dt * (ksns[io]);
        double tn = (vol / ffx) * dt * (knns[io]);
        if (!symm)
        {
          wp[c] -= tw;
          ep[c] += te;
          sop[c] -= ts;
          np[c] += tn;
        }
        else
        {
          if (i > 0) ep[c - 1] -= tw;
          else if (wghost) wghost[j + (long)ny * (nz - 1)] -= tw;
          ep[c] += te;
          if (j > 0) np[c - sy] -= ts;
          np[c] += tn;
        }
      }
    free(buf);
  }
  free(sat);
  free(dsat);
  free(kr);
  free(dkr);
}

/* y = J x, stencil order C W E S N L U (PL/matvec.c:35-330: y = 0, then one
 * accumulation pass per stencil entry). */
void pfo_matvec7(const pfo_problem *pb, double *const *J, const double *x, double *y)
{
  const int nx = pb->nx, ny = pb->ny, nz = pb->nz;
  const long sy = nx, sz = (long)nx * ny;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        double acc = 0.0;
        acc += J[0][c] * x[c];
        acc += J[1][c] * (i > 0 ? x[c - 1] : 0.0);
        acc += J[2][c] * (i + 1 < nx ? x[c + 1] : 0.0);
        acc += J[3][c] * (j > 0 ? x[c - sy] : 0.0);
        acc += J[4][c] * (j + 1 < ny ? x[c + sy] : 0.0);
        acc += J[5][c] * (k > 0 ? x[c - sz] : 0.0);
        acc += J[6][c] * (k + 1 < nz ? x[c + sz] : 0.0);
        y[c] = acc;
      }
}

/* -------------------------------------------------------------------------
 * MGSemi  (PL/mg_semi.c, mg_semi_restrict.c, mg_semi_prolong.c, rb_GS_point.c)
 * Every level stores a symmetric 7-point operator as C E N U; the lower
 * entries are the upper entries of the neighbour (PL/matrix.c:258-310,
 * 477-490).  Boundary-face coefficients are zero.  With PCMatrixType
 * FullJacobian the finest operator is the non-symmetric Jacobian, whose
 * lower entries W S L are stored apart (richards_jacobian_eval.c:2246-2258);
 * the coarse operators are symmetric all the same (mg_semi.c:1071-1072).
 * ------------------------------------------------------------------------- */
typedef struct {
  int nx, ny, nz;
  long n;
  double *a[4];       /* C E N U */
  double *x, *b, *t;  /* solution, rhs, temp */
  int dir;            /* coarsening direction to the next level */
  double *p1, *p2;    /* prolongation weights, fine-grid sized (used at odd points) */
  double *wg;         /* (ny*nz) W entries of the i = 0 cells: the x_lower ghost column
                       * of E in the symmetric storage; zero unless the finest
                       * operator has one (diffusive overland terms) */
  double *sg, *lg;    /* (nx*nz) S entries of the j = 0 cells and (nx*ny) L entries
                       * of the k = 0 cells: the y_lower / z_lower ghost planes of
                       * N and U, which the setup of a coarse operator writes */
  double *lo[3];      /* W S L of a non-symmetric operator (finest level with
                       * FullJacobian), else NULL */
} mg_level;

struct pfo_mg {
  int nlev;
  mg_level *L;
  int smoother;
  double weight;
  int max_iter;       /* Solver.Linear.Preconditioner.MGSemi.MaxIter */
};

static void lvl_alloc(mg_level *l, int nx, int ny, int nz)
{
  l->nx = nx; l->ny = ny; l->nz = nz;
  l->n = (long)nx * ny * nz;
  for (int s = 0; s < 4; s++)
    l->a[s] = (double*)calloc(l->n, sizeof(double));
  l->x = (double*)calloc(l->n, sizeof(double));
  l->b = (double*)calloc(l->n, sizeof(double));
  l->t = (double*)calloc(l->n, sizeof(double));
  l->p1 = (double*)calloc(l->n, sizeof(double));
  l->p2 = (double*)calloc(l->n, sizeof(double));
  l->wg = (double*)calloc((size_t)ny * nz, sizeof(double));
  l->sg = (double*)calloc((size_t)nx * nz, sizeof(double));
  l->lg = (double*)calloc((size_t)nx * ny, sizeof(double));
  for (int s = 0; s < 3; s++)
    l->lo[s] = NULL;
}

/* coarsening directions: PL/mg_semi.c:858-923 */
pfo_mg *pfo_mg_create(const pfo_problem *pb, const pfo_settings *st)
{
  int max_levels = st->mg_max_levels > 0 ? st->mg_max_levels : 100;
  double DX = pb->dx, DY = pb->dy, DZ = pb->dz;
  int NX = pb->nx, NY = pb->ny, NZ = pb->nz;
  /* max(2 MaxMinN - 1, 2) per direction (PL/mg_semi.c:869-872) */
  int minN[3];
  for (int q = 0; q < 3; q++)
  {
    int m = st->mg_max_min_n[q] > 1 ? st->mg_max_min_n[q] : 1;
    minN[q] = 2 * m - 1 > 2 ? 2 * m - 1 : 2;
  }
  int dirs[128];
  int l;
  for (l = 0; l < max_levels - 1 && l < 127; l++)
  {
    double min_spacing = DX + DY + DZ;
    int d = -1;
    if ((NX >= minN[0]) && (DX < min_spacing)) { min_spacing = DX; d = 0; }
    if ((NY >= minN[1]) && (DY < min_spacing)) { min_spacing = DY; d = 1; }
    if ((NZ >= minN[2]) && (DZ < min_spacing)) { min_spacing = DZ; d = 2; }
    if (d == -1)
      break;
    if (d == 0) { DX *= 2; NX = (NX + 1) / 2; }
    if (d == 1) { DY *= 2; NY = (NY + 1) / 2; }
    if (d == 2) { DZ *= 2; NZ = (NZ + 1) / 2; }
    dirs[l] = d;
  }
  pfo_mg *mg = (pfo_mg*)calloc(1, sizeof(pfo_mg));
  mg->nlev = l + 1;
  mg->L = (mg_level*)calloc(mg->nlev, sizeof(mg_level));
  mg->smoother = st->mg_smoother;
  mg->max_iter = st->mg_max_iter;
  mg->weight = st->wjacobi_weight > 0 ? st->wjacobi_weight : 1.0;
  int nx = pb->nx, ny = pb->ny, nz = pb->nz;
  for (int i = 0; i < mg->nlev; i++)
  {
    lvl_alloc(&mg->L[i], nx, ny, nz);
    if (i < mg->nlev - 1)
    {
      mg->L[i].dir = dirs[i];
      if (dirs[i] == 0) nx = (nx + 1) / 2;
      if (dirs[i] == 1) ny = (ny + 1) / 2;
      if (dirs[i] == 2) nz = (nz + 1) / 2;
    }
    else
      mg->L[i].dir = -1;
  }
  return mg;
}

int pfo_mg_num_levels(const pfo_mg *mg) { return mg->nlev; }

void pfo_mg_level_info(const pfo_mg *mg, int l, int *nx, int *ny, int *nz, int *dir)
{
  *nx = mg->L[l].nx; *ny = mg->L[l].ny; *nz = mg->L[l].nz; *dir = mg->L[l].dir;
}

void pfo_mg_destroy(pfo_mg *mg)
{
  for (int i = 0; i < mg->nlev; i++)
  {
    mg_level *l = &mg->L[i];
    for (int s = 0; s < 4; s++) free(l->a[s]);
    free(l->x); free(l->b); free(l->t); free(l->p1); free(l->p2); free(l->wg);
    free(l->sg); free(l->lg);
    for (int s = 0; s < 3; s++) free(l->lo[s]);
  }
  free(mg->L);
  free(mg);
}

/* Full 7-point coefficient s (0..6 = C W E S N L U) at (i,j,k) of a level,
 * from the symmetric C E N U storage (the lower entries of the first
 * row / column / plane from the ghost arrays) or from the W S L arrays of a
 * non-symmetric level; zero outside the level. */
static double coef(const mg_level *l, int s, int i, int j, int k)
{
  int nx = l->nx, ny = l->ny, nz = l->nz;
  if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz)
    return 0.0;
  if (l->lo[0] && (s == 1 || s == 3 || s == 5))
    return l->lo[(s - 1) / 2][IDX(i, j, k)];
  switch (s)
  {
    case 0: return l->a[0][IDX(i, j, k)];
    case 1: return (i > 0) ? l->a[1][IDX(i - 1, j, k)] : l->wg[j + (long)ny * k];
    case 2: return l->a[1][IDX(i, j, k)];
    case 3: return (j > 0) ? l->a[2][IDX(i, j - 1, k)] : l->sg[i + (long)nx * k];
    case 4: return l->a[2][IDX(i, j, k)];
    case 5: return (k > 0) ? l->a[3][IDX(i, j, k - 1)] : l->lg[i + (long)nx * j];
    default: return l->a[3][IDX(i, j, k)];
  }
}

static double vget(const mg_level *l, const double *v, int i, int j, int k)
{
  int nx = l->nx, ny = l->ny;
  if (i < 0 || j < 0 || k < 0 || i >= l->nx || j >= l->ny || k >= l->nz)
    return 0.0;
  return v[IDX(i, j, k)];
}

/* stencil reorder so that entries 1,2 are the coarsening direction
 * (PL/mg_semi.c:478-499) */
static void snum_for(int dir, int s[7])
{
  static const int sx[7] = { 0, 1, 2, 3, 4, 5, 6 };
  static const int sy[7] = { 0, 3, 4, 1, 2, 5, 6 };
  static const int sz[7] = { 0, 5, 6, 3, 4, 1, 2 };
  const int *src = dir == 0 ? sx : dir == 1 ? sy : sz;
  memcpy(s, src, sizeof(int) * 7);
}

/* PL/mg_semi.c:437-760 */
void pfo_mg_set_wghost(pfo_mg *mg, const double *wg)
{
  mg_level *L0 = &mg->L[0];
  size_t n = (size_t)L0->ny * L0->nz;
  if (wg)
    memcpy(L0->wg, wg, n * sizeof(double));
  else
    memset(L0->wg, 0, n * sizeof(double));
}

static void mg_setup_levels(pfo_mg *mg);

void pfo_mg_setup(pfo_mg *mg, double *const *A4)
{
  mg_level *L0 = &mg->L[0];
  for (int s = 0; s < 4; s++)
    memcpy(L0->a[s], A4[s], L0->n * sizeof(double));
  for (int s = 0; s < 3; s++)
  {
    free(L0->lo[s]);
    L0->lo[s] = NULL;
  }
  mg_setup_levels(mg);
}

/* PCMatrixType FullJacobian: the finest operator is the full Jacobian
 * C W E S N L U (kinsol_pc.c:215-246 -> richards_jacobian_eval.c with
 * symm_part 0) */
void pfo_mg_setup_full(pfo_mg *mg, double *const *A7)
{
  mg_level *L0 = &mg->L[0];
  static const int up[4] = { 0, 2, 4, 6 }, dn[3] = { 1, 3, 5 };
  for (int s = 0; s < 4; s++)
    memcpy(L0->a[s], A7[up[s]], L0->n * sizeof(double));
  for (int s = 0; s < 3; s++)
  {
    if (!L0->lo[s])
      L0->lo[s] = (double*)malloc(L0->n * sizeof(double));
    memcpy(L0->lo[s], A7[dn[s]], L0->n * sizeof(double));
  }
  mg_setup_levels(mg);
}

static void mg_setup_levels(pfo_mg *mg)
{
  for (int li = 0; li + 1 < mg->nlev; li++)
  {
    mg_level *F = &mg->L[li], *Cl = &mg->L[li + 1];
    int dir = F->dir;
    int s[7];
    snum_for(dir, s);
    int nx = F->nx, ny = F->ny;
    int ox = dir == 0, oy = dir == 1, oz = dir == 2;
    /* prolongation weights at fine (odd) points */
    for (int k = 0; k < F->nz; k++)
      for (int j = 0; j < F->ny; j++)
        for (int i = 0; i < F->nx; i++)
        {
          int ci = dir == 0 ? i : dir == 1 ? j : k;
          if (!(ci & 1))
            continue;
          double ap0 = coef(F, s[0], i, j, k) + coef(F, s[3], i, j, k) + coef(F, s[4], i, j, k)
                       + coef(F, s[5], i, j, k) + coef(F, s[6], i, j, k);
          long c = IDX(i, j, k);
          if (ap0)
          {
            F->p1[c] = -coef(F, s[1], i, j, k) / ap0;
            F->p2[c] = -coef(F, s[2], i, j, k) / ap0;
          }
          else
          {
            F->p1[c] = 0.0;
            F->p2[c] = 0.0;
          }
        }
    /* coarse operator at coarse points (even fine indices) */
    int cnx = Cl->nx, cny = Cl->ny;
    double *ac[7];
    long cn = Cl->n;
    for (int q = 0; q < 7; q++)
      ac[q] = (double*)calloc(cn, sizeof(double));
    for (int kc = 0; kc < Cl->nz; kc++)
      for (int jc = 0; jc < Cl->ny; jc++)
        for (int ic = 0; ic < Cl->nx; ic++)
        {
          int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
          int i1 = i - ox, j1 = j - oy, k1 = k - oz;   /* fine point below */
          int i2 = i + ox, j2 = j + oy, k2 = k + oz;   /* fine point above */
          long cc = ic + (long)cnx * (jc + (long)cny * kc);
          double p1_1 = vget(F, F->p1, i1, j1, k1), p2_1 = vget(F, F->p2, i1, j1, k1);
          double p1_2 = vget(F, F->p1, i2, j2, k2), p2_2 = vget(F, F->p2, i2, j2, k2);
          for (int q = 3; q <= 6; q++)
            ac[q][cc] = coef(F, s[q], i, j, k) + 0.5 * coef(F, s[q], i1, j1, k1)
                        + 0.5 * coef(F, s[q], i2, j2, k2);
          ac[1][cc] = coef(F, s[1], i, j, k) * p1_1;
          ac[2][cc] = coef(F, s[2], i, j, k) * p2_2;
          ac[0][cc] = coef(F, s[0], i, j, k) + coef(F, s[3], i, j, k) + coef(F, s[4], i, j, k)
                      + coef(F, s[5], i, j, k) + coef(F, s[6], i, j, k)
                      + coef(F, s[1], i, j, k) * p2_1 + coef(F, s[2], i, j, k) * p1_2;
        }
    /* symmetric storage of the coarse operator (the loop of mg_semi.c:667-687
     * runs over the coarse cells in order): a lower entry written by a cell
     * lands in the upper entry of its lower neighbour, so an upper entry is
     * the one its upper neighbour wrote as a lower entry when that neighbour
     * exists, and the lower entries of the first row / column / plane stay
     * in the ghost arrays.  For a symmetric fine operator both writes carry
     * the same value. */
    int q_of[7];
    for (int q = 0; q < 7; q++)
      q_of[s[q]] = q;
    const long csy = cnx, csz = (long)cnx * cny;
    for (int kc = 0; kc < Cl->nz; kc++)
      for (int jc = 0; jc < Cl->ny; jc++)
        for (int ic = 0; ic < Cl->nx; ic++)
        {
          long cc = ic + csy * jc + csz * kc;
          Cl->a[1][cc] = ic + 1 < cnx ? ac[q_of[1]][cc + 1] : ac[q_of[2]][cc];
          Cl->a[2][cc] = jc + 1 < cny ? ac[q_of[3]][cc + csy] : ac[q_of[4]][cc];
          Cl->a[3][cc] = kc + 1 < Cl->nz ? ac[q_of[5]][cc + csz] : ac[q_of[6]][cc];
          if (ic == 0) Cl->wg[jc + (long)cny * kc] = ac[q_of[1]][cc];
          if (jc == 0) Cl->sg[ic + (long)cnx * kc] = ac[q_of[3]][cc];
          if (kc == 0) Cl->lg[ic + (long)cnx * jc] = ac[q_of[5]][cc];
        }
    /* centre: ac0 -= (ac3 + ac4 + ac5 + ac6), the transverse entries as stored */
    for (int kc = 0; kc < Cl->nz; kc++)
      for (int jc = 0; jc < Cl->ny; jc++)
        for (int ic = 0; ic < Cl->nx; ic++)
        {
          long cc = ic + (long)cnx * (jc + (long)cny * kc);
          double t3 = coef(Cl, s[3], ic, jc, kc), t4 = coef(Cl, s[4], ic, jc, kc);
          double t5 = coef(Cl, s[5], ic, jc, kc), t6 = coef(Cl, s[6], ic, jc, kc);
          Cl->a[0][cc] = ac[0][cc] - (t3 + t4 + t5 + t6);
        }
    for (int q = 0; q < 7; q++)
      free(ac[q]);
  }
}

/* r = b - A x on a level (PL/matvec.c with alpha=-1, beta=1) */
static void lvl_residual(const mg_level *l, const double *x, const double *b, double *r)
{
  int nx = l->nx, ny = l->ny, nz = l->nz;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        double y = -b[c];
        y += coef(l, 0, i, j, k) * x[c];
        y += coef(l, 1, i, j, k) * vget(l, x, i - 1, j, k);
        y += coef(l, 2, i, j, k) * vget(l, x, i + 1, j, k);
        y += coef(l, 3, i, j, k) * vget(l, x, i, j - 1, k);
        y += coef(l, 4, i, j, k) * vget(l, x, i, j + 1, k);
        y += coef(l, 5, i, j, k) * vget(l, x, i, j, k - 1);
        y += coef(l, 6, i, j, k) * vget(l, x, i, j, k + 1);
        r[c] = -y;
      }
}

/* one colour sweep of RBGS; colour 0 = red = (i+j+k) odd
 * (PL/comm_pkg.c:132-139, PL/rb_GS_point.c:342-370) */
static void rb_sweep(const mg_level *l, double *x, const double *b, int colour, int init)
{
  int nx = l->nx, ny = l->ny, nz = l->nz;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        int odd = (i + j + k) & 1;
        if ((colour == 0) != (odd == 1))
          continue;
        long c = IDX(i, j, k);
        if (init)
        {
          x[c] = b[c] / coef(l, 0, i, j, k);
          continue;
        }
        x[c] = (b[c] - (coef(l, 1, i, j, k) * vget(l, x, i - 1, j, k)
                        + coef(l, 2, i, j, k) * vget(l, x, i + 1, j, k)
                        + coef(l, 3, i, j, k) * vget(l, x, i, j - 1, k)
                        + coef(l, 4, i, j, k) * vget(l, x, i, j + 1, k)
                        + coef(l, 5, i, j, k) * vget(l, x, i, j, k - 1)
                        + coef(l, 6, i, j, k) * vget(l, x, i, j, k + 1)))
               / coef(l, 0, i, j, k);
      }
}

/* RedBlackGSPoint with MaxIter 1: red, black, red with Symmetric True, red,
 * black with Symmetric False (the sweep count runs from 1 or 2 up to
 * 2 MaxIter + 1, PL/rb_GS_point.c:118-140, 221); with a zero initial guess
 * the first red sweep is x = b / a0 (PL/rb_GS_point.c:128-215) */
static void rbgs_sym(const mg_level *l, double *x, const double *b, int zero, int symmetric)
{
  rb_sweep(l, x, b, 0, zero);
  rb_sweep(l, x, b, 1, 0);
  if (symmetric)
    rb_sweep(l, x, b, 0, 0);
}
static void rbgs(const mg_level *l, double *x, const double *b, int zero)
{
  rbgs_sym(l, x, b, zero, 1);
}

/* WJacobi with MaxIter 1 (PL/w_jacobi.c:120-290) */
static void wjacobi(const mg_level *l, double *x, const double *b, int zero, double w)
{
  int nx = l->nx, ny = l->ny, nz = l->nz;
  if (zero)
  {
    for (long c = 0; c < l->n; c++)
      x[c] = b[c] / l->a[0][c];
    if (w != 1.0)
      for (long c = 0; c < l->n; c++)
        x[c] *= w;
    return;
  }
  double *t = (double*)malloc(l->n * sizeof(double));
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        long c = IDX(i, j, k);
        double v = b[c];
        v -= coef(l, 1, i, j, k) * vget(l, x, i - 1, j, k);
        v -= coef(l, 2, i, j, k) * vget(l, x, i + 1, j, k);
        v -= coef(l, 3, i, j, k) * vget(l, x, i, j - 1, k);
        v -= coef(l, 4, i, j, k) * vget(l, x, i, j + 1, k);
        v -= coef(l, 5, i, j, k) * vget(l, x, i, j, k - 1);
        v -= coef(l, 6, i, j, k) * vget(l, x, i, j, k + 1);
        t[c] = v / coef(l, 0, i, j, k);
      }
  if (w != 1.0)
    for (long c = 0; c < l->n; c++)
      x[c] = (1.0 - w) * x[c] + w * t[c];
  else
    memcpy(x, t, l->n * sizeof(double));
  free(t);
}

static void smooth(const pfo_mg *mg, const mg_level *l, double *x, const double *b, int zero)
{
  if (mg->smoother == 1)
    wjacobi(l, x, b, zero, mg->weight);
  else
    rbgs_sym(l, x, b, zero, mg->smoother != 2);
}

/* r_c = r_f(c) + p2(f below) r_f(f below) + p1(f above) r_f(f above)
 * (PL/mg_semi_restrict.c:161-169) */
static void restrict_lvl(const mg_level *F, const mg_level *Cl, const double *rf, double *rc)
{
  int dir = F->dir, ox = dir == 0, oy = dir == 1, oz = dir == 2;
  int nx = F->nx, ny = F->ny;
  for (int kc = 0; kc < Cl->nz; kc++)
    for (int jc = 0; jc < Cl->ny; jc++)
      for (int ic = 0; ic < Cl->nx; ic++)
      {
        int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
        long cc = ic + (long)Cl->nx * (jc + (long)Cl->ny * kc);
        rc[cc] = rf[IDX(i, j, k)]
                 + (vget(F, F->p2, i - ox, j - oy, k - oz) * vget(F, rf, i - ox, j - oy, k - oz)
                    + vget(F, F->p1, i + ox, j + oy, k + oz) * vget(F, rf, i + ox, j + oy, k + oz));
      }
}

/* e_f = injection at coarse points, p1 e(below) + p2 e(above) at fine points
 * (PL/mg_semi_prolong.c:119-124, 191-197) */
static void prolong_lvl(const mg_level *F, const mg_level *Cl, const double *ec, double *ef)
{
  int dir = F->dir, ox = dir == 0, oy = dir == 1, oz = dir == 2;
  int nx = F->nx, ny = F->ny;
  for (int k = 0; k < F->nz; k++)
    for (int j = 0; j < F->ny; j++)
      for (int i = 0; i < F->nx; i++)
      {
        int ci = dir == 0 ? i : dir == 1 ? j : k;
        if (ci & 1)
          continue;
        long cc = (ox ? i / 2 : i) + (long)Cl->nx * ((oy ? j / 2 : j) + (long)Cl->ny * (oz ? k / 2 : k));
        ef[IDX(i, j, k)] = ec[cc];
      }
  for (int k = 0; k < F->nz; k++)
    for (int j = 0; j < F->ny; j++)
      for (int i = 0; i < F->nx; i++)
      {
        int ci = dir == 0 ? i : dir == 1 ? j : k;
        if (!(ci & 1))
          continue;
        long c = IDX(i, j, k);
        ef[c] = (F->p1[c] * vget(F, ef, i - ox, j - oy, k - oz)
                 + F->p2[c] * vget(F, ef, i + ox, j + oy, k + oz));
      }
}

/* One V-cycle with zero initial guess (PL/mg_semi.c:93-432, MaxIter 1) */
/* MaxIter V-cycles, KinsolPC's tolerance 0 skipping every convergence test
 * (PL/mg_semi.c:198-365, kinsol_pc.c:65-72): MaxIter 0 returns x = b; each
 * cycle after the first starts with a smoothing of the current x */
void pfo_mg_apply(pfo_mg *mg, const double *b, double *x)
{
  int nl = mg->nlev;
  mg_level *L = mg->L;
  if (mg->max_iter < 1)
  {
    memcpy(x, b, L[0].n * sizeof(double));
    return;
  }
  if (nl == 1)
  {
    smooth(mg, &L[0], x, b, 1);
    return;
  }
  smooth(mg, &L[0], x, b, 1);
  for (int it = 1;; it++)
  {
    lvl_residual(&L[0], x, b, L[0].t);
    restrict_lvl(&L[0], &L[1], L[0].t, L[1].b);
    int l;
    for (l = 1; l <= nl - 2; l++)
    {
      smooth(mg, &L[l], L[l].x, L[l].b, 1);
      lvl_residual(&L[l], L[l].x, L[l].b, L[l].t);
      restrict_lvl(&L[l], &L[l + 1], L[l].t, L[l + 1].b);
    }
    /* coarse solve: RedBlackGSPoint, 1 iteration */
    rbgs(&L[l], L[l].x, L[l].b, 1);
    for (l = nl - 2; l >= 1; l--)
    {
      prolong_lvl(&L[l], &L[l + 1], L[l + 1].x, L[l].t);
      for (long c = 0; c < L[l].n; c++)
        L[l].x[c] += L[l].t[c];
      smooth(mg, &L[l], L[l].x, L[l].b, 0);
    }
    prolong_lvl(&L[0], &L[1], L[1].x, L[0].t);
    for (long c = 0; c < L[0].n; c++)
      x[c] += L[0].t[c];
    smooth(mg, &L[0], x, b, 0);
    if (it + 1 > mg->max_iter)
      break;
    smooth(mg, &L[0], x, b, 0);
  }
}

/* -------------------------------------------------------------------------
 * KINSOL / SPGMR  (KS/kinsol.c, KS/kinspgmr.c, KS/spgmr.c, KS/iterativ.c)
 * uscale = fscale = 1 (PL/kinsol_nonlin_solver.c:646-654)
 * ------------------------------------------------------------------------- */
typedef struct {
  const pfo_problem *pb;
  const pfo_settings *st;
  double dt;
  const double *p_old, *s_old;
  long N;
  double *J[7];
  double *PC[5];   /* C E N U, and the W ghost plane of the i = 0 column */
  double *PC7[7];  /* the full preconditioner matrix (PCMatrixType FullJacobian) */
  pfo_mg *mg;
  pfo_stats *stats;
  const double *fval;   /* F at the Newton iterate (difference quotients) */
  double *dq_u, *dq_f;  /* difference-quotient point and its F */
} kctx;

static double dot(const double *a, const double *b, long n)
{
  double s = 0.0;
  for (long i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

static double l1norm(const double *a, long n)
{
  double s = 0.0;
  for (long i = 0; i < n; i++)
    s += fabs(a[i]);
  return s;
}

static double maxabs(const double *a, long n)
{
  double m = 0.0;
  for (long i = 0; i < n; i++)
    if (fabs(a[i]) > m)
      m = fabs(a[i]);
  return m;
}

static void feval(kctx *kc, const double *u, double *f)
{
  pfo_residual(kc->pb, kc->dt, u, kc->p_old, kc->s_old, f);
  kc->stats->nfe++;
}

static void precond(kctx *kc, double *z)
{
  double *x = (double*)malloc(kc->N * sizeof(double));
  pfo_mg_apply(kc->mg, z, x);
  memcpy(z, x, kc->N * sizeof(double));
  free(x);
  kc->stats->nps++;
}

/* SpgmrSolve with x0 = 0, right preconditioning, MGS (KS/spgmr.c:168-450) */
/* KINSpgmrAtimesDQ (KS/kinspgmr.c:481-518) with uscale = 1:
 * J v ~ (F(u + sigma v) - F(u)) / sigma, sigma from Brown and Saad,
 * sign(u.v) sqrt(DerivativeEpsilon) max(|u.v|, |v|_1) / (v.v) */
static void atimes_dq(kctx *kc, const double *u, const double *v, double *z)
{
  long N = kc->N;
  double sutsv = dot(u, v, N);
  double vtv = dot(v, v, N);
  double sq1norm = l1norm(v, N);
  double sign = (sutsv >= 0.0) ? 1.0 : -1.0;
  double sqrt_relfunc = sqrt(kc->st->derivative_epsilon > 0.0 ? kc->st->derivative_epsilon
                                                              : DBL_EPSILON);
  double sigma = sign * sqrt_relfunc * (fabs(sutsv) > sq1norm ? fabs(sutsv) : sq1norm) / vtv;
  double sigma_inv = 1.0 / sigma;
  /* N_VLinearSum(1, u, sigma, v): sigma v + u */
  for (long q = 0; q < N; q++)
    kc->dq_u[q] = sigma * v[q] + u[q];
  feval(kc, kc->dq_u, kc->dq_f);
  /* N_VLinearSum(sigma_inv, F(u + sigma v), -sigma_inv, F(u)): the a == -b
   * case, sigma_inv (x - y) */
  for (long q = 0; q < N; q++)
    z[q] = sigma_inv * (kc->dq_f[q] - kc->fval[q]);
}

static int spgmr(kctx *kc, double *x, const double *b, double delta,
                 const double *u, int *jac_current, double *res_norm)
{
  long N = kc->N;
  int lmax = kc->st->krylov_dim;
  int max_restarts = kc->st->max_restarts;
  double **V = (double**)malloc((lmax + 1) * sizeof(double*));
  for (int i = 0; i <= lmax; i++)
    V[i] = (double*)malloc(N * sizeof(double));
  double *xcor = (double*)calloc(N, sizeof(double));
  double *vtemp = (double*)malloc(N * sizeof(double));
  double *H = (double*)calloc((lmax + 1) * lmax, sizeof(double));
#define Hs(i, j) H[(i) * lmax + (j)]
  double *givens = (double*)calloc(2 * lmax, sizeof(double));
  double *yg = (double*)calloc(lmax + 1, sizeof(double));
  double rho = 0.0, r_norm, beta, rotation_product;
  int krydim = 0, converged = 0, ret = 0;

  memset(x, 0, N * sizeof(double));
  memcpy(V[0], b, N * sizeof(double));
  *res_norm = r_norm = beta = sqrt(dot(V[0], V[0], N));
  if (r_norm <= delta)
  {
    ret = 0;
    goto done;
  }
  for (int ntries = 0; ntries <= max_restarts; ntries++)
  {
    memset(H, 0, (lmax + 1) * lmax * sizeof(double));
    rotation_product = 1.0;
    for (long i = 0; i < N; i++)
      V[0][i] *= 1.0 / r_norm;
    int l;
    for (l = 0; l < lmax; l++)
    {
      kc->stats->nli++;
      krydim = l + 1;
      memcpy(vtemp, V[l], N * sizeof(double));
      precond(kc, vtemp);
      if (!kc->st->use_jacobian)
        atimes_dq(kc, u, vtemp, V[l + 1]);
      else
      {
        if (!*jac_current)
        {
          pfo_jacobian(kc->pb, kc->dt, u, 0, kc->J);
          *jac_current = 1;
        }
        pfo_matvec7(kc->pb, kc->J, vtemp, V[l + 1]);
      }
      /* ModifiedGS (KS/iterativ.c:30-86) */
      {
        int k = l + 1;
        double vk_norm = sqrt(dot(V[k], V[k], N));
        for (int i = 0; i < k; i++)
        {
          Hs(i, k - 1) = dot(V[i], V[k], N);
          double h = -Hs(i, k - 1);
          for (long q = 0; q < N; q++)
            V[k][q] = V[k][q] + h * V[i][q];
        }
        double new_norm = sqrt(dot(V[k], V[k], N));
        double temp = 1000.0 * vk_norm;
        if (!((temp + new_norm) != temp))
        {
          double new_norm_2 = 0.0;
          for (int i = 0; i < k; i++)
          {
            double new_product = dot(V[i], V[k], N);
            double t2 = 1000.0 * Hs(i, k - 1);
            if ((t2 + new_product) == t2)
              continue;
            Hs(i, k - 1) += new_product;
            for (long q = 0; q < N; q++)
              V[k][q] = V[k][q] + (-new_product) * V[i][q];
            new_norm_2 += new_product * new_product;
          }
          if (new_norm_2 != 0.0)
          {
            double np2 = new_norm * new_norm - new_norm_2;
            new_norm = (np2 > 0.0) ? sqrt(np2) : 0.0;
          }
        }
        Hs(k, k - 1) = new_norm;
      }
      /* QRfact, job = l (KS/iterativ.c:147-252) */
      {
        int n = krydim;
        if (l == 0)
        {
          double t1 = Hs(0, 0), t2 = Hs(1, 0), c, s;
          if (t2 == 0.0) { c = 1.0; s = 0.0; }
          else if (fabs(t2) >= fabs(t1)) { double t3 = t1 / t2; s = -1.0 / sqrt(1.0 + t3 * t3); c = -s * t3; }
          else { double t3 = t2 / t1; c = 1.0 / sqrt(1.0 + t3 * t3); s = -c * t3; }
          givens[0] = c; givens[1] = s;
          Hs(0, 0) = c * t1 - s * t2;
        }
        else
        {
          int nm1 = n - 1;
          for (int k = 0; k < nm1; k++)
          {
            double t1 = Hs(k, nm1), t2 = Hs(k + 1, nm1);
            double c = givens[2 * k], s = givens[2 * k + 1];
            Hs(k, nm1) = c * t1 - s * t2;
            Hs(k + 1, nm1) = s * t1 + c * t2;
          }
          double t1 = Hs(nm1, nm1), t2 = Hs(n, nm1), c, s;
          if (t2 == 0.0) { c = 1.0; s = 0.0; }
          else if (fabs(t2) >= fabs(t1)) { double t3 = t1 / t2; s = -1.0 / sqrt(1.0 + t3 * t3); c = -s * t3; }
          else { double t3 = t2 / t1; c = 1.0 / sqrt(1.0 + t3 * t3); s = -c * t3; }
          givens[2 * nm1] = c; givens[2 * nm1 + 1] = s;
          Hs(nm1, nm1) = c * t1 - s * t2;
        }
      }
      rotation_product *= givens[2 * l + 1];
      *res_norm = rho = fabs(rotation_product * r_norm);
      if (rho <= delta)
      {
        converged = 1;
        break;
      }
      for (long q = 0; q < N; q++)
        V[l + 1][q] *= 1.0 / Hs(l + 1, l);
    }
    /* QRsol (KS/iterativ.c:253-286) */
    yg[0] = r_norm;
    for (int i = 1; i <= krydim; i++)
      yg[i] = 0.0;
    for (int k = 0; k < krydim; k++)
    {
      double c = givens[2 * k], s = givens[2 * k + 1];
      double t1 = yg[k], t2 = yg[k + 1];
      yg[k] = c * t1 - s * t2;
      yg[k + 1] = s * t1 + c * t2;
    }
    for (int k = krydim - 1; k >= 0; k--)
    {
      if (Hs(k, k) == 0.0) { ret = 6; goto done; }
      yg[k] /= Hs(k, k);
      for (int i = 0; i < k; i++)
        yg[i] -= yg[k] * Hs(i, k);
    }
    for (int k = 0; k < krydim; k++)
      for (long q = 0; q < N; q++)
        xcor[q] = yg[k] * V[k][q] + 1.0 * xcor[q];
    if (converged)
    {
      precond(kc, xcor);
      for (long q = 0; q < N; q++)
        x[q] = 1.0 * x[q] + 1.0 * xcor[q];
      ret = 0;
      goto done;
    }
    if (ntries == max_restarts)
      break;
    double s_product = 1.0;
    for (int i = krydim; i > 0; i--)
    {
      yg[i] = s_product * givens[2 * i - 2];
      s_product *= givens[2 * i - 1];
    }
    yg[0] = s_product;
    r_norm *= s_product;
    for (int i = 0; i <= krydim; i++)
      yg[i] *= r_norm;
    r_norm = fabs(r_norm);
    for (long q = 0; q < N; q++)
      V[0][q] *= yg[0];
    for (int k = 1; k <= krydim; k++)
      for (long q = 0; q < N; q++)
        V[0][q] = yg[k] * V[k][q] + 1.0 * V[0][q];
  }
  if (rho < beta)
  {
    precond(kc, xcor);
    for (long q = 0; q < N; q++)
      x[q] = x[q] + xcor[q];
    ret = 1;   /* SPGMR_RES_REDUCED */
  }
  else
    ret = 2;   /* SPGMR_CONV_FAIL */
done:
  for (int i = 0; i <= lmax; i++)
    free(V[i]);
  free(V); free(xcor); free(vtemp); free(H); free(givens); free(yg);
#undef Hs
  return ret;
}

/* KINSol (KS/kinsol.c:363-910) with LineSearch or InexactNewton
 * globalization */
void pfo_newton_solve(const pfo_problem *pb_in, const pfo_settings *st, double dt,
                      const double *p_old, const double *s_old, double *p,
                      pfo_stats *stats)
{
  kctx kc;
  /* the Jacobian of this step sees its old pressure (RichardsJacobianEval's
   * old_pressure argument) */
  pfo_problem pstep = *pb_in;
  pstep.ov_p_old = p_old;
  const pfo_problem *pb = &pstep;
  long N = (long)pb->nx * pb->ny * pb->nz;
  memset(stats, 0, sizeof(*stats));
  kc.pb = pb; kc.st = st; kc.dt = dt; kc.p_old = p_old; kc.s_old = s_old; kc.N = N;
  kc.stats = stats;
  for (int s = 0; s < 7; s++) kc.J[s] = (double*)malloc(N * sizeof(double));
  for (int s = 0; s < 4; s++) kc.PC[s] = (double*)malloc(N * sizeof(double));
  kc.PC[4] = (double*)malloc((long)pb->ny * pb->nz * sizeof(double));
  for (int s = 0; s < 7; s++)
    kc.PC7[s] = st->pc_full ? (double*)malloc(N * sizeof(double)) : NULL;
  kc.mg = pfo_mg_create(pb, st);

  double *uu = p;
  double *fval = (double*)malloc(N * sizeof(double));
  double *unew = (double*)malloc(N * sizeof(double));
  double *pp = (double*)malloc(N * sizeof(double));
  double *bb = (double*)malloc(N * sizeof(double));
  kc.fval = fval;
  kc.dq_u = (double*)malloc(N * sizeof(double));
  kc.dq_f = (double*)malloc(N * sizeof(double));
  const double uround = DBL_EPSILON;
  double fnormtol = st->residual_tol, scsteptol = st->step_tol;
  int mxiter = st->max_iter;
  double eta, ealpha = 0.0, egamma = 0.0;
  int etaflag = st->eta_choice;
  if (scsteptol <= 0.0) scsteptol = pow(uround, 2.0 / 3.0);
  if (fnormtol <= 0.0) fnormtol = pow(uround, 1.0 / 3.0);
  double mxnewtstep = 1000.0 * sqrt(dot(uu, uu, N));
  if (mxnewtstep < 1.0) mxnewtstep = 1.0;
  if (etaflag == 1) ealpha = (1.0 + sqrt(5.0)) / 2.0;
  if (etaflag == 2) { ealpha = st->eta_alpha; egamma = st->eta_gamma; }
  eta = (etaflag == 0) ? st->eta_value : 0.5;
  if (etaflag == 2)
  {
    if (ealpha <= 1.0 || ealpha > 2.0) ealpha = 2.0;
    if (egamma <= 0.0 || egamma > 1.0) egamma = 0.9;
  }
  if (eta <= 0.0 || eta > 1.0) eta = 0.1;
  int callForcingTerm = (etaflag != 0);
  double epsmin = 0.01 * fnormtol;
  int ret = 0, ncscmx = 0;
  double sJpnorm = 0.0, sfdotJp = 0.0;

  /* KINInitialStop */
  feval(&kc, uu, fval);
  if (maxabs(fval, N) <= 0.01 * fnormtol)
  {
    /* KINSol returns before loading its optional outputs, so the reported
     * counters stay at zero (KS/kinsol.c:726-731, 851-862) */
    stats->nfe = 0;
    stats->status = 2;
    stats->fnorm = sqrt(dot(fval, fval, N));
    goto out;
  }
  double fnorm = sqrt(dot(fval, fval, N));
  double f1norm = 0.5 * fnorm * fnorm;

  for (;;)
  {
    stats->nni++;
    double eps = (eta + uround) * fnorm;
    if (eps < epsmin) eps = epsmin;
    /* KINLinSolDrv: preconditioner setup every iteration (msbpre = 1) */
    if (st->pc_full)
    {
      pfo_jacobian_fd(pb, dt, uu, 0, !st->use_jacobian, kc.PC7);
      pfo_mg_setup_full(kc.mg, kc.PC7);
    }
    else
    {
      pfo_jacobian_fd(pb, dt, uu, 2, !st->use_jacobian, kc.PC);
      pfo_mg_set_wghost(kc.mg, kc.PC[4]);
      pfo_mg_setup(kc.mg, kc.PC);
    }
    stats->npe++;
    for (long q = 0; q < N; q++) bb[q] = -fval[q];
    int jac_current = 0;
    double res_norm;
    int sret = spgmr(&kc, pp, bb, eps, uu, &jac_current, &res_norm);
    if (sret != 0 && sret != 1)
    {
      stats->ncfl++;
      ret = 8;
      break;
    }
    /* sJpnorm, sfdotJp (KS/kinspgmr.c:384-398): J p by KINSpgmrAtimes, the
     * analytic matvec or the difference quotient */
    if (!st->use_jacobian)
      atimes_dq(&kc, uu, pp, bb);
    else
    {
      if (!jac_current)
      {
        pfo_jacobian(pb, dt, uu, 0, kc.J);
        jac_current = 1;
      }
      pfo_matvec7(pb, kc.J, pp, bb);
    }
    sJpnorm = sqrt(dot(bb, bb, N));
    sfdotJp = dot(fval, bb, N);

    int globalret = 0, maxStepTaken = 0;
    double fnormp, f1normp;
    if (st->globalization == 1)
    {
      /* KINInexactNewton (KS/kinsol.c:1152-1208): the full step, shortened
       * to mxnewtstep; no constraints are set */
      double pnorm = sqrt(dot(pp, pp, N));
      double ratio = 1.0;
      if (pnorm > mxnewtstep)
      {
        ratio = mxnewtstep / pnorm;
        for (long q = 0; q < N; q++) pp[q] *= ratio;
        pnorm = mxnewtstep;
      }
      sfdotJp = sfdotJp * ratio;
      sJpnorm = sJpnorm * ratio;
      for (long q = 0; q < N; q++) unew[q] = uu[q] + pp[q];
      feval(&kc, unew, fval);
      fnormp = sqrt(dot(fval, fval, N));
      f1normp = 0.5 * fnormp * fnormp;
      if (pnorm > 0.99 * mxnewtstep) maxStepTaken = 1;
      goto ls_done;
    }
    /* KINLineSearch (KS/kinsol.c:1228-1420) */
    {
      double pnorm = sqrt(dot(pp, pp, N));
      double ratio = 1.0, alpha = 0.0001, beta = 0.9;
      double rl, rlmin, rlength, slpi, rlprev = 0.0, rlmax, rllo, rldiff, rlincr, alpha_cond, beta_cond;
      if (pnorm > mxnewtstep)
      {
        ratio = mxnewtstep / pnorm;
        for (long q = 0; q < N; q++) pp[q] *= ratio;
        pnorm = mxnewtstep;
      }
      double stepl = pnorm;
      slpi = sfdotJp * ratio;
      rlength = 0.0;
      for (long q = 0; q < N; q++)
      {
        double v = pp[q] / (1.0 / 1.0 + fabs(uu[q]));
        if (fabs(v) > rlength) rlength = fabs(v);
      }
      rlmin = scsteptol / rlength;
      rl = 1.0;
      int nfesav = stats->nfe;
      for (;;)
      {
        for (long q = 0; q < N; q++) unew[q] = uu[q] + rl * pp[q];
        feval(&kc, unew, fval);
        fnormp = sqrt(dot(fval, fval, N));
        f1normp = 0.5 * fnormp * fnormp;
        alpha_cond = f1norm + alpha * slpi * rl;
        if (f1normp <= alpha_cond)
          break;
        if (rl < rlmin)
        {
          memcpy(unew, uu, N * sizeof(double));
          feval(&kc, unew, fval);
          fnormp = sqrt(dot(fval, fval, N));
          f1normp = 0.5 * fnormp * fnormp;
          stats->nbktrk = stats->nfe - nfesav - 1;
          globalret = 1;
          goto ls_done;
        }
        double rltmp = -slpi / (2.0 * (f1normp - f1norm - slpi));
        if (rltmp > 0.5 * rl) rltmp = 0.5 * rl;
        rlprev = rl;
        double pt1trl = 0.1 * rl;
        rl = (pt1trl > rltmp) ? pt1trl : rltmp;
      }
      beta_cond = f1norm + beta * slpi * rl;
      if (f1normp < beta_cond)
      {
        if (rl == 1.0 && pnorm < stepl)
        {
          rlmax = stepl / pnorm;
          do
          {
            rlprev = rl;
            rl = (2.0 * rl < rlmax) ? 2.0 * rl : rlmax;
            for (long q = 0; q < N; q++) unew[q] = uu[q] + rl * pp[q];
            feval(&kc, unew, fval);
            fnormp = sqrt(dot(fval, fval, N));
            f1normp = 0.5 * fnormp * fnormp;
            alpha_cond = f1norm + alpha * slpi * rl;
            beta_cond = f1norm + beta * slpi * rl;
          } while (f1normp <= alpha_cond && f1normp < beta_cond && rl < rlmax);
        }
        if (rl < 1.0 || ((rl > 1.0) && (f1normp > alpha_cond)))
        {
          rllo = (rl < rlprev) ? rl : rlprev;
          rldiff = fabs(rlprev - rl);
          do
          {
            rlincr = 0.5 * rldiff;
            rl = rllo + rlincr;
            for (long q = 0; q < N; q++) unew[q] = uu[q] + rl * pp[q];
            feval(&kc, unew, fval);
            fnormp = sqrt(dot(fval, fval, N));
            f1normp = 0.5 * fnormp * fnormp;
            alpha_cond = f1norm + alpha * slpi * rl;
            beta_cond = f1norm + beta * slpi * rl;
            if (f1normp > alpha_cond)
              rldiff = rlincr;
            else if (f1normp < beta_cond)
            {
              rllo = rl;
              rldiff = rldiff - rlincr;
            }
          } while (f1normp > alpha_cond || ((f1normp < beta_cond) && (rldiff > rlmin)));
          if (f1normp < beta_cond)
          {
            for (long q = 0; q < N; q++) unew[q] = uu[q] + rllo * pp[q];
            feval(&kc, unew, fval);
            fnormp = sqrt(dot(fval, fval, N));
            f1normp = 0.5 * fnormp * fnormp;
            stats->nbcf++;
          }
        }
      }
      stats->nbktrk = stats->nfe - nfesav - 1;
      sfdotJp = sfdotJp * rl * ratio;
      sJpnorm = sJpnorm * rl * ratio;
      if (rl * pnorm > 0.99 * mxnewtstep)
        maxStepTaken = 1;
    }
  ls_done:
    if (stats->nbcf > 10)
    {
      ret = 7;
      break;
    }
    /* KINForcingTerm (KS/kinsol.c:1054-1090) */
    if (callForcingTerm)
    {
      double eta_max = 0.9, eta_min = 0.0001, eta_safe = 0.5;
      if (etaflag == 1)
      {
        double linmodel_norm = sqrt(fnorm * fnorm + 2.0 * sfdotJp + sJpnorm * sJpnorm);
        eta_safe = pow(eta, ealpha);
        eta = fabs(fnormp - linmodel_norm) / fnorm;
      }
      if (etaflag == 2)
      {
        eta_safe = egamma * pow(eta, ealpha);
        eta = egamma * pow(fnormp / fnorm, ealpha);
      }
      if (eta_safe < 0.1) eta_safe = 0.0;
      if (eta < eta_safe) eta = eta_safe;
      if (eta < eta_min) eta = eta_min;
      if (eta > eta_max) eta = eta_max;
    }
    fnorm = fnormp;
    /* KINStop (KS/kinsol.c:1507-1589); the preconditioner is always current */
    int sret2 = 0;
    if (globalret == 1)
      sret2 = 3;
    else if (maxabs(fval, N) <= fnormtol)
      sret2 = 1;
    else
    {
      /* KS/kinsol.c:1540-1541 form the step in vtemp1 and pass it to
       * KINScSteplength (:1490-1498), which first overwrites vtemp1 with
       * 1/uscale + |unew| and then divides vtemp1 by itself: every component
       * is 1, and so is the scaled step length */
      double rlength = 0.0;
      for (long q = 0; q < N; q++)
      {
        double w = 1.0 / 1.0 + fabs(unew[q]);
        double v = w / w;
        if (fabs(v) > rlength) rlength = fabs(v);
      }
      if (rlength <= scsteptol)
        sret2 = 2;
      else if (stats->nni >= mxiter)
        sret2 = 4;
      else
      {
        ncscmx = maxStepTaken ? ncscmx + 1 : 0;
        if (ncscmx == 5)
          sret2 = 5;
      }
    }
    memcpy(uu, unew, N * sizeof(double));
    f1norm = f1normp;
    if (sret2 != 0)
    {
      ret = sret2;
      break;
    }
  }
  stats->status = ret;
  stats->fnorm = fnorm;
out:
  for (int s = 0; s < 7; s++) free(kc.J[s]);
  for (int s = 0; s < 5; s++) free(kc.PC[s]);
  for (int s = 0; s < 7; s++) free(kc.PC7[s]);
  pfo_mg_destroy(kc.mg);
  free(fval); free(unew); free(pp); free(bb); free(kc.dq_u); free(kc.dq_f);
}
