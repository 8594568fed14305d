// Device-side problem description and per-cell physics shared by the
// residual, Jacobian and saturation kernels.
//
// Internal layout: interior cells only, x fastest, c = i + nx*(j + ny*k).
// Boundary faces never read a neighbour: their contribution comes from the
// per-face BC tables, which is the net effect of ParFlow's ghost-cell
// insertion / correction / reset sequence for box domains
// (pfsimulator/parflow_lib/nl_function_eval.c:574-610, 979-1233, 2269-2311).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pfgpu {

struct DevProblem {
  int nx, ny, nz;
  long long n;
  double dx, dy, dz;
  double gravity, viscosity, density;
  double porosity, sstorage;
  // van Genuchten: per-cell arrays or (when the pointer is null) scalars
  const double *alpha, *vgn, *sres, *ssat;
  double alpha0, vgn0, sres0, ssat0;
  int vg_from_file;
  const double *kx, *ky, *kz;   // per cell
  // flow-barrier multipliers of the faces to the +x / +y / +z neighbour, or
  // null (1 everywhere)
  const double *fbx, *fby, *fbz;
  // OverlandFlowSpinUp and OverlandSpinupDampP1 / P2 of an OverlandFlow top
  // patch (nl_function_eval.c:1659-1673, richards_jacobian_eval.c:1258-1287,
  // 2044-2057)
  int ov_spinup;
  double ov_p1, ov_p2;
  const double *zmult;          // per layer
  // per z face between layers k and k+1: 1/sep, z_k/(z_k+z_k+1), z_k+1/(z_k+z_k+1)
  const double *zface;          // 3*nz
  double inv_dx, inv_dy, inv_visc;
  int bc_type[6];
  const double *bc_val[6];
  // terrain-following grid: per column (ny*nx) g sin(atan S) and g cos(atan S)
  // of the subsurface slopes; null = flat (0 and g)
  const double *tfg_xs, *tfg_xc, *tfg_ys, *tfg_yc;
  // kinematic (type 2) or diffusive (type 3) overland flow on the z_upper
  // patch: topographic slopes and Manning's n per column (ny*nx),
  // Solver.Overland{Kinematic,Diffusive}.Epsilon
  const double *ov_sx, *ov_sy, *ov_n;
  double ov_eps;
  // old pressure of the step (dense interior), read by the diffusive terms'
  // slope magnitude in the residual and the Jacobian
  const double *ov_pold;
  // relative-permeability lookup table (Geom.domain.RelPerm.NumSamplePoints
  // > 0, problem_phase_rel_perm.c:116-262), or null: krt holds x a d a_der
  // d_der slope slope_der, krt_npts + 1 values each
  const double *krt;
  int krt_method, krt_npts;  // method 0 spline, 1 linear
  double krt_interval, krt_min;
  // land-surface sink/source per cell [1/h] (the evap_trans vector,
  // nl_function_eval.c:533-541), dense interior layout, or null = 0
  const double *et;
  // timestep read from device memory by the residual and Jacobian kernels
  // (a graph captured once serves every dt), or null: the launch's dt
  const double *dtp;
  // thread-block shapes (bx, by) of the residual, Jacobian and matvec
  // launches picked by pfgpu_autotune; (0, 0) = the default heuristic.
  // Host-side launch configuration only: no kernel reads it.
  int tile[3][2];
};

// Gravity terms of the x face between columns i and i+1 (and of the y face
// between rows j and j+1): mean over the two columns of g sin(atan S) and
// g cos(atan S) (nl_function_eval.c:725-733, SlopeUpwindFormulation 0).
__device__ __forceinline__ void tfg_face_x(const DevProblem &P, int i, int j, double &gs,
                                           double &gc) {
  const double g = P.gravity;
  if (!P.tfg_xs) {
    gs = 0.5 * (g * 0.0 + g * 0.0);
    gc = 0.5 * (g * 1.0 + g * 1.0);
    return;
  }
  const long long a = i + (long long)P.nx * j;
  const bool in = i + 1 < P.nx;
  gs = 0.5 * (__ldg(P.tfg_xs + a) + (in ? __ldg(P.tfg_xs + a + 1) : g * 0.0));
  gc = 0.5 * (__ldg(P.tfg_xc + a) + (in ? __ldg(P.tfg_xc + a + 1) : g * 1.0));
}
__device__ __forceinline__ void tfg_face_y(const DevProblem &P, int i, int j, double &gs,
                                           double &gc) {
  const double g = P.gravity;
  if (!P.tfg_ys) {
    gs = 0.5 * (g * 0.0 + g * 0.0);
    gc = 0.5 * (g * 1.0 + g * 1.0);
    return;
  }
  const long long a = i + (long long)P.nx * j;
  const bool in = j + 1 < P.ny;
  gs = 0.5 * (__ldg(P.tfg_ys + a) + (in ? __ldg(P.tfg_ys + a + P.nx) : g * 0.0));
  gc = 0.5 * (__ldg(P.tfg_yc + a) + (in ? __ldg(P.tfg_yc + a + P.nx) : g * 1.0));
}

// ParFlow's mean macros (pfsimulator/parflow_lib/solver.h:42-47)
__device__ __forceinline__ double harmonic(double a, double b) {
  return (a + b) ? (2.0 * a * b) / (a + b) : 0.0;
}
__device__ __forceinline__ double harmonic_dz(double a, double b, double c, double d) {
  return ((c * b) + (a * d)) ? (((c + d) * a * b) / ((b * c) + (a * d))) : 0.0;
}
__device__ __forceinline__ double upstream(double a, double b, double c, double d) {
  return ((a - b) >= 0) ? c : d;
}
__device__ __forceinline__ double amean(double a, double b) { return 0.5 * (a + b); }

struct VG {
  double alpha, n, sres, ssat;
};

__device__ __forceinline__ VG vg_at(const DevProblem &P, long long c) {
  VG v;
  v.alpha = P.alpha ? __ldg(P.alpha + c) : P.alpha0;
  v.n = P.vgn ? __ldg(P.vgn + c) : P.vgn0;
  v.sres = P.sres ? __ldg(P.sres + c) : P.sres0;
  v.ssat = P.ssat ? __ldg(P.ssat + c) : P.ssat0;
  return v;
}

// Saturation (pfsimulator/parflow_lib/problem_saturation.c:221-415)
__device__ __forceinline__ double vg_sat(const DevProblem &P, double p, const VG &v) {
  double m = 1.0 - (1.0 / v.n);
  double s_dif = v.ssat - v.sres;
  if (p >= 0.0) return P.vg_from_file ? v.ssat : s_dif + v.sres;
  double head = fabs(p) / (P.density * P.gravity);
  return s_dif / pow(1.0 + pow(v.alpha * head, v.n), m) + v.sres;
}

__device__ __forceinline__ double vg_dsat(const DevProblem &P, double p, const VG &v) {
  double m = 1.0 - (1.0 / v.n);
  double s_dif = v.ssat - v.sres;
  if (p >= 0.0) return 0.0;
  double head = fabs(p) / (P.density * P.gravity);
  return (m * v.n * v.alpha * pow(v.alpha * head, (v.n - 1))) * s_dif /
         (pow(1.0 + pow(v.alpha * head, v.n), m + 1));
}

// Relative permeability (pfsimulator/parflow_lib/problem_phase_rel_perm.c:788, :981)
// table lookup at a pressure head >= 0: kr (der = 0) or the table's
// derivative (der = 1) (VanGLookupSpline :265-355, linear :357-400, 718-758)
__device__ __forceinline__ double krt_lookup(const DevProblem &P, double head, int der) {
  if (head >= fabs(P.krt_min)) return 0.0;
  const int m1 = P.krt_npts + 1;
  const double *x = P.krt, *a = P.krt + m1, *d = P.krt + 2 * m1, *a_der = P.krt + 3 * m1,
               *d_der = P.krt + 4 * m1, *slope = P.krt + 5 * m1, *slope_der = P.krt + 6 * m1;
  int pt = (int)floor(head / P.krt_interval);
  if (P.krt_method == 1)
    return der ? a_der[pt] + slope_der[pt] * (head - x[pt]) : a[pt] + slope[pt] * (head - x[pt]);
  if (pt > m1) pt = m1 - 1;
  const double *A = der ? a_der : a, *Dd = der ? d_der : d;
  const double x0 = x[pt], x1 = x[pt + 1];
  const double t = (head - x0) / (x1 - x0);
  return (2.0 * pow(t, 3) - 3.0 * pow(t, 2) + 1.0) * A[pt] +
         (pow(t, 3) - 2.0 * pow(t, 2) + t) * (x1 - x0) * Dd[pt] +
         (-2.0 * pow(t, 3) + 3.0 * pow(t, 2)) * (A[pt + 1]) +
         (pow(t, 3) - pow(t, 2)) * (x1 - x0) * (Dd[pt + 1]);
}

__device__ __forceinline__ double vg_kr(const DevProblem &P, double p, double alpha, double n) {
  if (p >= 0.0) return 1.0;
  if (P.krt) return krt_lookup(P, fabs(p) / (P.density * P.gravity), 0);
  double m = 1.0 - (1.0 / n);
  double head = fabs(p) / (P.density * P.gravity);
  double opahn = 1.0 + pow(alpha * head, n);
  double ahnm1 = pow(alpha * head, n - 1);
  double t = 1.0 - ahnm1 / pow(opahn, m);
  return (t * t) / pow(opahn, m / 2);
}

__device__ __forceinline__ double vg_dkr(const DevProblem &P, double p, double alpha, double n) {
  if (p >= 0.0) return 0.0;
  double m = 1.0 - (1.0 / n);
  double head = fabs(p) / (P.density * P.gravity);
  double opahn = 1.0 + pow(alpha * head, n);
  double ahnm1 = pow(alpha * head, n - 1);
  double coeff = 1.0 - ahnm1 * pow(opahn, -m);
  return 2.0 * (coeff / (pow(opahn, (m / 2)))) *
             ((n - 1) * pow(alpha * head, n - 2) * alpha * pow(opahn, -m) -
              ahnm1 * m * pow(opahn, -(m + 1)) * n * alpha * ahnm1) +
         (coeff * coeff) * (m / 2) * pow(opahn, (-(m + 2) / 2)) * n * alpha * ahnm1;
}

// All four van Genuchten quantities of one cell from one log(alpha h) and one
// log1p((alpha h)^n): every power of the reference formulas
// (problem_saturation.c:221-415, problem_phase_rel_perm.c:788, :981) comes
// from two exponentials of these logarithms, one reciprocal of alpha h (for
// the (alpha h)^(n-1), (alpha h)^(n-2) factors), one reciprocal of
// 1 + (alpha h)^n and one square root ((1+A)^(-m/2) = sqrt((1+A)^(-m))).
struct VGAll {
  double kr, dkr, s, ds;
};

__device__ __forceinline__ VGAll vg_all(const DevProblem &P, double p, const VG &v) {
  VGAll r;
  const double s_dif = v.ssat - v.sres;
  if (p >= 0.0) {
    r.kr = 1.0;
    r.dkr = 0.0;
    r.s = P.vg_from_file ? v.ssat : s_dif + v.sres;
    r.ds = 0.0;
    return r;
  }
  const double n = v.n, alpha = v.alpha;
  const double m = 1.0 - (1.0 / n);
  const double head = fabs(p) / (P.density * P.gravity);
  const double ah = alpha * head;
  const double ahn = exp(n * log(ah));     // (alpha h)^n
  const double inv_ah = 1.0 / ah;
  const double ahnm1 = ahn * inv_ah;       // (alpha h)^(n-1)
  const double ahnm2 = ahnm1 * inv_ah;     // (alpha h)^(n-2)
  const double lop = log1p(ahn);           // log(1 + (alpha h)^n)
  const double inv_opm = exp(-m * lop);    // opahn^-m
  const double inv_opm2 = sqrt(inv_opm);   // opahn^(-m/2)
  const double inv_op = 1.0 / (1.0 + ahn);
  const double t = 1.0 - ahnm1 * inv_opm;
  r.kr = (t * t) * inv_opm2;
  r.dkr = 2.0 * (t * inv_opm2) *
              ((n - 1) * ahnm2 * alpha * inv_opm - ahnm1 * m * (inv_opm * inv_op) * n * alpha * ahnm1) +
          (t * t) * (m / 2) * (inv_opm2 * inv_op) * n * alpha * ahnm1;
  r.s = s_dif * inv_opm + v.sres;
  r.ds = (m * n * alpha * ahnm1) * s_dif * (inv_opm * inv_op);
  return r;
}

// ---------------------------------------------------------------------------
// Face fluxes of the residual (nl_function_eval.c:696-854) with the face's
// gravity terms x_dir_g / x_dir_g_c (tfg_face_x).
// a = lower/left cell, b = upper/right cell.
// ---------------------------------------------------------------------------
// flow-barrier multiplier of the face between cell c and its +x / +y / +z
// neighbour (nl_function_eval.c:841-843)
__device__ __forceinline__ double fb_x(const DevProblem &P, long long c) {
  return P.fbx ? __ldg(P.fbx + c) : 1.0;
}
__device__ __forceinline__ double fb_y(const DevProblem &P, long long c) {
  return P.fby ? __ldg(P.fby + c) : 1.0;
}
__device__ __forceinline__ double fb_z(const DevProblem &P, long long c) {
  return P.fbz ? __ldg(P.fbz + c) : 1.0;
}

__device__ __forceinline__ double flux_x(const DevProblem &P, double pa, double pb, double ka,
                                         double kb, double kra, double krb, double zm,
                                         double x_dir_g, double x_dir_g_c) {
  double diff_l = pa - pb;
  double updir = (diff_l * P.inv_dx) * x_dir_g_c - x_dir_g;
  double km = harmonic(ka, kb);
  double up = upstream(updir, 0.0, kra * P.density, krb * P.density);
  double ffx = P.dy * P.dz;
  double u = zm * ffx * 1.0 * km * (diff_l * P.inv_dx) * x_dir_g_c * up * P.inv_visc;
  u += zm * ffx * 1.0 * km * (-x_dir_g) * up * P.inv_visc;
  return u;
}

__device__ __forceinline__ double flux_y(const DevProblem &P, double pa, double pb, double ka,
                                         double kb, double kra, double krb, double zm,
                                         double y_dir_g, double y_dir_g_c) {
  double diff_l = pa - pb;
  double updir = (diff_l * P.inv_dy) * y_dir_g_c - y_dir_g;
  double km = harmonic(ka, kb);
  double up = upstream(updir, 0.0, kra * P.density, krb * P.density);
  double ffy = P.dx * P.dz;
  double u = zm * ffy * 1.0 * km * (diff_l * P.inv_dy) * y_dir_g_c * up * P.inv_visc;
  u += zm * ffy * 1.0 * km * (-y_dir_g) * up * P.inv_visc;
  return u;
}

// z face between layer k (a, below) and k+1 (b, above)
__device__ __forceinline__ double flux_z(const DevProblem &P, double pa, double pb, double ka,
                                         double kb, double kra, double krb, double za,
                                         double zb, int k) {
  const double g = P.gravity, rho = P.density;
  const double inv_sep = __ldg(P.zface + 3 * k);
  double lower = pa * inv_sep - __ldg(P.zface + 3 * k + 1) * rho * g * 1.0;
  double upper = pb * inv_sep + __ldg(P.zface + 3 * k + 2) * rho * g * 1.0;
  double diff_l = lower - upper;
  double ffz = P.dx * P.dy;
  return ffz * 1.0 * 1.0 * harmonic_dz(ka, kb, za, zb) * diff_l *
         upstream(lower, upper, kra * rho, krb * rho) * P.inv_visc;
}

// ---------------------------------------------------------------------------
// Kinematic overland flow on the top layer (overlandflow_eval_Kin.c).  The
// domain top is layer nz-1 in every column and -1 outside the domain, the
// patch index is uniform (no internal patch edges), and the pressure beyond
// the upper x / y edge is a ghost value that never exceeds zero, so it
// enters as 0.  PFMAX(a, 0) as in the reference: (a < 0) ? 0 : a.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pmax0(double a) { return (a < 0.0) ? 0.0 : a; }

struct OvCell {
  double sfx, sfy, sq, n;  // slopes, |S_f|^(1/2) (floored magnitude), Manning's n
};
__device__ __forceinline__ OvCell ov_cell(const DevProblem &P, int i, int j) {
  const long long a = i + (long long)P.nx * j;
  OvCell o;
  o.sfx = __ldg(P.ov_sx + a);
  o.sfy = __ldg(P.ov_sy + a);
  o.n = __ldg(P.ov_n + a);
  double mag = pow(o.sfx * o.sfx + o.sfy * o.sfy, 0.5);
  if (mag < P.ov_eps) mag = P.ov_eps;
  o.sq = pow(fabs(mag), 0.5);
  return o;
}
// pressure of the top cell of column (i, j); 0 beyond the upper edges
__device__ __forceinline__ double p_top(const DevProblem &P, const double *p, int i, int j) {
  if (i >= P.nx || j >= P.ny) return 0.0;
  return p[i + (long long)P.nx * (j + (long long)P.ny * (P.nz - 1))];
}
// upwinded ponded depth of the x face (i | i+1) and the y face (j | j+1)
__device__ __forceinline__ double ov_press_x(const DevProblem &P, const double *p, int i, int j,
                                             const OvCell &o) {
  return upstream(-o.sfx, 0.0, pmax0(p_top(P, p, i, j)), pmax0(p_top(P, p, i + 1, j)));
}
__device__ __forceinline__ double ov_press_y(const DevProblem &P, const double *p, int i, int j,
                                             const OvCell &o) {
  return upstream(-o.sfy, 0.0, pmax0(p_top(P, p, i, j)), pmax0(p_top(P, p, i, j + 1)));
}

// ---------------------------------------------------------------------------
// Overland flow of the OverlandFlow patch type (overlandflow_eval.c): each
// column's flux q = dir(S) |S|^(1/2) / n max(p, 0)^(5/3) along the sign of
// its own slope (dir = -1 for S > 0, +1 for S < 0, 0 for S = 0), upwinded
// between neighbouring columns; no flux outside the domain.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ovf_dir(double s) {
  return (s > 0.0) ? -1.0 : (s < 0.0) ? 1.0 : 0.0;
}
// q of column (i, j) along x (AX) or y; 0 outside the domain
template <bool AX>
__device__ __forceinline__ double ovf_q(const DevProblem &P, const double *p, int i, int j) {
  if (i < 0 || j < 0 || i >= P.nx || j >= P.ny) return 0.0;
  const long long a = i + (long long)P.nx * j;
  const double s = AX ? __ldg(P.ov_sx + a) : __ldg(P.ov_sy + a);
  return ovf_dir(s) * (pow(fabs(s), 0.5) / __ldg(P.ov_n + a)) *
         pow(pmax0(p_top(P, p, i, j)), (5.0 / 3.0));
}
// CALCDER: derivative of a column's own flux, q' = dir 5/3 |S|^(1/2) / n
// max(p, 0)^(2/3), along x (AX) or y
template <bool AX>
__device__ __forceinline__ double ovf_qder(const DevProblem &P, double ptop, int i, int j) {
  const long long a = i + (long long)P.nx * j;
  const double s = AX ? __ldg(P.ov_sx + a) : __ldg(P.ov_sy + a);
  return ovf_dir(s) * (5.0 / 3.0) * (pow(fabs(s), 0.5) / __ldg(P.ov_n + a)) *
         pow(pmax0(ptop), (2.0 / 3.0));
}

// ---------------------------------------------------------------------------
// Diffusive overland flow on the top layer (overlandflow_eval_diffusive.c):
// the friction slope adds the gradient of the ponded depth to the
// topographic slope, S_f = S_0 + (max(p_up, 0) - max(p, 0)) / dx, and its
// magnitude comes from the old pressure.  Same box conventions as the
// kinematic form.  Gather form: a column's terms are computed by every cell
// that needs them (its own, and its +x / +y neighbours).
// ---------------------------------------------------------------------------
struct OvdCol {
  double sx, sy, n;          // topographic slopes, Manning's n
  double pd, pux, puy;       // max(p, 0) at (i,j), (i+1,j), (i,j+1)
  double pdo;                // max(p_old, 0) at (i,j)
  double sfx, sfy;           // friction slopes
  double sfxo, sfyo;         // friction slopes of the old pressure
  double sq;                 // |S_f,old|^(1/2), magnitude floored at eps
};
__device__ __forceinline__ OvdCol ovd_col(const DevProblem &P, const double *p, int i, int j) {
  const long long a = i + (long long)P.nx * j;
  OvdCol o;
  o.sx = __ldg(P.ov_sx + a);
  o.sy = __ldg(P.ov_sy + a);
  o.n = __ldg(P.ov_n + a);
  const double *po = P.ov_pold;
  o.pd = pmax0(p_top(P, p, i, j));
  o.pux = pmax0(p_top(P, p, i + 1, j));
  o.puy = pmax0(p_top(P, p, i, j + 1));
  o.pdo = pmax0(p_top(P, po, i, j));
  const double puxo = pmax0(p_top(P, po, i + 1, j)), puyo = pmax0(p_top(P, po, i, j + 1));
  o.sfx = o.sx + (o.pux - o.pd) / P.dx;
  o.sfy = o.sy + (o.puy - o.pd) / P.dy;
  o.sfxo = o.sx + (puxo - o.pdo) / P.dx;
  o.sfyo = o.sy + (puyo - o.pdo) / P.dy;
  double mag = pow(o.sfxo * o.sfxo + o.sfyo * o.sfyo, 0.5);
  if (mag < P.ov_eps) mag = P.ov_eps;
  o.sq = pow(fabs(mag), 0.5);
  return o;
}
// |S_f|^(1/2) of two slope components, magnitude floored at eps
__device__ __forceinline__ double ovd_sqrt_mag(const DevProblem &P, double a, double b) {
  double m = pow(a * a + b * b, 0.5);
  if (m < P.ov_eps) m = P.ov_eps;
  return pow(fabs(m), 0.5);
}
// CALCFCN (:125-250): the face fluxes q_x (i | i+1), q_y (j | j+1) of a column
__device__ __forceinline__ double ovd_qx(const OvdCol &o) {
  return -(o.sfx / (o.sq * o.n)) * pow(upstream(-o.sfx, 0.0, o.pd, o.pux), (5.0 / 3.0));
}
__device__ __forceinline__ double ovd_qy(const OvdCol &o) {
  return -(o.sfy / (o.sq * o.n)) * pow(upstream(-o.sfy, 0.0, o.pd, o.puy), (5.0 / 3.0));
}
// the edge fixes of CALCFCN for column (i, j): the flux through the lower x
// edge when i = 0 (:179-195; recomputed with the magnitude of the lower y
// fix when j = 0 too, :215-227) and through the lower y edge when j = 0
// (:197-213, whose differences divide by dx, as the reference's do)
__device__ __forceinline__ void ovd_q_edges(const DevProblem &P, const OvdCol &o, int i, int j,
                                            double &qxw, double &qys) {
  double sfxo = o.sfxo, sfx = 0.0;
  qxw = 0.0;
  qys = 0.0;
  if (i == 0) {
    sfx = o.sx + (o.pd - 0.0) / P.dx;
    sfxo = o.sx + (o.pdo - 0.0) / P.dx;
    const double sm = ovd_sqrt_mag(P, sfxo, o.sfyo);
    if (sfx > 0.0) qxw = -(sfx / (sm * o.n)) * pow(o.pd, (5.0 / 3.0));
  }
  if (j == 0) {
    const double sfy = o.sy + (o.pd - 0.0) / P.dx;
    const double sfyo = o.sy + (o.pdo - 0.0) / P.dx;
    const double sm = ovd_sqrt_mag(P, sfxo, sfyo);
    if (sfy > 0.0) qys = -(sfy / (sm * o.n)) * pow(o.pd, (5.0 / 3.0));
    if (i == 0 && sfx > 0.0) qxw = -(sfx / (sm * o.n)) * pow(o.pd, (5.0 / 3.0));
  }
}
// CALCDER (:252-342): derivative terms of a column's x face (i | i+1):
// a = ke(i) = kwns(i+1) (with respect to this column's depth) and
// b = kw(i+1) = kens(i) (with respect to the +x column's depth); likewise y
__device__ __forceinline__ void ovd_der_x(const DevProblem &P, const OvdCol &o, double &a,
                                          double &b) {
  const double dx = P.dx;
  if (o.sfx < 0) {
    a = (5.0 / 3.0) * (-o.sx - (o.pux / dx)) / (o.sq * o.n) * pow(o.pd, (2.0 / 3.0)) +
        (8.0 / 3.0) * pow(o.pd, (5.0 / 3.0)) / (o.sq * o.n * dx);
    b = -pow(o.pd, (5.0 / 3.0)) / (o.sq * o.n * dx);
  } else {
    a = pow(o.pux, (5.0 / 3.0)) / (o.sq * o.n * dx);
    b = (5.0 / 3.0) * (-o.sx + (o.pd / dx)) / (o.sq * o.n) * pow(o.pux, (2.0 / 3.0)) -
        (8.0 / 3.0) * pow(o.pux, (5.0 / 3.0)) / (o.sq * o.n * dx);
  }
}
__device__ __forceinline__ void ovd_der_y(const DevProblem &P, const OvdCol &o, double &a,
                                          double &b) {
  const double dy = P.dy;
  if (o.sfy < 0) {
    a = (5.0 / 3.0) * (-o.sy - (o.puy / dy)) / (o.sq * o.n) * pow(o.pd, (2.0 / 3.0)) +
        (8.0 / 3.0) * pow(o.pd, (5.0 / 3.0)) / (o.sq * o.n * dy);
    b = -pow(o.pd, (5.0 / 3.0)) / (o.sq * o.n * dy);
  } else {
    a = pow(o.puy, (5.0 / 3.0)) / (o.sq * o.n * dy);
    b = (5.0 / 3.0) * (-o.sy + (o.pd / dy)) / (o.sq * o.n) * pow(o.puy, (2.0 / 3.0)) -
        (8.0 / 3.0) * pow(o.puy, (5.0 / 3.0)) / (o.sq * o.n * dy);
  }
}
// the edge fixes of CALCDER for column (i, j) (:343-421): kw / kwns of the
// lower x edge (i = 0) and ks / ksns of the lower y edge (j = 0); the
// corner (i = j = 0) recomputes the x terms with the lower y fix's
// magnitude and, when the x edge slope is negative, clears the y terms
__device__ __forceinline__ void ovd_der_edges(const DevProblem &P, const OvdCol &o, int i, int j,
                                              double &kw, double &kwns, double &ks,
                                              double &ksns) {
  const double dx = P.dx, dy = P.dy;
  double sfxo = o.sfxo, sfx = 0.0;
  const double pux = o.pd;  // the edge fixes take the column's own depth
  if (i == 0) {
    sfx = o.sx + (pux - 0.0) / dx;
    sfxo = o.sx + (o.pdo - 0.0) / dx;
    const double sm = ovd_sqrt_mag(P, sfxo, o.sfyo);
    if (sfx < 0) {
      kw = 0.0;
      kwns = 0.0;
    } else {
      kwns = pow(pux, (5.0 / 3.0)) / (sm * o.n * dx);
      kw = (5.0 / 3.0) * (-o.sx + 0.0) / (sm * o.n) * pow(pux, (2.0 / 3.0)) -
           (8.0 / 3.0) * pow(pux, (5.0 / 3.0)) / (sm * o.n * dx);
    }
  }
  if (j == 0) {
    const double puy = o.pd;
    const double sfy = o.sy + (puy - 0.0) / dy;
    const double sfyo = o.sy + (o.pdo - 0.0) / dy;
    const double sm = ovd_sqrt_mag(P, sfxo, sfyo);
    ksns = 0.0;  // the ghost row's kn, never written
    if (sfy < 0)
      ks = 0.0;
    else
      ks = (5.0 / 3.0) * (-o.sy + 0.0) / (sm * o.n) * pow(puy, (2.0 / 3.0)) -
           (8.0 / 3.0) * pow(puy, (5.0 / 3.0)) / (sm * o.n * dy);
    if (i == 0) {
      if (sfx < 0) {
        ks = 0.0;
      } else {
        kwns = pow(pux, (5.0 / 3.0)) / (sm * o.n * dx);
        kw = (5.0 / 3.0) * (-o.sx + 0.0) / (sm * o.n) * pow(pux, (2.0 / 3.0)) -
             (8.0 / 3.0) * pow(pux, (5.0 / 3.0)) / (sm * o.n * dx);
      }
    }
  }
}

// Face velocities and overland fluxes a residual evaluation writes (all
// dense, x fastest; null pointers are skipped): vx (nz, ny, nx+1) with face i
// between cells i-1 and i, vy (nz, ny+1, nx), vz (nz+1, ny, nx), qx / qy
// (ny, nx) on the top layer of an overland z_upper face.
struct VelOut {
  double *vx, *vy, *vz, *qx, *qy;
};

// Index of a boundary cell in its face table.
__device__ __forceinline__ int face_slot(const DevProblem &P, int face, int i, int j, int k) {
  if (face < 2) return j + P.ny * k;
  if (face < 4) return i + P.nx * k;
  return i + P.nx * j;
}

}  // namespace pfgpu
