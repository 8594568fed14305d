// Discrete adjoint of the implicit Richards timesteps (no counterpart in the
// reference).  For a trajectory p_0 .. p_N with F_n(p_n, p_{n-1}; theta) = 0
// and an objective g = sum_n g_n(p_n), the multipliers solve, backwards in n,
//
//   J_n^T lambda_n = -dg_n/dp_n - B_{n+1} lambda_{n+1},   B = dF_{n+1}/dp_n,
//
// where J_n is the analytic Jacobian the forward solve assembles at p_n and
// B is diagonal (p_n enters F_{n+1} only through p_old and S_old = S(p_old)).
// The gradient is dg/dtheta = sum_n lambda_n^T dF_n/dtheta for the per-cell
// parameters ln K, van Genuchten alpha and n.  The kernels below are the
// transposed matvec, the right-hand side and the per-step gradient gather.
#include "pfgpu_device.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

namespace {

__device__ __forceinline__ bool ijk(int nx, int ny, int nz, int &i, int &j, int &k) {
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y;
  k = blockIdx.z;
  return i < nx && j < ny && k < nz;
}

inline void shape(int nx, int ny, int nz, dim3 &grid, dim3 &block) {
  int bx = 32;
  while (bx < nx && bx < 128) bx *= 2;
  int by = 128 / bx;
  if (by > ny) by = ny;
  block = dim3(bx, by, 1);
  grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
}

// Derivatives of S and kr with respect to the van Genuchten alpha and n of a
// cell at pressure p (zero where p >= 0: S and kr are constant there).
// A = (alpha h)^n, B = (alpha h)^(n-1), D = 1 + A, m = 1 - 1/n:
// S = s_dif D^-m + s_res, kr = (1 - B D^-m)^2 D^(-m/2).
struct VGDer {
  double s_a, s_n, kr_a, kr_n;
};
__device__ __forceinline__ VGDer vg_param_der(const DevProblem &P, double p, const VG &v) {
  VGDer d{0.0, 0.0, 0.0, 0.0};
  if (p >= 0.0) return d;
  const double a = v.alpha, n = v.n;
  const double m = 1.0 - 1.0 / n;
  const double h = fabs(p) / (P.density * P.gravity);
  const double L = log(a * h);
  const double A = exp(n * L), B = exp((n - 1.0) * L);
  const double D = 1.0 + A, lD = log1p(A);
  const double Dm = exp(-m * lD), Dm2 = exp(-0.5 * m * lD);
  const double T = 1.0 - B * Dm;
  const double s_dif = v.ssat - v.sres;
  // alpha
  {
    const double dA = n * A / a, dB = (n - 1.0) * B / a;
    const double dDm = Dm * (-m * dA / D), dDm2 = Dm2 * (-0.5 * m * dA / D);
    const double dT = -(dB * Dm + B * dDm);
    d.s_a = s_dif * dDm;
    d.kr_a = 2.0 * T * dT * Dm2 + T * T * dDm2;
  }
  // n (dm/dn = 1/n^2)
  {
    const double dm = 1.0 / (n * n);
    const double dA = A * L, dB = B * L;
    const double dDm = Dm * (-dm * lD - m * dA / D);
    const double dDm2 = Dm2 * (-0.5 * dm * lD - 0.5 * m * dA / D);
    const double dT = -(dB * Dm + B * dDm);
    d.s_n = s_dif * dDm;
    d.kr_n = 2.0 * T * dT * Dm2 + T * T * dDm2;
  }
  return d;
}

}  // namespace

// y = J^T x for the 7-array stencil J (C W E S N L U): row c of J^T gathers
// the entries of the neighbouring rows that couple to c
template <typename TJ>
__global__ void k_matvec7_t(int nx, int ny, int nz, JacIn<TJ> J, const double *__restrict__ x,
                            double *__restrict__ y) {
  int i, j, k;
  if (!ijk(nx, ny, nz, i, j, k)) return;
  const long long c = i + (long long)nx * (j + (long long)ny * k);
  const long long sy = nx, sz = (long long)nx * ny;
  double acc = (double)J.c[c] * x[c];
  if (i > 0) acc += (double)J.e[c - 1] * x[c - 1];
  if (i + 1 < nx) acc += (double)J.w[c + 1] * x[c + 1];
  if (j > 0) acc += (double)J.n[c - sy] * x[c - sy];
  if (j + 1 < ny) acc += (double)J.s[c + sy] * x[c + sy];
  if (k > 0) acc += (double)J.u[c - sz] * x[c - sz];
  if (k + 1 < nz) acc += (double)J.l[c + sz] * x[c + sz];
  y[c] = acc;
}

// rhs = -B_{n+1} lambda_{n+1}: the storage (and ponding) coupling of F_{n+1}
// to p_n, evaluated at p_n with its saturation state
__global__ void k_adj_rhs(DevProblem P, const double *__restrict__ p,
                          const double *__restrict__ sat, const double *__restrict__ dsat,
                          const double *__restrict__ lam_next, double *__restrict__ rhs) {
  int i, j, k;
  if (!ijk(P.nx, P.ny, P.nz, i, j, k)) return;
  const long long c = i + (long long)P.nx * (j + (long long)P.ny * k);
  const double rho = P.density, vol = P.dx * P.dy * P.dz, zm = __ldg(P.zmult + k);
  double b = rho * P.porosity * vol * zm * dsat[c] +
             P.sstorage * vol * zm * rho * (sat[c] + p[c] * dsat[c]);
  if (k == P.nz - 1 && (P.bc_type[5] == 2 || P.bc_type[5] == 4) && p[c] > 0.0) b += vol / P.dz;
  rhs[c] = b * lam_next[c];
}

// rhs[cell_m] -= 2 (p[cell_m] - obs_m): the misfit term of this step
__global__ void k_adj_obs(int nobs, const long long *__restrict__ cells,
                          const double *__restrict__ obs, const double *__restrict__ p,
                          double *__restrict__ rhs) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nobs) return;
  const long long c = cells[m];
  rhs[c] += -2.0 * (p[c] - obs[m]);
}

// One step's gradient contribution lambda_n^T dF_n/dtheta, gathered per cell:
// storage terms (S at p_n and at p_{n-1}), the six face fluxes through the
// harmonic mean of K and the upwind kr, and Dirichlet boundary faces.
__global__ void k_adj_grad(DevProblem P, const double *__restrict__ p,
                           const double *__restrict__ p_prev, const double *__restrict__ lam,
                           const double *__restrict__ kr, double dt,
                           double *__restrict__ g_lnk, double *__restrict__ g_a,
                           double *__restrict__ g_n) {
  int i, j, k;
  if (!ijk(P.nx, P.ny, P.nz, i, j, k)) return;
  const long long c = i + (long long)P.nx * (j + (long long)P.ny * k);
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double rho = P.density, g = P.gravity;
  const double vol = P.dx * P.dy * P.dz, zm = __ldg(P.zmult + k);
  const double ffx = P.dy * P.dz, ffy = P.dx * P.dz, ffz = P.dx * P.dy;
  const VG v = vg_at(P, c);
  const double pc = p[c], lc = lam[c];
  const VGDer d = vg_param_der(P, pc, v), d0 = vg_param_der(P, p_prev[c], v);
  double ga = 0.0, gn = 0.0, gk = 0.0;

  // storage
  const double cs = rho * P.porosity * vol * zm, css = P.sstorage * vol * zm * rho;
  ga += lc * (cs * (d.s_a - d0.s_a) + css * (pc * d.s_a - p_prev[c] * d0.s_a));
  gn += lc * (cs * (d.s_n - d0.s_n) + css * (pc * d.s_n - p_prev[c] * d0.s_n));

  // x and y faces: u = km * Q * up with Q = zm ff ((diff/dd) g_c - g_s) / visc;
  // ln K scales every direction's permeability of the cell
  auto face_xy = [&](const double *K, long long a, long long b, bool c_is_a, double ff,
                     double inv_dd, double gs, double gc) {
    const double Ka = __ldg(K + a), Kb = __ldg(K + b);
    const double diff = p[a] - p[b];
    const double updir = (diff * inv_dd) * gc - gs;
    const double km = harmonic(Ka, Kb);
    const double Q = zm * ff * ((diff * inv_dd) * gc - gs) * P.inv_visc;
    const double up = upstream(updir, 0.0, kr[a] * rho, kr[b] * rho);
    const double w = dt * (lam[a] - lam[b]);
    if (Ka + Kb > 0.0) gk += w * km * Q * up * (c_is_a ? Kb : Ka) / (Ka + Kb);
    const bool c_up = c_is_a ? (updir >= 0.0) : !(updir >= 0.0);
    if (c_up) {
      ga += w * km * Q * rho * d.kr_a;
      gn += w * km * Q * rho * d.kr_n;
    }
  };
  double gs, gcv;
  if (i + 1 < P.nx) {
    tfg_face_x(P, i, j, gs, gcv);
    face_xy(P.kx, c, c + 1, true, ffx, P.inv_dx, gs, gcv);
  }
  if (i > 0) {
    tfg_face_x(P, i - 1, j, gs, gcv);
    face_xy(P.kx, c - 1, c, false, ffx, P.inv_dx, gs, gcv);
  }
  if (j + 1 < P.ny) {
    tfg_face_y(P, i, j, gs, gcv);
    face_xy(P.ky, c, c + sy, true, ffy, P.inv_dy, gs, gcv);
  }
  if (j > 0) {
    tfg_face_y(P, i, j - 1, gs, gcv);
    face_xy(P.ky, c - sy, c, false, ffy, P.inv_dy, gs, gcv);
  }

  // z faces between layers kl and kl+1: u = hdz * ffz * diff / visc * up
  auto face_z = [&](long long a, long long b, int kl, bool c_is_a) {
    const double Ka = __ldg(P.kz + a), Kb = __ldg(P.kz + b);
    const double za = __ldg(P.zmult + kl), zb = __ldg(P.zmult + kl + 1);
    const double inv_sep = __ldg(P.zface + 3 * kl);
    const double lower = p[a] * inv_sep - __ldg(P.zface + 3 * kl + 1) * rho * g;
    const double upper = p[b] * inv_sep + __ldg(P.zface + 3 * kl + 2) * rho * g;
    const double diff = lower - upper;
    const double hdz = harmonic_dz(Ka, Kb, za, zb);
    const double Q = ffz * diff * P.inv_visc;
    const double up = upstream(lower, upper, kr[a] * rho, kr[b] * rho);
    const double w = dt * (lam[a] - lam[b]);
    const double den = Kb * za + Ka * zb;
    if (den != 0.0) gk += w * hdz * Q * up * (c_is_a ? Kb * za : Ka * zb) / den;
    const bool c_up = c_is_a ? (diff >= 0.0) : !(diff >= 0.0);
    if (c_up) {
      ga += w * hdz * Q * rho * d.kr_a;
      gn += w * hdz * Q * rho * d.kr_n;
    }
  };
  if (k + 1 < P.nz) face_z(c, c + sz, k, true);
  if (k > 0) face_z(c - sz, c, k - 1, false);

  // Dirichlet faces: u_new is linear in K_c; the upwind kr is the ghost's
  // (the face value with this cell's VG parameters) or this cell's
  const bool onf[6] = {i == 0, i == P.nx - 1, j == 0, j == P.ny - 1, k == 0, k == P.nz - 1};
  const double krc = kr[c];
#pragma unroll
  for (int face = 0; face < 6; face++) {
    if (!onf[face] || P.bc_type[face] != 1) continue;
    const double value = __ldg(P.bc_val[face] + face_slot(P, face, i, j, k));
    const double dir = (face & 1) ? 1.0 : -1.0;
    const double krg = vg_kr(P, value, v.alpha, v.n);
    const VGDer dg = vg_param_der(P, value, v);
    double base, u_kr_a, u_kr_n, u_new;  // u_new = up * base
    bool ghost_up;
    if (face < 4) {
      const double h = (face < 2) ? ffx * zm : ffy * zm;
      const double dd = (face < 2) ? P.dx : P.dy;
      const double diff = (dir < 0) ? value - pc : pc - value;
      const double kk = (face < 2) ? __ldg(P.kx + c) : __ldg(P.ky + c);
      base = h * (kk * P.inv_visc) * 2.0 * (diff / dd);
      ghost_up = (dir < 0) ? (value - pc >= 0.0) : !(pc - value >= 0.0);
    } else {
      const double sep = P.dz * zm;
      double lower, upper;
      if (dir < 0) {
        lower = value / sep - 0.25 * rho * g;
        upper = pc / sep + 0.25 * rho * g;
        ghost_up = (lower - upper >= 0.0);
      } else {
        lower = (pc / sep) - 0.25 * rho * g;
        upper = (value / sep) + 0.25 * rho * g;
        ghost_up = !(lower - upper >= 0.0);
      }
      base = ffz * (__ldg(P.kz + c) * P.inv_visc) * 2.0 * (lower - upper);
    }
    const double up = ghost_up ? krg * rho : krc * rho;
    u_new = up * base;
    u_kr_a = (ghost_up ? dg.kr_a : d.kr_a) * rho * base;
    u_kr_n = (ghost_up ? dg.kr_n : d.kr_n) * rho * base;
    const double w = dt * dir * lc;
    gk += w * u_new;
    ga += w * u_kr_a;
    gn += w * u_kr_n;
  }
  g_lnk[c] += gk;
  g_a[c] += ga;
  g_n[c] += gn;
}

__global__ void k_gather(int n, const long long *__restrict__ idx, const double *__restrict__ src,
                         double *__restrict__ dst) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) dst[m] = src[idx[m]];
}

void launch_gather(int n, const long long *idx, const double *src, double *dst, cudaStream_t st) {
  if (n <= 0) return;
  k_gather<<<(n + 127) / 128, 128, 0, st>>>(n, idx, src, dst);
}

template <typename TJ>
void launch_matvec7_t(int nx, int ny, int nz, JacIn<TJ> J, const double *x, double *y,
                      cudaStream_t st) {
  dim3 g, b;
  shape(nx, ny, nz, g, b);
  k_matvec7_t<TJ><<<g, b, 0, st>>>(nx, ny, nz, J, x, y);
}
template void launch_matvec7_t<float>(int, int, int, JacIn<float>, const double *, double *,
                                      cudaStream_t);
template void launch_matvec7_t<double>(int, int, int, JacIn<double>, const double *, double *,
                                       cudaStream_t);

void launch_adj_rhs(const DevProblem &P, const double *p, const double *sat, const double *dsat,
                    const double *lam_next, double *rhs, cudaStream_t st) {
  dim3 g, b;
  shape(P.nx, P.ny, P.nz, g, b);
  k_adj_rhs<<<g, b, 0, st>>>(P, p, sat, dsat, lam_next, rhs);
}

void launch_adj_obs(int nobs, const long long *cells, const double *obs, const double *p,
                    double *rhs, cudaStream_t st) {
  if (nobs <= 0) return;
  k_adj_obs<<<(nobs + 127) / 128, 128, 0, st>>>(nobs, cells, obs, p, rhs);
}

void launch_adj_grad(const DevProblem &P, const double *p, const double *p_prev,
                     const double *lam, const double *kr, double dt, double *g_lnk, double *g_a,
                     double *g_n, cudaStream_t st) {
  dim3 g, b;
  shape(P.nx, P.ny, P.nz, g, b);
  k_adj_grad<<<g, b, 0, st>>>(P, p, p_prev, lam, kr, dt, g_lnk, g_a, g_n);
}

}  // namespace pfgpu
