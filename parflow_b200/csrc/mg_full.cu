// Semicoarsening multigrid on the full non-symmetric Jacobian
// (Solver.Linear.Preconditioner.PCMatrixType FullJacobian,
// pfsimulator/parflow_lib/kinsol_pc.c:215-246).
//
// The reference hands MGSemi the Jacobian in non-symmetric storage
// (richards_jacobian_eval.c:2246-2258) while the coarse operators stay
// symmetric (mg_semi.c:1071-1072).  The setup loop (mg_semi.c:667-687) then
// writes a coarse cell's lower entries through the symmetric aliasing into
// the upper entries of its lower neighbours, in loop order: an upper entry
// ends up as the lower entry its upper neighbour wrote, where that neighbour
// exists, and the lower entries of the first row / column / plane stay in
// the ghost planes wg / sg / lg.  For a symmetric fine operator both writes
// carry the same value, so the rule also holds for the coarse levels.
//
// Kernels: generic prolongation weights and coarse operator for every level
// (the fine level symmetric with ghost planes, or level 0 non-symmetric), and
// the red/black Gauss-Seidel sweep and residual of the non-symmetric finest
// level.  The coarse levels smooth with the symmetric kernels of
// mg_kernels.cu, whose ghost entries multiply the zero ghost iterate.
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {
namespace {

__device__ __forceinline__ bool in_level(int nx, int ny, int nz, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
}

// coefficient s (0..6 = C W E S N L U) of cell (i,j,k) as the reference's
// setup reads it: the W S L arrays of a non-symmetric level, else the
// neighbour's upper entry or, on the first row / column / plane, the ghost
// plane; zero outside the level
template <typename T>
__device__ __forceinline__ T gcoef(const MGLevel<T> &L, int s, int i, int j, int k) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (!in_level(nx, ny, nz, i, j, k)) return T(0);
  const long long c = i + (long long)nx * (j + (long long)ny * k);
  if (L.lo[0] && (s == 1 || s == 3 || s == 5)) return L.lo[(s - 1) / 2][c];
  switch (s) {
    case 0: return L.a[0][c];
    case 1: return i > 0 ? L.a[1][c - 1] : (L.wg ? L.wg[j + (long long)ny * k] : T(0));
    case 2: return L.a[1][c];
    case 3: return j > 0 ? L.a[2][c - nx] : (L.sg ? L.sg[i + (long long)nx * k] : T(0));
    case 4: return L.a[2][c];
    case 5:
      return k > 0 ? L.a[3][c - (long long)nx * ny] : (L.lg ? L.lg[i + (long long)nx * j] : T(0));
    default: return L.a[3][c];
  }
}

// stencil entries reordered so that 1, 2 lie along the coarsening direction
// (mg_semi.c:478-499), and the inverse map
__device__ __forceinline__ int sq(int dir, int q) {
  const int sx[7] = {0, 1, 2, 3, 4, 5, 6};
  const int sy[7] = {0, 3, 4, 1, 2, 5, 6};
  const int sz[7] = {0, 5, 6, 3, 4, 1, 2};
  return dir == 0 ? sx[q] : dir == 1 ? sy[q] : sz[q];
}
__device__ __forceinline__ int qs(int dir, int s) {
  for (int q = 0; q < 7; q++)
    if (sq(dir, q) == s) return q;
  return 0;
}

template <typename T>
__device__ __forceinline__ T vat(const MGLevel<T> &L, const T *v, int i, int j, int k) {
  if (!in_level(L.nx, L.ny, L.nz, i, j, k)) return T(0);
  return v[i + (long long)L.nx * (j + (long long)L.ny * k)];
}

// prolongation weights at the fine (odd) points along the coarsening
// direction (mg_semi.c:534-575)
template <typename T>
__global__ void __launch_bounds__(256) k_gen_weights(MGLevel<T> F) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= F.nx || j >= F.ny) return;
  const int d = F.dir;
  const int ci = d == 0 ? i : d == 1 ? j : k;
  if (!(ci & 1)) return;
  const long long c = i + (long long)F.nx * (j + (long long)F.ny * k);
  const T ap0 = gcoef(F, sq(d, 0), i, j, k) + gcoef(F, sq(d, 3), i, j, k) +
                gcoef(F, sq(d, 4), i, j, k) + gcoef(F, sq(d, 5), i, j, k) +
                gcoef(F, sq(d, 6), i, j, k);
  if (ap0 != T(0)) {
    F.p1[c] = -gcoef(F, sq(d, 1), i, j, k) / ap0;
    F.p2[c] = -gcoef(F, sq(d, 2), i, j, k) / ap0;
  } else {
    F.p1[c] = T(0);
    F.p2[c] = T(0);
  }
}

// reordered entry q of the coarse cell (ic,jc,kc) as the setup loop computes
// it before any aliasing (mg_semi.c:667-687)
template <typename T>
__device__ __forceinline__ T coarse_entry(const MGLevel<T> &F, int q, int ic, int jc, int kc) {
  const int d = F.dir, ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const int i1 = i - ox, j1 = j - oy, k1 = k - oz;  // fine point below
  const int i2 = i + ox, j2 = j + oy, k2 = k + oz;  // fine point above
  const int s = sq(d, q);
  if (q >= 3)
    return gcoef(F, s, i, j, k) + T(0.5) * gcoef(F, s, i1, j1, k1) +
           T(0.5) * gcoef(F, s, i2, j2, k2);
  if (q == 1) return gcoef(F, s, i, j, k) * vat(F, F.p1, i1, j1, k1);
  if (q == 2) return gcoef(F, s, i, j, k) * vat(F, F.p2, i2, j2, k2);
  return gcoef(F, sq(d, 0), i, j, k) + gcoef(F, sq(d, 3), i, j, k) + gcoef(F, sq(d, 4), i, j, k) +
         gcoef(F, sq(d, 5), i, j, k) + gcoef(F, sq(d, 6), i, j, k) +
         gcoef(F, sq(d, 1), i, j, k) * vat(F, F.p2, i1, j1, k1) +
         gcoef(F, sq(d, 2), i, j, k) * vat(F, F.p1, i2, j2, k2);
}

// the stored coarse coefficient s (0..6) of coarse cell (ic,jc,kc) after the
// setup loop and its aliasing; the centre before its final correction
template <typename T>
__device__ __forceinline__ T stored_entry(const MGLevel<T> &F, const MGLevel<T> &C, int s, int ic,
                                          int jc, int kc) {
  const int d = F.dir;
  switch (s) {
    case 1: return coarse_entry(F, qs(d, 1), ic, jc, kc);
    case 3: return coarse_entry(F, qs(d, 3), ic, jc, kc);
    case 5: return coarse_entry(F, qs(d, 5), ic, jc, kc);
    case 2:
      return ic + 1 < C.nx ? coarse_entry(F, qs(d, 1), ic + 1, jc, kc)
                           : coarse_entry(F, qs(d, 2), ic, jc, kc);
    case 4:
      return jc + 1 < C.ny ? coarse_entry(F, qs(d, 3), ic, jc + 1, kc)
                           : coarse_entry(F, qs(d, 4), ic, jc, kc);
    case 6:
      return kc + 1 < C.nz ? coarse_entry(F, qs(d, 5), ic, jc, kc + 1)
                           : coarse_entry(F, qs(d, 6), ic, jc, kc);
    default: return coarse_entry(F, 0, ic, jc, kc);
  }
}

// coarse operator C E N U, the ghost planes and the centre correction
// ac0 -= (ac3 + ac4 + ac5 + ac6) with the stored transverse entries
// (mg_semi.c:588-760)
template <typename T>
__global__ void __launch_bounds__(256) k_gen_coarse(MGLevel<T> F, MGLevel<T> C) {
  pdl_enter();
  const int ic = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = blockIdx.y * blockDim.y + threadIdx.y;
  const int kc = blockIdx.z;
  if (ic >= C.nx || jc >= C.ny) return;
  const long long cc = ic + (long long)C.nx * (jc + (long long)C.ny * kc);
  const int d = F.dir;
  C.a[1][cc] = stored_entry(F, C, 2, ic, jc, kc);
  C.a[2][cc] = stored_entry(F, C, 4, ic, jc, kc);
  C.a[3][cc] = stored_entry(F, C, 6, ic, jc, kc);
  if (ic == 0 && C.wg) C.wg[jc + (long long)C.ny * kc] = stored_entry(F, C, 1, ic, jc, kc);
  if (jc == 0 && C.sg) C.sg[ic + (long long)C.nx * kc] = stored_entry(F, C, 3, ic, jc, kc);
  if (kc == 0 && C.lg) C.lg[ic + (long long)C.nx * jc] = stored_entry(F, C, 5, ic, jc, kc);
  const T t3 = stored_entry(F, C, sq(d, 3), ic, jc, kc);
  const T t4 = stored_entry(F, C, sq(d, 4), ic, jc, kc);
  const T t5 = stored_entry(F, C, sq(d, 5), ic, jc, kc);
  const T t6 = stored_entry(F, C, sq(d, 6), ic, jc, kc);
  C.a[0][cc] = coarse_entry(F, 0, ic, jc, kc) - (t3 + t4 + t5 + t6);
}

// one colour sweep of red/black Gauss-Seidel on the non-symmetric finest
// level (rb_GS_point.c:342-370; colour 0 = red = (i + j + k) odd); init: the
// first sweep of a zero initial guess, x = b / C (rb_GS_point.c:128-215)
template <typename T>
__global__ void __launch_bounds__(256) k_rb_full(MGLevel<T> L, T *__restrict__ x,
                                                 const T *__restrict__ b, int colour, int init) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= L.nx || j >= L.ny) return;
  if ((colour == 0) != (((i + j + k) & 1) == 1)) return;
  const long long c = i + (long long)L.nx * (j + (long long)L.ny * k);
  const int xo = xb_index(L, i, j, k);
  if (init) {
    x[xo] = b[xo] / L.a[0][c];
    return;
  }
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const long long sy = nx, sz = (long long)nx * ny;
  const T xw = i > 0 ? x[xb_index(L, i - 1, j, k)] : T(0);
  const T xe = i + 1 < nx ? x[xb_index(L, i + 1, j, k)] : T(0);
  const T xs = j > 0 ? x[xb_index(L, i, j - 1, k)] : T(0);
  const T xn = j + 1 < ny ? x[xb_index(L, i, j + 1, k)] : T(0);
  const T xl = k > 0 ? x[xb_index(L, i, j, k - 1)] : T(0);
  const T xu = k + 1 < nz ? x[xb_index(L, i, j, k + 1)] : T(0);
  (void)sy;
  (void)sz;
  const T acc = L.lo[0][c] * xw + L.a[1][c] * xe + L.lo[1][c] * xs + L.a[2][c] * xn +
                L.lo[2][c] * xl + L.a[3][c] * xu;
  x[xo] = (b[xo] - acc) / L.a[0][c];
}

// r = b - A x on the non-symmetric finest level (matvec.c with alpha -1,
// beta 1), r in the natural layout
template <typename T>
__global__ void __launch_bounds__(256) k_res_full(MGLevel<T> L, const T *__restrict__ x,
                                                  const T *__restrict__ b, T *__restrict__ r) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= L.nx || j >= L.ny) return;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const long long c = i + (long long)nx * (j + (long long)ny * k);
  const int xo = xb_index(L, i, j, k);
  T y = -b[xo];
  y += L.a[0][c] * x[xo];
  y += L.lo[0][c] * (i > 0 ? x[xb_index(L, i - 1, j, k)] : T(0));
  y += L.a[1][c] * (i + 1 < nx ? x[xb_index(L, i + 1, j, k)] : T(0));
  y += L.lo[1][c] * (j > 0 ? x[xb_index(L, i, j - 1, k)] : T(0));
  y += L.a[2][c] * (j + 1 < ny ? x[xb_index(L, i, j + 1, k)] : T(0));
  y += L.lo[2][c] * (k > 0 ? x[xb_index(L, i, j, k - 1)] : T(0));
  y += L.a[3][c] * (k + 1 < nz ? x[xb_index(L, i, j, k + 1)] : T(0));
  r[c] = -y;
}

template <typename T>
void level_grid(const MGLevel<T> &L, dim3 &g, dim3 &b) {
  b = dim3(32, 8, 1);
  g = dim3((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz);
}

}  // namespace

template <typename T>
int launch_mg_full_setup(const MGLevel<T> *L, int nl, cudaStream_t st) {
  int k = 0;
  for (int l = 0; l + 1 < nl; l++) {
    dim3 g, b;
    level_grid(L[l], g, b);
    launch_pdl(k_gen_weights<T>, g, b, st, L[l]);
    level_grid(L[l + 1], g, b);
    launch_pdl(k_gen_coarse<T>, g, b, st, L[l], L[l + 1]);
    k += 2;
  }
  return k;
}

template <typename T>
int launch_mg_full_smooth(const MGLevel<T> &L, T *x, const T *b, int zero, int symmetric,
                          cudaStream_t st) {
  dim3 g, bl;
  level_grid(L, g, bl);
  launch_pdl(k_rb_full<T>, g, bl, st, L, x, b, 0, zero);
  launch_pdl(k_rb_full<T>, g, bl, st, L, x, b, 1, 0);
  if (!symmetric) return 2;
  launch_pdl(k_rb_full<T>, g, bl, st, L, x, b, 0, 0);
  return 3;
}

template <typename T>
void launch_mg_full_residual(const MGLevel<T> &L, const T *x, const T *b, T *r,
                             cudaStream_t st) {
  dim3 g, bl;
  level_grid(L, g, bl);
  launch_pdl(k_res_full<T>, g, bl, st, L, x, b, r);
}

template int launch_mg_full_setup<double>(const MGLevel<double> *, int, cudaStream_t);
template int launch_mg_full_setup<float>(const MGLevel<float> *, int, cudaStream_t);
template int launch_mg_full_smooth<double>(const MGLevel<double> &, double *, const double *,
                                           int, int, cudaStream_t);
template int launch_mg_full_smooth<float>(const MGLevel<float> &, float *, const float *, int,
                                          int, cudaStream_t);
template void launch_mg_full_residual<double>(const MGLevel<double> &, const double *,
                                              const double *, double *, cudaStream_t);
template void launch_mg_full_residual<float>(const MGLevel<float> &, const float *,
                                             const float *, float *, cudaStream_t);

}  // namespace pfgpu
