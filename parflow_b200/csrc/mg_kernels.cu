// Semicoarsening multigrid (MGSemi) kernels, templated on the storage and
// arithmetic type (double for the plain FP64 solver, float for the mixed
// solver).  Every level holds a symmetric 7-point operator as C E N U; the
// lower entries are the upper entries of the neighbour (W(i) = E(i-1) etc.,
// pfsimulator/parflow_lib/matrix.c:258-310, 477-490).  Coarse grids take the
// even fine indices in the coarsening direction; fine points are the odd ones
// (pfsimulator/parflow_lib/mg_semi.c:960-1058).
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

template <typename T>
struct LV {
  int nx, ny, nz;
  long long n;
  const T *a0, *ae, *an, *au;
};

template <typename T>
__device__ __forceinline__ LV<T> lv(const MGLevel<T> &L) {
  LV<T> v;
  v.nx = L.nx; v.ny = L.ny; v.nz = L.nz; v.n = L.n;
  v.a0 = L.a[0]; v.ae = L.a[1]; v.an = L.a[2]; v.au = L.a[3];
  return v;
}

__device__ __forceinline__ bool inside(int nx, int ny, int nz, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
}

// coefficient s (0..6 = C W E S N L U) of cell (i,j,k), zero outside
template <typename T>
__device__ __forceinline__ T coef(const LV<T> &L, int s, int i, int j, int k) {
  if (!inside(L.nx, L.ny, L.nz, i, j, k)) return T(0);
  long long c = i + (long long)L.nx * (j + (long long)L.ny * k);
  switch (s) {
    case 0: return L.a0[c];
    case 1: return i > 0 ? L.ae[c - 1] : T(0);
    case 2: return L.ae[c];
    case 3: return j > 0 ? L.an[c - L.nx] : T(0);
    case 4: return L.an[c];
    case 5: return k > 0 ? L.au[c - (long long)L.nx * L.ny] : T(0);
    default: return L.au[c];
  }
}

template <typename T>
__device__ __forceinline__ T vget(int nx, int ny, int nz, const T *v, int i, int j, int k) {
  if (!inside(nx, ny, nz, i, j, k)) return T(0);
  return v[i + (long long)nx * (j + (long long)ny * k)];
}

// stencil entries reordered so that 1, 2 lie along the coarsening direction
// (pfsimulator/parflow_lib/mg_semi.c:478-499)
__device__ __forceinline__ int snum(int dir, int q) {
  const int sx[7] = {0, 1, 2, 3, 4, 5, 6};
  const int sy[7] = {0, 3, 4, 1, 2, 5, 6};
  const int sz[7] = {0, 5, 6, 3, 4, 1, 2};
  return dir == 0 ? sx[q] : dir == 1 ? sy[q] : sz[q];
}

// (i, j, k) of a thread in a 3-D launch: x from blockIdx.x/threadIdx.x,
// y from blockIdx.y/threadIdx.y, one plane per blockIdx.z (no integer division)
__device__ __forceinline__ void thread_ijk(int &i, int &j, int &k) {
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y;
  k = blockIdx.z;
}
// (i, j, k) of linear index t inside a level (32-bit; single-block loops)
__device__ __forceinline__ void split_ijk(int t, int nx, int ny, int &i, int &j, int &k) {
  i = t % nx;
  const int r = t / nx;
  j = r % ny;
  k = r / ny;
}

// prolongation weights of one fine point (mg_semi.c:534-575): the
// along-direction entries over the collapsed diagonal
template <typename T>
__device__ __forceinline__ void weights_at(const LV<T> &L, int d, int i, int j, int k, T &w1,
                                           T &w2) {
  T ap0 = coef(L, snum(d, 0), i, j, k) + coef(L, snum(d, 3), i, j, k) +
          coef(L, snum(d, 4), i, j, k) + coef(L, snum(d, 5), i, j, k) +
          coef(L, snum(d, 6), i, j, k);
  if (ap0 != T(0)) {
    w1 = -coef(L, snum(d, 1), i, j, k) / ap0;
    w2 = -coef(L, snum(d, 2), i, j, k) / ap0;
  } else {
    w1 = T(0);
    w2 = T(0);
  }
}

// prolongation weights at fine points (mg_semi.c:534-575)
template <typename T>
__device__ __forceinline__ void prolong_weights_cell(const MGLevel<T> &F, int i, int j, int k) {
  if (i >= F.nx || j >= F.ny || k >= F.nz) return;
  const long long c = i + (long long)F.nx * (j + (long long)F.ny * k);
  int ci = F.dir == 0 ? i : F.dir == 1 ? j : k;
  if (!(ci & 1)) return;
  LV<T> L = lv(F);
  T w1, w2;
  weights_at(L, F.dir, i, j, k, w1, w2);
  F.p1[c] = w1;
  F.p2[c] = w2;
}

template <typename T>
__global__ void k_prolong_weights(MGLevel<T> F) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  prolong_weights_cell(F, i, j, k);
}

// collapsed-stencil coarse operator (mg_semi.c:577-740), stored symmetric:
// the along-direction upper entry of coarse point c is the value ParFlow
// leaves there last, i.e. the lower entry written for c+1 when it exists.
// p2_1 = p2 at fine 2c-1, p1_2 / p2_2 = p1 / p2 at fine 2c+1 (zero outside).
template <typename T>
__device__ __forceinline__ void coarse_op_core(const MGLevel<T> &F, const MGLevel<T> &C, int ic,
                                               int jc, int kc, T p2_1, T p1_2, T p2_2) {
  const long long cc = ic + (long long)C.nx * (jc + (long long)C.ny * kc);
  const int d = F.dir;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const int i1 = i - ox, j1 = j - oy, k1 = k - oz;
  const int i2 = i + ox, j2 = j + oy, k2 = k + oz;
  LV<T> L = lv(F);
  T ac[7];
#pragma unroll
  for (int q = 3; q <= 6; q++)
    ac[q] = coef(L, snum(d, q), i, j, k) + T(0.5) * coef(L, snum(d, q), i1, j1, k1) +
            T(0.5) * coef(L, snum(d, q), i2, j2, k2);
  ac[2] = coef(L, snum(d, 2), i, j, k) * p2_2;
  ac[0] = coef(L, snum(d, 0), i, j, k) + coef(L, snum(d, 3), i, j, k) +
          coef(L, snum(d, 4), i, j, k) + coef(L, snum(d, 5), i, j, k) +
          coef(L, snum(d, 6), i, j, k) + coef(L, snum(d, 1), i, j, k) * p2_1 +
          coef(L, snum(d, 2), i, j, k) * p1_2;
  const int last = d == 0 ? (ic + 1 >= C.nx) : d == 1 ? (jc + 1 >= C.ny) : (kc + 1 >= C.nz);
  T along_up;
  if (last) {
    along_up = ac[2];
  } else {
    // lower entry of coarse point c+1: a1(fine 2c+2) * p1(fine 2c+1)
    along_up = coef(L, snum(d, 1), i + 2 * ox, j + 2 * oy, k + 2 * oz) * p1_2;
  }
  T E, N, U;
  if (d == 0) { E = along_up; N = ac[4]; U = ac[6]; }
  else if (d == 1) { E = ac[4]; N = along_up; U = ac[6]; }
  else { E = ac[6]; N = ac[4]; U = along_up; }
  C.a[1][cc] = E;
  C.a[2][cc] = N;
  C.a[3][cc] = U;
  C.a[0][cc] = ac[0] - (ac[3] + ac[4] + ac[5] + ac[6]);
}

// coarse operator from stored weights (single-block setup tail)
template <typename T>
__device__ __forceinline__ void coarse_op_cell(const MGLevel<T> &F, const MGLevel<T> &C, int ic,
                                               int jc, int kc) {
  if (ic >= C.nx || jc >= C.ny || kc >= C.nz) return;
  const int d = F.dir;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const T p2_1 = vget(F.nx, F.ny, F.nz, (const T *)F.p2, i - ox, j - oy, k - oz);
  const T p1_2 = vget(F.nx, F.ny, F.nz, (const T *)F.p1, i + ox, j + oy, k + oz);
  const T p2_2 = vget(F.nx, F.ny, F.nz, (const T *)F.p2, i + ox, j + oy, k + oz);
  coarse_op_core(F, C, ic, jc, kc, p2_1, p1_2, p2_2);
}

// weights and coarse operator of one level in one pass: the thread of
// coarse point c computes the weights of fine points 2c-1 and 2c+1 itself
// (the same arithmetic as prolong_weights_cell) and stores those of 2c+1,
// so every fine point's weights are written once and the fine operator is
// read in a single sweep
template <typename T>
__device__ __forceinline__ void setup_level_cell(const MGLevel<T> &F, const MGLevel<T> &C,
                                                 int ic, int jc, int kc) {
  if (ic >= C.nx || jc >= C.ny || kc >= C.nz) return;
  const int d = F.dir;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  LV<T> L = lv(F);
  T p2_1 = T(0), p1_2 = T(0), p2_2 = T(0), w1;
  if (inside(F.nx, F.ny, F.nz, i - ox, j - oy, k - oz))
    weights_at(L, d, i - ox, j - oy, k - oz, w1, p2_1);
  if (inside(F.nx, F.ny, F.nz, i + ox, j + oy, k + oz)) {
    weights_at(L, d, i + ox, j + oy, k + oz, p1_2, p2_2);
    const long long f = (i + ox) + (long long)F.nx * ((j + oy) + (long long)F.ny * (k + oz));
    F.p1[f] = p1_2;
    F.p2[f] = p2_2;
  }
  coarse_op_core(F, C, ic, jc, kc, p2_1, p1_2, p2_2);
}

template <typename T>
__global__ void k_setup_level(MGLevel<T> F, MGLevel<T> C) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  setup_level_cell(F, C, i, j, k);
}

template <typename T>
__global__ void k_coarse_op(MGLevel<T> F, MGLevel<T> C) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  coarse_op_cell(F, C, i, j, k);
}

// one colour of red/black Gauss-Seidel; colour 0 = red = (i+j+k) odd
// (pfsimulator/parflow_lib/comm_pkg.c:132-139, rb_GS_point.c:342-370)
template <typename T>
__device__ __forceinline__ void rb_cell(const MGLevel<T> &Lv, T *__restrict__ x,
                                        const T *__restrict__ b, int colour, int init, int q,
                                        int j, int k) {
  // q-th cell of the colour in row (j, k): rows hold alternating colours
  const int nx = Lv.nx, ny = Lv.ny;
  if (j >= ny || k >= Lv.nz) return;
  const int want = colour == 0 ? 1 : 0;  // parity of (i+j+k)
  const int i = 2 * q + ((want ^ (j + k)) & 1);
  if (i >= nx) return;
  const long long c = i + (long long)nx * (j + (long long)ny * k);
  LV<T> L = lv(Lv);
  if (init) {
    x[c] = b[c] / L.a0[c];
    return;
  }
  const long long sy = nx, sz = (long long)nx * ny;
  x[c] = rb_update<T>(L.a0[c], b[c], coef(L, 1, i, j, k), i > 0 ? x[c - 1] : T(0),
                      coef(L, 2, i, j, k), i + 1 < nx ? x[c + 1] : T(0),
                      coef(L, 3, i, j, k), j > 0 ? x[c - sy] : T(0),
                      coef(L, 4, i, j, k), j + 1 < ny ? x[c + sy] : T(0),
                      coef(L, 5, i, j, k), k > 0 ? x[c - sz] : T(0),
                      coef(L, 6, i, j, k), k + 1 < Lv.nz ? x[c + sz] : T(0));
}

template <typename T>
__global__ void k_rb_sweep(MGLevel<T> Lv, T *__restrict__ x, const T *__restrict__ b,
                           int colour, int init) {
  pdl_enter();
  int q, j, k;
  thread_ijk(q, j, k);
  rb_cell(Lv, x, b, colour, init, q, j, k);
}

// weighted Jacobi (pfsimulator/parflow_lib/w_jacobi.c:120-290)
template <typename T>
__device__ __forceinline__ void wjacobi_cell(const MGLevel<T> &Lv, const T *__restrict__ x,
                                             const T *__restrict__ b, T *__restrict__ t,
                                             int zero, int i, int j, int k) {
  if (i >= Lv.nx || j >= Lv.ny || k >= Lv.nz) return;
  const long long c = i + (long long)Lv.nx * (j + (long long)Lv.ny * k);
  LV<T> L = lv(Lv);
  if (zero) {
    t[c] = b[c] / L.a0[c];
    return;
  }
  const int nx = Lv.nx, ny = Lv.ny, nz = Lv.nz;
  T v = b[c];
  v -= coef(L, 1, i, j, k) * vget(nx, ny, nz, x, i - 1, j, k);
  v -= coef(L, 2, i, j, k) * vget(nx, ny, nz, x, i + 1, j, k);
  v -= coef(L, 3, i, j, k) * vget(nx, ny, nz, x, i, j - 1, k);
  v -= coef(L, 4, i, j, k) * vget(nx, ny, nz, x, i, j + 1, k);
  v -= coef(L, 5, i, j, k) * vget(nx, ny, nz, x, i, j, k - 1);
  v -= coef(L, 6, i, j, k) * vget(nx, ny, nz, x, i, j, k + 1);
  t[c] = v / L.a0[c];
}

template <typename T>
__global__ void k_wjacobi(MGLevel<T> Lv, const T *__restrict__ x, const T *__restrict__ b,
                          T *__restrict__ t, int zero) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  wjacobi_cell(Lv, x, b, t, zero, i, j, k);
}

template <typename T>
__device__ __forceinline__ void wjacobi_update_cell(T *__restrict__ x, const T *__restrict__ t,
                                                    long long n, T w, int zero, long long c) {
  if (c >= n) return;
  if (zero)
    x[c] = (w != T(1)) ? t[c] * w : t[c];
  else
    x[c] = (w != T(1)) ? (T(1) - w) * x[c] + w * t[c] : t[c];
}

template <typename T>
__global__ void k_wjacobi_update(T *__restrict__ x, const T *__restrict__ t, long long n,
                                 T w, int zero) {
  pdl_enter();
  wjacobi_update_cell(x, t, n, w, zero, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// r = b - A x in ParFlow's Matvec order (alpha = -1, beta = 1)
template <typename T>
__device__ __forceinline__ void mg_residual_cell(const MGLevel<T> &Lv, const T *__restrict__ x,
                                                 const T *__restrict__ b, T *__restrict__ r,
                                                 int i, int j, int k) {
  if (i >= Lv.nx || j >= Lv.ny || k >= Lv.nz) return;
  const long long c = i + (long long)Lv.nx * (j + (long long)Lv.ny * k);
  const int nx = Lv.nx, ny = Lv.ny, nz = Lv.nz;
  LV<T> L = lv(Lv);
  T y = -b[c];
  y += L.a0[c] * x[c];
  y += coef(L, 1, i, j, k) * vget(nx, ny, nz, x, i - 1, j, k);
  y += coef(L, 2, i, j, k) * vget(nx, ny, nz, x, i + 1, j, k);
  y += coef(L, 3, i, j, k) * vget(nx, ny, nz, x, i, j - 1, k);
  y += coef(L, 4, i, j, k) * vget(nx, ny, nz, x, i, j + 1, k);
  y += coef(L, 5, i, j, k) * vget(nx, ny, nz, x, i, j, k - 1);
  y += coef(L, 6, i, j, k) * vget(nx, ny, nz, x, i, j, k + 1);
  r[c] = -y;
}

template <typename T>
__global__ void k_mg_residual(MGLevel<T> Lv, const T *__restrict__ x, const T *__restrict__ b,
                              T *__restrict__ r) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  mg_residual_cell(Lv, x, b, r, i, j, k);
}

// r_c = r_f(c) + (p2(f-1) r_f(f-1) + p1(f+1) r_f(f+1)) (mg_semi_restrict.c:161-169)
template <typename T>
__device__ __forceinline__ void restrict_cell(const MGLevel<T> &F, const MGLevel<T> &C,
                                              const T *__restrict__ rf, T *__restrict__ rc,
                                              int ic, int jc, int kc) {
  if (ic >= C.nx || jc >= C.ny || kc >= C.nz) return;
  const long long cc = ic + (long long)C.nx * (jc + (long long)C.ny * kc);
  const int d = F.dir;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  rc[cc] = rf[i + (long long)nx * (j + (long long)ny * k)] +
           (vget(nx, ny, nz, (const T *)F.p2, i - ox, j - oy, k - oz) *
                vget(nx, ny, nz, rf, i - ox, j - oy, k - oz) +
            vget(nx, ny, nz, (const T *)F.p1, i + ox, j + oy, k + oz) *
                vget(nx, ny, nz, rf, i + ox, j + oy, k + oz));
}

template <typename T>
__global__ void k_restrict(MGLevel<T> F, MGLevel<T> C, const T *__restrict__ rf,
                           T *__restrict__ rc) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  restrict_cell(F, C, rf, rc, i, j, k);
}

// x_f += P e_c: injection at coarse points, p1 e(f-1) + p2 e(f+1) at fine
// points (mg_semi_prolong.c:119-124, 191-197), followed by Axpy(1, e, x)
template <typename T>
__device__ __forceinline__ void prolong_add_cell(const MGLevel<T> &F, const MGLevel<T> &C,
                                                 const T *__restrict__ ec, T *__restrict__ xf,
                                                 int i, int j, int k) {
  if (i >= F.nx || j >= F.ny || k >= F.nz) return;
  const long long c = i + (long long)F.nx * (j + (long long)F.ny * k);
  const int d = F.dir;
  const int ci = d == 0 ? i : d == 1 ? j : k;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  T e;
  if (!(ci & 1)) {
    e = ec[(ox ? i / 2 : i) + (long long)C.nx * ((oy ? j / 2 : j) + (long long)C.ny * (oz ? k / 2 : k))];
  } else {
    int il = i - ox, jl = j - oy, kl = k - oz;  // coarse point below (even)
    int ih = i + ox, jh = j + oy, kh = k + oz;  // coarse point above (even), may be outside
    T el = ec[(ox ? il / 2 : il) + (long long)C.nx * ((oy ? jl / 2 : jl) + (long long)C.ny * (oz ? kl / 2 : kl))];
    T eh = inside(F.nx, F.ny, F.nz, ih, jh, kh)
               ? ec[(ox ? ih / 2 : ih) + (long long)C.nx * ((oy ? jh / 2 : jh) + (long long)C.ny * (oz ? kh / 2 : kh))]
               : T(0);
    e = (F.p1[c] * el + F.p2[c] * eh);
  }
  xf[c] = xf[c] + e;
}

template <typename T>
__global__ void k_prolong_add(MGLevel<T> F, MGLevel<T> C, const T *__restrict__ ec,
                              T *__restrict__ xf) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  prolong_add_cell(F, C, ec, xf, i, j, k);
}

// ---------------------------------------------------------------------------
// The coarse tail of the hierarchy (levels from `first` down to the coarsest)
// in one single-block kernel: each level there holds only a few thousand
// cells, so launching a grid per smoothing sweep costs more than the sweep.
// The block walks the same sequence of phases as the per-level kernels
// (smooth, residual, restrict, ..., coarse solve, prolong + correct, smooth),
// separated by __syncthreads(); the arithmetic per cell is identical.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void blk_smooth(const MGLevel<T> &L, T *x, const T *b, int zero,
                                           int smoother, T w, T *tmp) {
  if (smoother == 1) {
    for (int t = threadIdx.x; t < (int)L.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, L.nx, L.ny, i, j, k);
      wjacobi_cell(L, x, b, tmp, zero, i, j, k);
    }
    __syncthreads();
    for (long long c = threadIdx.x; c < L.n; c += blockDim.x)
      wjacobi_update_cell(x, (const T *)tmp, L.n, w, zero, c);
    __syncthreads();
    return;
  }
  const int hx = (L.nx + 1) / 2;
  const int half = hx * L.ny * L.nz;
  for (int sweep = 0; sweep < 3; sweep++) {
    const int colour = sweep == 1 ? 1 : 0;
    const int init = (sweep == 0) ? zero : 0;
    for (int t = threadIdx.x; t < half; t += blockDim.x) {
      int q, j, k;
      split_ijk(t, hx, L.ny, q, j, k);
      rb_cell(L, x, b, colour, init, q, j, k);
    }
    __syncthreads();
  }
}

// the tail cycle over levels first .. nl-1 of the table Ls (global or shared)
template <typename T>
__device__ __forceinline__ void tail_cycle(const MGLevel<T> *Ls, int first, int nl,
                                           int smoother, T w, T *tmp) {
  // down: levels first .. nl-2
  for (int l = first; l <= nl - 2; l++) {
    const MGLevel<T> L = Ls[l];
    const MGLevel<T> C = Ls[l + 1];
    blk_smooth(L, L.x, (const T *)L.b, 1, smoother, w, tmp);
    for (int t = threadIdx.x; t < (int)L.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, L.nx, L.ny, i, j, k);
      mg_residual_cell(L, (const T *)L.x, (const T *)L.b, L.t, i, j, k);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < (int)C.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, C.nx, C.ny, i, j, k);
      restrict_cell(L, C, (const T *)L.t, C.b, i, j, k);
    }
    __syncthreads();
  }
  // coarse solve: red/black Gauss-Seidel
  {
    const MGLevel<T> L = Ls[nl - 1];
    blk_smooth(L, L.x, (const T *)L.b, 1, 0, T(1), tmp);
  }
  // up: levels nl-2 .. first
  for (int l = nl - 2; l >= first; l--) {
    const MGLevel<T> L = Ls[l];
    const MGLevel<T> C = Ls[l + 1];
    for (int t = threadIdx.x; t < (int)L.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, L.nx, L.ny, i, j, k);
      prolong_add_cell(L, C, (const T *)C.x, L.x, i, j, k);
    }
    __syncthreads();
    blk_smooth(L, L.x, (const T *)L.b, 0, smoother, w, tmp);
  }
}

// Tail levels in global memory (used when they do not fit in shared memory).
template <typename T>
__global__ void __launch_bounds__(512) k_vcycle_tail(const MGLevel<T> *__restrict__ Ls,
                                                      int first, int nl, int smoother, T w,
                                                      T *tmp) {
  pdl_enter();
  tail_cycle(Ls, first, nl, smoother, w, tmp);
}

// Tail levels in shared memory: the block copies every tail level's C E N U,
// prolongation weights and the first tail level's right-hand side into
// shared memory (x and b of the coarser levels live there too, plus one
// scratch vector for residuals and Jacobi updates), runs the cycle with each
// phase waiting on shared-memory rather than L2 latency, and writes the first
// tail level's x back.  The copy-in is one flattened loop over all arrays
// with eight loads in flight per thread.
template <typename T>
struct TailSeg {
  T *dst;
  const T *src;
  int start;  // first flattened element of this array
};

template <typename T>
__host__ __device__ inline long long tail_pad(long long n) {
  const long long q = 16 / (long long)sizeof(T);
  return (n + q - 1) / q * q;
}

template <typename T>
__global__ void __launch_bounds__(TAIL_THREADS) k_vcycle_tail_smem(
    const MGLevel<T> *__restrict__ Ls, int first, int nl, int smoother, T w) {
  extern __shared__ __align__(16) unsigned char tail_raw[];
  __shared__ MGLevel<T> S[TAIL_MAX_LEVELS];
  __shared__ TailSeg<T> seg[7 * TAIL_MAX_LEVELS + 1];
  __shared__ int nseg;
  pdl_enter();
  const int nt = nl - first;
  if ((int)threadIdx.x < nt) S[threadIdx.x] = Ls[first + threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    T *p = reinterpret_cast<T *>(tail_raw);
    int ns = 0, e = 0, maxn = 0;
    auto place = [&](T *&ptr, int n, bool load) {
      if (load) {
        seg[ns].dst = p;
        seg[ns].src = ptr;
        seg[ns].start = e;
        ns++;
        e += n;
      }
      ptr = p;
      p += tail_pad<T>(n);
    };
    for (int q = 0; q < nt; q++) {
      MGLevel<T> &L = S[q];
      const int n = (int)L.n;
      for (int s = 0; s < 4; s++) place(L.a[s], n, true);
      place(L.x, n, false);
      place(L.b, n, q == 0);
      if (q < nt - 1) {
        place(L.p1, n, true);
        place(L.p2, n, true);
      }
      maxn = n > maxn ? n : maxn;
    }
    for (int q = 0; q < nt; q++) S[q].t = p;
    seg[ns].start = e;  // sentinel
    nseg = ns;
  }
  __syncthreads();
  const int E = seg[nseg].start;
  int sg = 0;
  for (int e0 = threadIdx.x; e0 < E; e0 += 8 * blockDim.x) {
    T v[8];
    T *d[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * (int)blockDim.x;
      d[u] = nullptr;
      if (e < E) {
        while (seg[sg + 1].start <= e) sg++;
        const int o = e - seg[sg].start;
        v[u] = seg[sg].src[o];
        d[u] = seg[sg].dst + o;
      }
    }
#pragma unroll
    for (int u = 0; u < 8; u++)
      if (d[u]) *d[u] = v[u];
  }
  __syncthreads();
  tail_cycle(S, 0, nt, smoother, w, S[0].t);
  T *xo = Ls[first].x;
  for (int c = threadIdx.x; c < (int)S[0].n; c += blockDim.x) xo[c] = S[0].x[c];
}

template <typename T>
size_t tail_smem_bytes(const MGLevel<T> *L, int first, int nl) {
  if (nl - first > TAIL_MAX_LEVELS) return ~(size_t)0;
  long long elems = 0, maxn = 0;
  for (int q = first; q < nl; q++) {
    elems += tail_pad<T>(L[q].n) * (q < nl - 1 ? 8 : 6);
    maxn = L[q].n > maxn ? L[q].n : maxn;
  }
  elems += tail_pad<T>(maxn);
  return (size_t)elems * sizeof(T);
}

// multigrid setup of the tail levels in one block (mg_semi.c:534-740)
template <typename T>
__global__ void __launch_bounds__(512) k_setup_tail(const MGLevel<T> *__restrict__ Ls,
                                                     int first, int nl) {
  pdl_enter();
  for (int l = first; l <= nl - 2; l++) {
    const MGLevel<T> F = Ls[l];
    const MGLevel<T> C = Ls[l + 1];
    for (int t = threadIdx.x; t < (int)F.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, F.nx, F.ny, i, j, k);
      prolong_weights_cell(F, i, j, k);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < (int)C.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, C.nx, C.ny, i, j, k);
      coarse_op_cell(F, C, i, j, k);
    }
    __syncthreads();
  }
}

// four consecutive elements per vector access (16-byte aligned pointers)
__device__ __forceinline__ void ld4(const double *p, double v[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, float v[4]) {
  const float4 a = reinterpret_cast<const float4 *>(p)[0];
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void st4(double *p, const double v[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(float *p, const float v[4]) {
  reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
}

// out = (TO) in; with vec set (both pointers 16-byte aligned) each thread
// moves four elements per vector access, which keeps enough bytes in flight
// for a streaming conversion to run at HBM bandwidth
template <typename TI, typename TO>
__global__ void k_convert(const TI *__restrict__ in, TO *__restrict__ out, long long n,
                          int vec) {
  pdl_enter();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n4 = vec ? n / 4 : 0;
  if (t < n4) {
    TI a[4];
    TO b[4];
    ld4(in + 4 * t, a);
#pragma unroll
    for (int u = 0; u < 4; u++) b[u] = (TO)a[u];
    st4(out + 4 * t, b);
  }
  const long long c = 4 * n4 + t;
  if (c < n && t < (vec ? 4 : n)) out[c] = (TO)in[c];
}

// ---------------------------------------------------------------------------
static inline unsigned nb(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// 3-D launch shape covering (nx, ny, nz): x in warps, rows stacked in y
struct Shape3 {
  dim3 grid, block;
};
static inline Shape3 shape3(int nx, int ny, int nz) {
  int bx = 32;
  while (bx < nx && bx < 128) bx *= 2;
  if (nx <= 16) bx = nx <= 1 ? 1 : (nx <= 2 ? 2 : (nx <= 4 ? 4 : (nx <= 8 ? 8 : 16)));
  int by = 256 / bx;
  if (by > ny) by = ny < 1 ? 1 : ny;
  Shape3 s;
  s.block = dim3(bx, by, 1);
  s.grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
  return s;
}

template <typename T>
void launch_mg_prolong_weights(const MGLevel<T> &F, cudaStream_t st) {
  Shape3 g = shape3(F.nx, F.ny, F.nz);
  launch_pdl(k_prolong_weights<T>, dim3(g.grid), dim3(g.block), st, F);
}
template <typename T>
void launch_mg_coarse_op(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st) {
  Shape3 g = shape3(C.nx, C.ny, C.nz);
  launch_pdl(k_coarse_op<T>, dim3(g.grid), dim3(g.block), st, F, C);
}
template <typename T>
void launch_mg_setup_level(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st) {
  Shape3 g = shape3(C.nx, C.ny, C.nz);
  launch_pdl(k_setup_level<T>, dim3(g.grid), dim3(g.block), st, F, C);
}
template <typename T>
static void rb_sweep(const MGLevel<T> &L, T *x, const T *b, int colour, int init,
                     cudaStream_t st) {
  Shape3 g = shape3((L.nx + 1) / 2, L.ny, L.nz);
  launch_pdl(k_rb_sweep<T>, dim3(g.grid), dim3(g.block), st, L, x, b, colour, init);
}
// RedBlackGSPoint, MaxIter 1, Symmetric: red, black, red; a zero initial
// guess turns the first red sweep into x = b / a0 (rb_GS_point.c:107-240)
template <typename T>
void launch_mg_smooth(const MGLevel<T> &L, T *x, const T *b, int zero, int smoother,
                      double weight, T *tmp, cudaStream_t st) {
  if (smoother == 1) {
    Shape3 g = shape3(L.nx, L.ny, L.nz);
    launch_pdl(k_wjacobi<T>, dim3(g.grid), dim3(g.block), st, L, x, b, tmp, zero);
    launch_pdl(k_wjacobi_update<T>, dim3(nb(L.n, 256)), dim3(256), st, x, tmp, L.n, (T)weight,
               zero);
    return;
  }
  if (smoother == 2) {  // a single red sweep (kernel timing)
    rb_sweep(L, x, b, 0, 0, st);
    return;
  }
  rb_sweep(L, x, b, 0, zero, st);
  rb_sweep(L, x, b, 1, 0, st);
  rb_sweep(L, x, b, 0, 0, st);
}
// opt the fused smoother into its dynamic shared memory (> 48 KB); called
// once per device before any launch or graph capture
cudaError_t mg_prepare_kernels() {
  cudaError_t e = rbr_fused_prepare<float>();
  if (e != cudaSuccess) return e;
  e = rbr_fused_prepare<double>();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_vcycle_tail_smem<float>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM_MAX);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_vcycle_tail_smem<double>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM_MAX);
}

template <typename T>
void launch_mg_residual(const MGLevel<T> &L, const T *x, const T *b, T *r, cudaStream_t st) {
  Shape3 g = shape3(L.nx, L.ny, L.nz);
  launch_pdl(k_mg_residual<T>, dim3(g.grid), dim3(g.block), st, L, x, b, r);
}
template <typename T>
void launch_mg_restrict(const MGLevel<T> &F, const MGLevel<T> &C, const T *rf, T *rc,
                        cudaStream_t st) {
  Shape3 g = shape3(C.nx, C.ny, C.nz);
  launch_pdl(k_restrict<T>, dim3(g.grid), dim3(g.block), st, F, C, rf, rc);
}
template <typename T>
void launch_mg_prolong_add(const MGLevel<T> &F, const MGLevel<T> &C, const T *ec, T *xf,
                           cudaStream_t st) {
  Shape3 g = shape3(F.nx, F.ny, F.nz);
  launch_pdl(k_prolong_add<T>, dim3(g.grid), dim3(g.block), st, F, C, ec, xf);
}
template <typename T>
void launch_vcycle_tail(const MGLevel<T> *levels_dev, int first, int nl, int smoother,
                        double weight, T *tmp, size_t smem, cudaStream_t st) {
  if (smem > 0)
    launch_pdl_smem(k_vcycle_tail_smem<T>, dim3(1), dim3(TAIL_THREADS), smem, st, levels_dev,
                    first, nl, smoother, (T)weight);
  else
    launch_pdl(k_vcycle_tail<T>, dim3(1), dim3(512), st, levels_dev, first, nl, smoother,
               (T)weight, tmp);
}
template <typename T>
void launch_setup_tail(const MGLevel<T> *levels_dev, int first, int nl, cudaStream_t st) {
  launch_pdl(k_setup_tail<T>, dim3(1), dim3(512), st, levels_dev, first, nl);
}

template <typename TI, typename TO>
void launch_convert(const TI *in, TO *out, long long n, cudaStream_t st) {
  const int vec = (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
  const long long threads = vec ? (n / 4 > 4 ? n / 4 : 4) : (n > 1 ? n : 1);
  launch_pdl(k_convert<TI, TO>, dim3(nb(threads, 256)), dim3(256), st, in, out, n, vec);
}

#define INST(T)                                                                              \
  template void launch_mg_prolong_weights<T>(const MGLevel<T> &, cudaStream_t);               \
  template void launch_mg_coarse_op<T>(const MGLevel<T> &, const MGLevel<T> &, cudaStream_t); \
  template void launch_mg_setup_level<T>(const MGLevel<T> &, const MGLevel<T> &, cudaStream_t); \
  template void launch_mg_smooth<T>(const MGLevel<T> &, T *, const T *, int, int, double, T *, \
                                    cudaStream_t);                                            \
  template void launch_mg_residual<T>(const MGLevel<T> &, const T *, const T *, T *,          \
                                      cudaStream_t);                                          \
  template void launch_mg_restrict<T>(const MGLevel<T> &, const MGLevel<T> &, const T *, T *, \
                                      cudaStream_t);                                          \
  template void launch_mg_prolong_add<T>(const MGLevel<T> &, const MGLevel<T> &, const T *,   \
                                         T *, cudaStream_t);                                  \
  template void launch_vcycle_tail<T>(const MGLevel<T> *, int, int, int, double, T *, size_t, \
                                      cudaStream_t);                                          \
  template size_t tail_smem_bytes<T>(const MGLevel<T> *, int, int);                          \
  template void launch_setup_tail<T>(const MGLevel<T> *, int, int, cudaStream_t);
INST(double)
INST(float)
template void launch_convert<double, float>(const double *, float *, long long, cudaStream_t);
template void launch_convert<float, double>(const float *, double *, long long, cudaStream_t);
template void launch_convert<double, double>(const double *, double *, long long, cudaStream_t);

}  // namespace pfgpu
