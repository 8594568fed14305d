// Semicoarsening multigrid (MGSemi) kernels, templated on the storage and
// arithmetic type (double for the plain FP64 solver, float for the mixed
// solver).  Every level holds a symmetric 7-point operator as C E N U; the
// lower entries are the upper entries of the neighbour (W(i) = E(i-1) etc.,
// pfsimulator/parflow_lib/matrix.c:258-310, 477-490).  Coarse grids take the
// even fine indices in the coarsening direction; fine points are the odd ones
// (pfsimulator/parflow_lib/mg_semi.c:960-1058).
#include <cstdint>
#include <type_traits>

#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

template <typename T>
struct LV {
  int nx, ny, nz;
  long long n;
  const T *a0, *ae, *an, *au;
  const T *wg;                       // W of the i = 0 cells (MGLevel::wg)
  const __half *he, *hn, *hu, *hd;  // scaled FP16 operator (H mode)
  const int *hflag;                  // nonzero: read the scaled diagonal hd
};

template <typename T>
__device__ __forceinline__ LV<T> lv(const MGLevel<T> &L) {
  LV<T> v;
  v.nx = L.nx; v.ny = L.ny; v.nz = L.nz; v.n = L.n;
  v.a0 = L.a[0]; v.ae = L.a[1]; v.an = L.a[2]; v.au = L.a[3];
  v.wg = L.wg;
  v.he = L.h[0]; v.hn = L.h[1]; v.hu = L.h[2]; v.hd = L.h[3];
  v.hflag = L.hflag;
  return v;
}

// Template flag H selects the scaled FP16 operator (unit diagonal, E^ N^ U^
// in h, transfer weights q1/q2); H = false is the plain operator C E N U.
template <typename T, bool H>
__device__ __forceinline__ T ld_off(const T *a, const __half *h, long long c) {
  if constexpr (H)
    return (T)__half2float(h[c]);
  else
    return a[c];
}
template <typename T, bool H>
__device__ __forceinline__ T diag(const LV<T> &L, long long c) {
  if constexpr (H)
    return *L.hflag ? (T)__half2float(L.hd[c]) : T(1);
  else
    return L.a0[c];
}

__device__ __forceinline__ bool inside(int nx, int ny, int nz, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
}

// coefficient s (0..6 = C W E S N L U) of cell (i,j,k), zero outside
template <typename T, bool H = false>
__device__ __forceinline__ T coef(const LV<T> &L, int s, int i, int j, int k) {
  if (!inside(L.nx, L.ny, L.nz, i, j, k)) return T(0);
  long long c = i + (long long)L.nx * (j + (long long)L.ny * k);
  switch (s) {
    case 0: return diag<T, H>(L, c);
    case 1:
      if (i > 0) return ld_off<T, H>(L.ae, L.he, c - 1);
      // the ghost column: read by the setup (plain operator) only
      if constexpr (H) return T(0);
      else return L.wg ? L.wg[j + L.ny * k] : T(0);
    case 2: return ld_off<T, H>(L.ae, L.he, c);
    case 3: return j > 0 ? ld_off<T, H>(L.an, L.hn, c - L.nx) : T(0);
    case 4: return ld_off<T, H>(L.an, L.hn, c);
    case 5: return k > 0 ? ld_off<T, H>(L.au, L.hu, c - (long long)L.nx * L.ny) : T(0);
    default: return ld_off<T, H>(L.au, L.hu, c);
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
// the same with the block order along y and z reversed when flip is set:
// consecutive sweeps over a level that alternate direction begin on the
// planes the previous launch touched last, which are still in L2
__device__ __forceinline__ void thread_ijk_flip(int &i, int &j, int &k, int flip) {
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = by * blockDim.y + threadIdx.y;
  k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
}
// (i, j, k) of linear index t inside a level (32-bit; single-block loops)
__device__ __forceinline__ void split_ijk(int t, int nx, int ny, int &i, int &j, int &k) {
  i = t % nx;
  const int r = t / nx;
  j = r % ny;
  k = r / ny;
}
// A divisor with its float reciprocal: t / d from one multiplication and a
// one-step correction (exact while the float product errs by less than one,
// i.e. for t < 2^22; larger t take the integer division).  The single-block
// tail splits a linear index per cell and phase, where integer division
// would dominate its instruction count.
struct FastDiv {
  int d;
  float inv;
};
__device__ __forceinline__ FastDiv fast_div(int d) { return FastDiv{d, 1.0f / (float)d}; }
__device__ __forceinline__ int quot(int t, FastDiv f) {
  if (t >= (1 << 22)) return t / f.d;
  int q = (int)((float)t * f.inv);
  if ((q + 1) * f.d <= t) q++;
  if (q * f.d > t) q--;
  return q;
}
__device__ __forceinline__ void split_ijk(int t, FastDiv fx, FastDiv fy, int &i, int &j,
                                          int &k) {
  const int r = quot(t, fx);
  i = t - r * fx.d;
  k = quot(r, fy);
  j = r - k * fy.d;
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
  // the coarse W of an i = 0 cell goes to the coarse ghost column: the
  // transverse sum when coarsening along y or z, and along x the fine W
  // times the zero weight of the fine ghost point
  if (ic == 0 && C.wg) C.wg[jc + C.ny * kc] = d == 1 ? ac[3] : d == 2 ? ac[5] : T(0);
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

// PFGPU_SWEEP_ONE_CELL=1: one cell per thread in every colour sweep (A/B)
static bool getenv_flag_one_cell() {
  static const bool v = [] {
    const char *e = getenv("PFGPU_SWEEP_ONE_CELL");
    return e && *e == '1';
  }();
  return v;
}

// PFGPU_SKIP_ZERO_SWEEP=0: launch the zero-guess red sweep of the
// pre-smoother even where the black sweep can read its values from b (A/B)
static bool skip_zero_sweep() {
  static const bool v = [] {
    const char *e = getenv("PFGPU_SKIP_ZERO_SWEEP");
    return !(e && *e == '0');
  }();
  return v;
}

// H-mode kernels exist for float storage only
template <typename T>
constexpr bool kHasH16 = std::is_same<T, float>::value;

// ---- scaled FP16 operator helpers (H mode) --------------------------------
// 1/S for S = sqrt(|c|), 1 where c is 0 or not finite (hardware reciprocal
// square root: the scaled values are stored as 11-bit FP16 significands)
__device__ __forceinline__ float inv_scale_of(float c) {
  const float a = fabsf(c);
  return (a > 0.0f && isfinite(a)) ? rsqrtf(a) : 1.0f;
}
// S from c and 1/S without a division
__device__ __forceinline__ float scale_from(float c, float inv) {
  const float a = fabsf(c);
  return (a > 0.0f && isfinite(a)) ? a * inv : 1.0f;
}
// scaled operator of fine cell c: off-diagonals E N U over S_c S_nb (a0 of
// the +x, +y, +z neighbours, ignored where has_* is false), the diagonal
// C / S^2 (raising *hflag when it is not +1) and, on level 0, 1/S; returns 1/S
__device__ __forceinline__ float h16_store(const MGLevel<float> &F, int c, float cd, float e,
                                           float n, float u, bool has_e, float ae, bool has_n,
                                           float an, bool has_u, float au) {
  const float ic = inv_scale_of(cd);
  const float ie = has_e ? inv_scale_of(ae) : 0.0f;
  const float in = has_n ? inv_scale_of(an) : 0.0f;
  const float iu = has_u ? inv_scale_of(au) : 0.0f;
  F.h[0][c] = __float2half_rn(e * ic * ie);
  F.h[1][c] = __float2half_rn(n * ic * in);
  F.h[2][c] = __float2half_rn(u * ic * iu);
  const __half hd = __float2half_rn(cd * ic * ic);
  F.h[3][c] = hd;
  if (__half2float(hd) != 1.0f && *(volatile const int *)F.hflag == 0)
    atomicExch(const_cast<int *>(F.hflag), 1);
  if (F.sinv) F.sinv[c] = ic;
  return ic;
}

// The seven entries C W E S N L U of fine cell (i,j,k), zero outside the
// level: the values coef() returns, gathered with predicated loads so that
// a thread issues all its loads at once.
template <typename T>
__device__ __forceinline__ void gather7(const LV<T> &L, int i, int j, int k, T st[7]) {
  const bool in = i >= 0 && j >= 0 && k >= 0 && i < L.nx && j < L.ny && k < L.nz;
  const int sy = L.nx, sz = L.nx * L.ny;
  const int c = in ? i + sy * j + sz * k : 0;
  st[0] = in ? L.a0[c] : T(0);
  st[1] = in && i > 0 ? L.ae[c - 1] : (in && L.wg ? L.wg[j + L.ny * k] : T(0));
  st[2] = in ? L.ae[c] : T(0);
  st[3] = in && j > 0 ? L.an[c - sy] : T(0);
  st[4] = in ? L.an[c] : T(0);
  st[5] = in && k > 0 ? L.au[c - sz] : T(0);
  st[6] = in ? L.au[c] : T(0);
}

// setup_level_cell with the coarsening direction D fixed at compile time and
// every fine operand gathered up front (fine points 2c-1, 2c, 2c+1 along D;
// the lower entry of 2c+2 is the upper entry of 2c+1 in symmetric storage).
// Same operations in the same order as weights_at + coarse_op_core, so the
// result is bitwise that of setup_level_cell.
//
// H (float only): the same thread also writes the scaled FP16 operator of
// its fine points 2c and 2c+1 and the scaled weights q1(2c) = s_c,
// q1(2c+1), q2(2c-1) (all against its own coarse diagonal; q2(2c+1) comes
// from the thread of c+1, or is 0 on the last coarse point), exactly as
// h16_scale_cell computes them; the plain weights p1/p2 are not stored then.
template <typename T, int D, bool H>
__global__ void __launch_bounds__(256) k_setup_level(MGLevel<T> F, MGLevel<T> C) {
  pdl_enter();
  int ic, jc, kc;
  thread_ijk(ic, jc, kc);
  if (ic >= C.nx || jc >= C.ny || kc >= C.nz) return;
  constexpr int ox = D == 0, oy = D == 1, oz = D == 2;
  constexpr int s0 = D == 0 ? 0 : D == 1 ? 0 : 0;
  constexpr int s1 = D == 0 ? 1 : D == 1 ? 3 : 5;  // along-D lower
  constexpr int s2 = D == 0 ? 2 : D == 1 ? 4 : 6;  // along-D upper
  constexpr int s3 = D == 0 ? 3 : D == 1 ? 1 : 3;
  constexpr int s4 = D == 0 ? 4 : D == 1 ? 2 : 4;
  constexpr int s5 = D == 0 ? 5 : D == 1 ? 5 : 1;
  constexpr int s6 = D == 0 ? 6 : D == 1 ? 6 : 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  LV<T> L = lv(F);
  T sm[7], sc[7], sp[7];  // fine cells f-1, f, f+1 along D
  gather7(L, i - ox, j - oy, k - oz, sm);
  gather7(L, i, j, k, sc);
  gather7(L, i + ox, j + oy, k + oz, sp);
  // prolongation weights of f-1 (its p2) and f+1 (p1, p2): weights_at
  T p2_1 = T(0), p1_2 = T(0), p2_2 = T(0);
  {
    const T ap0 = sm[s0] + sm[s3] + sm[s4] + sm[s5] + sm[s6];
    if (ap0 != T(0)) p2_1 = -sm[s2] / ap0;
  }
  {
    const T ap0 = sp[s0] + sp[s3] + sp[s4] + sp[s5] + sp[s6];
    if (ap0 != T(0)) {
      p1_2 = -sp[s1] / ap0;
      p2_2 = -sp[s2] / ap0;
    }
  }
  const int ip = i + ox, jp = j + oy, kp = k + oz;
  const bool has_p = ip < F.nx && jp < F.ny && kp < F.nz;
  if (!H && has_p) {
    const long long f = ip + (long long)F.nx * (jp + (long long)F.ny * kp);
    F.p1[f] = p1_2;
    F.p2[f] = p2_2;
  }
  // coarse operator: coarse_op_core
  const long long cc = ic + (long long)C.nx * (jc + (long long)C.ny * kc);
  const T ac3 = sc[s3] + T(0.5) * sm[s3] + T(0.5) * sp[s3];
  const T ac4 = sc[s4] + T(0.5) * sm[s4] + T(0.5) * sp[s4];
  const T ac5 = sc[s5] + T(0.5) * sm[s5] + T(0.5) * sp[s5];
  const T ac6 = sc[s6] + T(0.5) * sm[s6] + T(0.5) * sp[s6];
  const T ac2 = sc[s2] * p2_2;
  const T ac0 = sc[s0] + sc[s3] + sc[s4] + sc[s5] + sc[s6] + sc[s1] * p2_1 + sc[s2] * p1_2;
  const int last = D == 0 ? (ic + 1 >= C.nx) : D == 1 ? (jc + 1 >= C.ny) : (kc + 1 >= C.nz);
  // not last: fine 2c+2 exists, and its lower entry is the upper entry of 2c+1
  const T along_up = last ? ac2 : sp[s2] * p1_2;
  T E, N, U;
  if (D == 0) { E = along_up; N = ac4; U = ac6; }
  else if (D == 1) { E = ac4; N = along_up; U = ac6; }
  else { E = ac6; N = ac4; U = along_up; }
  C.a[1][cc] = E;
  C.a[2][cc] = N;
  C.a[3][cc] = U;
  const T cdiag = ac0 - (ac3 + ac4 + ac5 + ac6);
  C.a[0][cc] = cdiag;
  // coarse ghost column (see coarse_op_core)
  if (ic == 0 && C.wg) C.wg[jc + C.ny * kc] = D == 1 ? ac3 : D == 2 ? ac5 : T(0);
  if constexpr (H) {
    const int nx = F.nx, ny = F.ny, nz = F.nz;
    const int sy = nx, sz = nx * ny;
    const float *a0 = F.a[0];
    const float ics = inv_scale_of(cdiag);
    // fine point 2c
    const int f0 = i + sy * j + sz * k;
    const float ae0 = i + 1 < nx ? a0[f0 + 1] : 0.0f;
    const float an0 = j + 1 < ny ? a0[f0 + sy] : 0.0f;
    const float au0 = k + 1 < nz ? a0[f0 + sz] : 0.0f;
    const float ic0 = h16_store(F, f0, sc[0], sc[2], sc[4], sc[6], i + 1 < nx, ae0, j + 1 < ny,
                                an0, k + 1 < nz, au0);
    F.q1[f0] = scale_from(sc[0], ic0) * ics;
    F.q2[f0] = 0.0f;
    // fine point 2c-1: its q2 pairs with this coarse point
    const int im = i - ox, jm = j - oy, km = k - oz;
    if (im >= 0 && jm >= 0 && km >= 0) {
      const int fm = im + sy * jm + sz * km;
      F.q2[fm] = p2_1 * scale_from(sm[0], inv_scale_of(sm[0])) * ics;
    }
    // fine point 2c+1
    if (has_p) {
      const int f1 = ip + sy * jp + sz * kp;
      const float ae1 = ip + 1 < nx ? a0[f1 + 1] : 0.0f;
      const float an1 = jp + 1 < ny ? a0[f1 + sy] : 0.0f;
      const float au1 = kp + 1 < nz ? a0[f1 + sz] : 0.0f;
      const float ic1 = h16_store(F, f1, sp[0], sp[2], sp[4], sp[6], ip + 1 < nx, ae1,
                                  jp + 1 < ny, an1, kp + 1 < nz, au1);
      F.q1[f1] = p1_2 * scale_from(sp[0], ic1) * ics;
      if (last) F.q2[f1] = 0.0f;
    }
  }
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
template <typename T, bool H = false>
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
    x[c] = b[c] / diag<T, H>(L, c);
    return;
  }
  const long long sy = nx, sz = (long long)nx * ny;
  x[c] = rb_update<T>(diag<T, H>(L, c), b[c], coef<T, H>(L, 1, i, j, k), i > 0 ? x[c - 1] : T(0),
                      coef<T, H>(L, 2, i, j, k), i + 1 < nx ? x[c + 1] : T(0),
                      coef<T, H>(L, 3, i, j, k), j > 0 ? x[c - sy] : T(0),
                      coef<T, H>(L, 4, i, j, k), j + 1 < ny ? x[c + sy] : T(0),
                      coef<T, H>(L, 5, i, j, k), k > 0 ? x[c - sz] : T(0),
                      coef<T, H>(L, 6, i, j, k), k + 1 < Lv.nz ? x[c + sz] : T(0));
}

// Grid form of rb_cell with lean index arithmetic: 32-bit cell indices (a
// level that fits in device memory has fewer than 2^31 cells), the grid's z
// extent equal to nz, predicated neighbour loads, no neighbour loads on the
// zero-guess sweep and, for the scaled operator with unit diagonal, no
// division.  Bitwise the same result as rb_cell.
template <typename T>
__device__ __forceinline__ T ldro(const T *p) {
  return __ldg(p);
}
__device__ __forceinline__ float ldro_h(const __half *p) {
  return __half2float(__ldg(p));
}

// Grid form of rb_cell with lean index arithmetic: 32-bit cell indices (a
// level that fits in device memory has fewer than 2^31 cells), the grid's z
// extent equal to nz, predicated neighbour loads, no neighbour loads on the
// zero-guess sweep and, for the scaled operator with unit diagonal, no
// division.  Every array the sweep reads is read-only for the launch (it
// writes one colour and reads only the other), so all loads take the
// read-only data path.  Bitwise the same result as rb_cell.
template <typename T, bool H>
__global__ void __launch_bounds__(256) k_rb_sweep(MGLevel<T> L, T *__restrict__ x,
                                                  const T *__restrict__ b, int colour, int init,
                                                  int flip) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (j >= ny) return;
  const int r = (colour ^ 1 ^ j ^ k) & 1;
  const int i = 2 * q + r;  // red: (i+j+k) odd
  if (i >= nx) return;
  const int sy = nx, sz = nx * ny;
  const int c = i + sy * j + sz * k;
  // x / b storage of this cell and of its six (other-colour) neighbours
  int xo, xw, xe, xs, xn, xl, xu;
  if (L.split) {
    const int hx = L.hx, hs = hx * ny, half = hs * nz;
    const int base = q + hx * j + hs * k;
    xo = (colour ^ 1) * half + base;  // this colour's parity block
    const int ob = colour * half + base;
    xw = ob - 1 + r; xe = ob + r; xs = ob - hx; xn = ob + hx; xl = ob - hs; xu = ob + hs;
  } else {
    xo = c; xw = c - 1; xe = c + 1; xs = c - sy; xn = c + sy; xl = c - sz; xu = c + sz;
  }
  bool unit = false;  // scaled operator with unit diagonal everywhere
  T d = T(1);
  if constexpr (H) {
    unit = ldro(L.hflag) == 0;
    if (!unit) d = (T)ldro_h(L.h[3] + c);
  } else {
    d = ldro(L.a[0] + c);
  }
  if (init) {
    x[xo] = unit ? ldro(b + xo) : ldro(b + xo) / d;
    return;
  }
  const bool hw = i > 0, he = i + 1 < nx, hs = j > 0, hn = j + 1 < ny, hl = k > 0,
             hu = k + 1 < nz;
  T cw, ce, cs, cn, cl, cu;
  if constexpr (H) {
    cw = hw ? (T)ldro_h(L.h[0] + c - 1) : T(0);
    ce = (T)ldro_h(L.h[0] + c);
    cs = hs ? (T)ldro_h(L.h[1] + c - sy) : T(0);
    cn = (T)ldro_h(L.h[1] + c);
    cl = hl ? (T)ldro_h(L.h[2] + c - sz) : T(0);
    cu = (T)ldro_h(L.h[2] + c);
  } else {
    cw = hw ? ldro(L.a[1] + c - 1) : T(0);
    ce = ldro(L.a[1] + c);
    cs = hs ? ldro(L.a[2] + c - sy) : T(0);
    cn = ldro(L.a[2] + c);
    cl = hl ? ldro(L.a[3] + c - sz) : T(0);
    cu = ldro(L.a[3] + c);
  }
  const T *xr = x;  // the other colour: not written by this launch
  T acc = cw * (hw ? ldro(xr + xw) : T(0));
  acc = fma(ce, he ? ldro(xr + xe) : T(0), acc);
  acc = fma(cs, hs ? ldro(xr + xs) : T(0), acc);
  acc = fma(cn, hn ? ldro(xr + xn) : T(0), acc);
  acc = fma(cl, hl ? ldro(xr + xl) : T(0), acc);
  acc = fma(cu, hu ? ldro(xr + xu) : T(0), acc);
  const T bc = ldro(b + xo);
  x[xo] = unit ? bc - acc : (bc - acc) / d;
}

// Colour sweep of a colour-split level with two cells per thread: cells q
// and q+1 of one colour in a row (x indices i and i+2, adjacent in the colour
// block) share the row's index arithmetic, the predicates, the diagonal flag
// and the other-colour cell between them.  Same per-cell arithmetic, in the
// same order, as k_rb_sweep.
// from_b: the sweep that follows a zero-guess red sweep reads the red values
// that sweep would have written, b / a0, straight from b (and the diagonal),
// so the zero-guess sweep itself is not launched
template <typename T, bool H, bool FROM_B = false>
__global__ void __launch_bounds__(256) k_rb_sweep2(MGLevel<T> L, T *__restrict__ x,
                                                   const T *__restrict__ b, int colour,
                                                   int init, int flip) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int q0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = by * blockDim.y + threadIdx.y;
  const int k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (j >= ny) return;
  const int r = (colour ^ 1 ^ j ^ k) & 1;
  const int i0 = 2 * q0 + r;  // red: (i+j+k) odd
  if (i0 >= nx) return;
  const bool two = i0 + 2 < nx;  // the second cell, i0 + 2, exists
  const int sy = nx, sz = nx * ny;
  const int c0 = i0 + sy * j + sz * k, c1 = c0 + 2;
  const int hx = L.hx, hs = hx * ny, half = hs * nz;
  const int base = q0 + hx * j + hs * k;
  const int xo = (colour ^ 1) * half + base;  // own cells: xo, xo + 1
  const int ob = colour * half + base;        // other colour, same (q, j, k)
  bool unit = false;
  T d0 = T(1), d1 = T(1);
  if constexpr (H) {
    unit = ldro(L.hflag) == 0;
    if (!unit) {
      d0 = (T)ldro_h(L.h[3] + c0);
      if (two) d1 = (T)ldro_h(L.h[3] + c1);
    }
  } else {
    d0 = ldro(L.a[0] + c0);
    if (two) d1 = ldro(L.a[0] + c1);
  }
  if (init) {
    x[xo] = unit ? ldro(b + xo) : ldro(b + xo) / d0;
    if (two) x[xo + 1] = unit ? ldro(b + xo + 1) : ldro(b + xo + 1) / d1;
    return;
  }
  const bool hw = i0 > 0, he0 = i0 + 1 < nx, he1 = i0 + 3 < nx, hsj = j > 0, hn = j + 1 < ny,
             hl = k > 0, hu = k + 1 < nz;
  auto coef = [&](int s, int c) -> T {  // E / N / U entry s of cell c
    if constexpr (H)
      return (T)ldro_h(L.h[s] + c);
    else
      return ldro(L.a[s + 1] + c);
  };
  const T *xr = x;  // the other colour: not written by this launch
  // the other colour's value at split index q (natural index cn)
  auto xv = [&](int q, int cn) -> T {
    if constexpr (!FROM_B) {
      return ldro(xr + q);
    } else {
      const T bv = ldro(b + q);
      if constexpr (H)
        return unit ? bv : bv / (T)ldro_h(L.h[3] + cn);
      else
        return bv / ldro(L.a[0] + cn);
    }
  };
  const T xm = he0 ? xv(ob + r, c0 + 1) : T(0);  // between the two cells
  {
    const T cw = hw ? coef(0, c0 - 1) : T(0), ce = coef(0, c0);
    const T cs = hsj ? coef(1, c0 - sy) : T(0), cn = coef(1, c0);
    const T cl = hl ? coef(2, c0 - sz) : T(0), cu = coef(2, c0);
    T acc = cw * (hw ? xv(ob - 1 + r, c0 - 1) : T(0));
    acc = fma(ce, xm, acc);
    acc = fma(cs, hsj ? xv(ob - hx, c0 - sy) : T(0), acc);
    acc = fma(cn, hn ? xv(ob + hx, c0 + sy) : T(0), acc);
    acc = fma(cl, hl ? xv(ob - hs, c0 - sz) : T(0), acc);
    acc = fma(cu, hu ? xv(ob + hs, c0 + sz) : T(0), acc);
    const T bc = ldro(b + xo);
    x[xo] = unit ? bc - acc : (bc - acc) / d0;
  }
  if (two) {
    const int o1 = ob + 1;
    const T cw = coef(0, c1 - 1), ce = coef(0, c1);
    const T cs = hsj ? coef(1, c1 - sy) : T(0), cn = coef(1, c1);
    const T cl = hl ? coef(2, c1 - sz) : T(0), cu = coef(2, c1);
    T acc = cw * xm;
    acc = fma(ce, he1 ? xv(o1 + r, c1 + 1) : T(0), acc);
    acc = fma(cs, hsj ? xv(o1 - hx, c1 - sy) : T(0), acc);
    acc = fma(cn, hn ? xv(o1 + hx, c1 + sy) : T(0), acc);
    acc = fma(cl, hl ? xv(o1 - hs, c1 - sz) : T(0), acc);
    acc = fma(cu, hu ? xv(o1 + hs, c1 + sz) : T(0), acc);
    const T bc = ldro(b + xo + 1);
    x[xo + 1] = unit ? bc - acc : (bc - acc) / d1;
  }
}

// weighted Jacobi (pfsimulator/parflow_lib/w_jacobi.c:120-290)
template <typename T, bool H = false>
__device__ __forceinline__ void wjacobi_cell(const MGLevel<T> &Lv, const T *__restrict__ x,
                                             const T *__restrict__ b, T *__restrict__ t,
                                             int zero, int i, int j, int k) {
  if (i >= Lv.nx || j >= Lv.ny || k >= Lv.nz) return;
  const long long c = i + (long long)Lv.nx * (j + (long long)Lv.ny * k);
  LV<T> L = lv(Lv);
  if (zero) {
    t[c] = b[c] / diag<T, H>(L, c);
    return;
  }
  const int nx = Lv.nx, ny = Lv.ny, nz = Lv.nz;
  T v = b[c];
  v -= coef<T, H>(L, 1, i, j, k) * vget(nx, ny, nz, x, i - 1, j, k);
  v -= coef<T, H>(L, 2, i, j, k) * vget(nx, ny, nz, x, i + 1, j, k);
  v -= coef<T, H>(L, 3, i, j, k) * vget(nx, ny, nz, x, i, j - 1, k);
  v -= coef<T, H>(L, 4, i, j, k) * vget(nx, ny, nz, x, i, j + 1, k);
  v -= coef<T, H>(L, 5, i, j, k) * vget(nx, ny, nz, x, i, j, k - 1);
  v -= coef<T, H>(L, 6, i, j, k) * vget(nx, ny, nz, x, i, j, k + 1);
  t[c] = v / diag<T, H>(L, c);
}

template <typename T, bool H>
__global__ void k_wjacobi(MGLevel<T> Lv, const T *__restrict__ x, const T *__restrict__ b,
                          T *__restrict__ t, int zero) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  wjacobi_cell<T, H>(Lv, x, b, t, zero, i, j, k);
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
template <typename T, bool H = false>
__device__ __forceinline__ void mg_residual_cell(const MGLevel<T> &Lv, const T *__restrict__ x,
                                                 const T *__restrict__ b, T *__restrict__ r,
                                                 int i, int j, int k) {
  if (i >= Lv.nx || j >= Lv.ny || k >= Lv.nz) return;
  const long long c = i + (long long)Lv.nx * (j + (long long)Lv.ny * k);
  const int nx = Lv.nx, ny = Lv.ny, nz = Lv.nz;
  LV<T> L = lv(Lv);
  T y = -b[c];
  y += diag<T, H>(L, c) * x[c];
  y += coef<T, H>(L, 1, i, j, k) * vget(nx, ny, nz, x, i - 1, j, k);
  y += coef<T, H>(L, 2, i, j, k) * vget(nx, ny, nz, x, i + 1, j, k);
  y += coef<T, H>(L, 3, i, j, k) * vget(nx, ny, nz, x, i, j - 1, k);
  y += coef<T, H>(L, 4, i, j, k) * vget(nx, ny, nz, x, i, j + 1, k);
  y += coef<T, H>(L, 5, i, j, k) * vget(nx, ny, nz, x, i, j, k - 1);
  y += coef<T, H>(L, 6, i, j, k) * vget(nx, ny, nz, x, i, j, k + 1);
  r[c] = -y;
}

// grid form of mg_residual_cell (same operation order, lean indices)
// r = b - A x of one cell (the grid residual kernels' shared arithmetic)
template <typename T, bool H>
__device__ __forceinline__ T mg_residual_cell(const MGLevel<T> &L, const T *__restrict__ x,
                                              const T *__restrict__ b, int i, int j, int k) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int sy = nx, sz = nx * ny;
  const int c = i + sy * j + sz * k;
  const bool hw = i > 0, he = i + 1 < nx, hs = j > 0, hn = j + 1 < ny, hl = k > 0,
             hu = k + 1 < nz;
  int xo, xw, xe, xs, xn, xl, xu;  // x / b storage of the cell and its neighbours
  if (L.split) {
    const int hx = L.hx, hsl = hx * ny, half = hsl * nz;
    const int p = (i + j + k) & 1, base = (i >> 1) + hx * j + hsl * k, r = i & 1;
    xo = p * half + base;
    const int ob = (p ^ 1) * half + base;
    xw = ob - 1 + r; xe = ob + r; xs = ob - hx; xn = ob + hx; xl = ob - hsl; xu = ob + hsl;
  } else {
    xo = c; xw = c - 1; xe = c + 1; xs = c - sy; xn = c + sy; xl = c - sz; xu = c + sz;
  }
  T d, cw, ce, cs, cn, cl, cu;
  if constexpr (H) {
    d = ldro(L.hflag) ? (T)ldro_h(L.h[3] + c) : T(1);
    cw = hw ? (T)ldro_h(L.h[0] + c - 1) : T(0);
    ce = (T)ldro_h(L.h[0] + c);
    cs = hs ? (T)ldro_h(L.h[1] + c - sy) : T(0);
    cn = (T)ldro_h(L.h[1] + c);
    cl = hl ? (T)ldro_h(L.h[2] + c - sz) : T(0);
    cu = (T)ldro_h(L.h[2] + c);
  } else {
    d = ldro(L.a[0] + c);
    cw = hw ? ldro(L.a[1] + c - 1) : T(0);
    ce = ldro(L.a[1] + c);
    cs = hs ? ldro(L.a[2] + c - sy) : T(0);
    cn = ldro(L.a[2] + c);
    cl = hl ? ldro(L.a[3] + c - sz) : T(0);
    cu = ldro(L.a[3] + c);
  }
  T y = -ldro(b + xo);
  y += d * ldro(x + xo);
  y += cw * (hw ? ldro(x + xw) : T(0));
  y += ce * (he ? ldro(x + xe) : T(0));
  y += cs * (hs ? ldro(x + xs) : T(0));
  y += cn * (hn ? ldro(x + xn) : T(0));
  y += cl * (hl ? ldro(x + xl) : T(0));
  y += cu * (hu ? ldro(x + xu) : T(0));
  return -y;
}

template <typename T, bool H>
__global__ void __launch_bounds__(256) k_mg_residual(MGLevel<T> L, const T *__restrict__ x,
                                                     const T *__restrict__ b,
                                                     T *__restrict__ r, int flip) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  if (i >= L.nx || j >= L.ny) return;
  r[i + L.nx * (j + L.ny * k)] = mg_residual_cell<T, H>(L, x, b, i, j, k);
}

// The residual right after a red/black sweep of colour zc: the cells of that
// colour were just solved against their current neighbours, so their
// residual is zero up to rounding and is written as zero; one thread per
// pair of cells (i, i+1) of a row, one of each colour, computes the other
// cell's residual as k_mg_residual does.
template <typename T, bool H>
__global__ void __launch_bounds__(256) k_mg_residual_pair(MGLevel<T> L, const T *__restrict__ x,
                                                          const T *__restrict__ b,
                                                          T *__restrict__ r, int flip, int zc) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int i0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = by * blockDim.y + threadIdx.y;
  const int k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  const int nx = L.nx;
  if (i0 >= nx || j >= L.ny) return;
  // colour 0 (red) is parity 1 of i + j + k
  const int zpar = zc == 0 ? 1 : 0;
  const int iz = ((i0 + j + k) & 1) == zpar ? i0 : i0 + 1;  // the zero-residual cell
  const int ic = iz == i0 ? i0 + 1 : i0;                     // the computed cell
  const int row = nx * (j + L.ny * k);
  if (iz < nx) r[iz + row] = T(0);
  if (ic < nx) r[ic + row] = mg_residual_cell<T, H>(L, x, b, ic, j, k);
}

// r_c = r_f(c) + (p2(f-1) r_f(f-1) + p1(f+1) r_f(f+1)) (mg_semi_restrict.c:161-169)
// (H: r^_c = s_c r^_f(c) + (q2(f-1) r^_f(f-1) + q1(f+1) r^_f(f+1)), the
// scaled form of the same operator, s_c = q1 at the coarse point)
template <typename T, bool H = false>
__device__ __forceinline__ void restrict_cell(const MGLevel<T> &F, const MGLevel<T> &C,
                                              const T *__restrict__ rf, T *__restrict__ rc,
                                              int ic, int jc, int kc) {
  if (ic >= C.nx || jc >= C.ny || kc >= C.nz) return;
  const long long cc = ic + (long long)C.nx * (jc + (long long)C.ny * kc);
  const int d = F.dir;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const T *w1 = H ? F.q1 : F.p1;
  const T *w2 = H ? F.q2 : F.p2;
  const long long f = i + (long long)nx * (j + (long long)ny * k);
  T centre = rf[f];
  if constexpr (H) centre = w1[f] * centre;
  rc[cc] = centre + (vget(nx, ny, nz, w2, i - ox, j - oy, k - oz) *
                         vget(nx, ny, nz, rf, i - ox, j - oy, k - oz) +
                     vget(nx, ny, nz, w1, i + ox, j + oy, k + oz) *
                         vget(nx, ny, nz, rf, i + ox, j + oy, k + oz));
}

// grid form of restrict_cell with the direction D fixed at compile time and
// 32-bit indices (same operations, same order)
template <typename T, bool H, int D>
__global__ void __launch_bounds__(256) k_restrict(MGLevel<T> F, MGLevel<T> C,
                                                  const T *__restrict__ rf, T *__restrict__ rc,
                                                  int flip) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int ic = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = by * blockDim.y + threadIdx.y;
  const int kc = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  if (ic >= C.nx || jc >= C.ny) return;
  constexpr int ox = D == 0, oy = D == 1, oz = D == 2;
  const int nx = F.nx, ny = F.ny;
  const int i = ox ? 2 * ic : ic, j = oy ? 2 * jc : jc, k = oz ? 2 * kc : kc;
  const int so = D == 0 ? 1 : D == 1 ? nx : nx * ny;  // fine stride along D
  const int nd = D == 0 ? nx : D == 1 ? ny : F.nz;
  const int cd = D == 0 ? i : D == 1 ? j : k;
  const int f = i + nx * (j + ny * k);
  const T *w1 = H ? F.q1 : F.p1;
  const T *w2 = H ? F.q2 : F.p2;
  const bool lo = cd > 0, hi = cd + 1 < nd;
  T centre = ldro(rf + f);
  if constexpr (H) centre = ldro(w1 + f) * centre;
  rc[xb_index(C, ic, jc, kc)] =
      centre + ((lo ? ldro(w2 + f - so) : T(0)) * (lo ? ldro(rf + f - so) : T(0)) +
                (hi ? ldro(w1 + f + so) : T(0)) * (hi ? ldro(rf + f + so) : T(0)));
}

// x_f += P e_c: injection at coarse points, p1 e(f-1) + p2 e(f+1) at fine
// points (mg_semi_prolong.c:119-124, 191-197), followed by Axpy(1, e, x)
// (H: s_c e at coarse points, q1 e(f-1) + q2 e(f+1) at fine points)
template <typename T, bool H = false>
__device__ __forceinline__ void prolong_add_cell(const MGLevel<T> &F, const MGLevel<T> &C,
                                                 const T *__restrict__ ec, T *__restrict__ xf,
                                                 int i, int j, int k) {
  if (i >= F.nx || j >= F.ny || k >= F.nz) return;
  const long long c = i + (long long)F.nx * (j + (long long)F.ny * k);
  const int d = F.dir;
  const int ci = d == 0 ? i : d == 1 ? j : k;
  const int ox = d == 0, oy = d == 1, oz = d == 2;
  const T *w1 = H ? F.q1 : F.p1;
  const T *w2 = H ? F.q2 : F.p2;
  T e;
  if (!(ci & 1)) {
    e = ec[(ox ? i / 2 : i) + (long long)C.nx * ((oy ? j / 2 : j) + (long long)C.ny * (oz ? k / 2 : k))];
    if constexpr (H) e = w1[c] * e;
  } else {
    int il = i - ox, jl = j - oy, kl = k - oz;  // coarse point below (even)
    int ih = i + ox, jh = j + oy, kh = k + oz;  // coarse point above (even), may be outside
    T el = ec[(ox ? il / 2 : il) + (long long)C.nx * ((oy ? jl / 2 : jl) + (long long)C.ny * (oz ? kl / 2 : kl))];
    T eh = inside(F.nx, F.ny, F.nz, ih, jh, kh)
               ? ec[(ox ? ih / 2 : ih) + (long long)C.nx * ((oy ? jh / 2 : jh) + (long long)C.ny * (oz ? kh / 2 : kh))]
               : T(0);
    e = (w1[c] * el + w2[c] * eh);
  }
  xf[c] = xf[c] + e;
}

// grid form of prolong_add_cell with the direction D fixed at compile time:
// one branch-free formula for both parities (at a coarse point the weights
// are (1, 0), or (s_c, 0) in H mode, and both coarse neighbours coincide),
// bitwise the same values as prolong_add_cell
template <typename T, bool H, int D>
__global__ void __launch_bounds__(256) k_prolong_add(MGLevel<T> F, MGLevel<T> C,
                                                     const T *__restrict__ ec,
                                                     T *__restrict__ xf, int flip, int skip_red) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
  const int nx = F.nx, ny = F.ny;
  if (i >= nx || j >= ny) return;
  // a red/black post-smoother starts with a red sweep, which overwrites the
  // red cells without reading them: only the black cells need the correction
  if (skip_red && ((i + j + k) & 1)) return;
  const int c = i + nx * (j + ny * k);
  const int cd = D == 0 ? i : D == 1 ? j : k;
  const int nd = D == 0 ? nx : D == 1 ? ny : F.nz;
  const int lo = cd >> 1, hi = (cd + 1) >> 1;  // coarse points at/below, at/above
  const bool odd = cd & 1;
  const bool has_hi = hi < (nd + 1) / 2;
  const int clo = D == 0 ? xb_index(C, lo, j, k) : D == 1 ? xb_index(C, i, lo, k)
                                                         : xb_index(C, i, j, lo);
  const int chi = D == 0 ? xb_index(C, hi, j, k) : D == 1 ? xb_index(C, i, hi, k)
                                                         : xb_index(C, i, j, hi);
  const T el = ldro(ec + clo);
  const T eh = has_hi ? ldro(ec + chi) : T(0);
  const T *w1p = H ? F.q1 : F.p1;
  const T *w2p = H ? F.q2 : F.p2;
  T e;
  if constexpr (H) {
    // coarse points: q1 = s_c, q2 = 0
    const T w1 = ldro(w1p + c);
    e = odd ? (w1 * el + ldro(w2p + c) * eh) : w1 * el;
  } else {
    e = odd ? (ldro(w1p + c) * el + ldro(w2p + c) * eh) : el;
  }
  const int xc = xb_index(F, i, j, k);
  xf[xc] = xf[xc] + e;
}

// ---------------------------------------------------------------------------
// The coarse tail of the hierarchy (levels from `first` down to the coarsest)
// in one single-block kernel: each level there holds only a few thousand
// cells, so launching a grid per smoothing sweep costs more than the sweep.
// The block walks the same sequence of phases as the per-level kernels
// (smooth, residual, restrict, ..., coarse solve, prolong + correct, smooth),
// separated by barriers; the arithmetic per cell is identical.
//
// A team is the set of threads that walks those phases together:
// BlockTeam is one thread block (barrier __syncthreads); ClusterTeam is every
// block of a thread-block cluster (barrier.cluster with release / acquire
// semantics, which orders one phase's global-memory writes before the next
// phase's reads on every SM of the cluster).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return (int)r;
}
__device__ __forceinline__ int cluster_blocks() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return (int)r;
}
struct BlockTeam {
  __device__ static int rank() { return threadIdx.x; }
  __device__ static int size() { return blockDim.x; }
  __device__ static void sync() { __syncthreads(); }
};
struct ClusterTeam {
  __device__ static int rank() { return cluster_rank() * blockDim.x + threadIdx.x; }
  __device__ static int size() { return cluster_blocks() * blockDim.x; }
  __device__ static void sync() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
  }
};

// GridTeam is every block of a cooperative launch (all blocks resident at
// once): its barrier is a counter and a generation word in global memory.
// The last block to arrive resets the counter and advances the generation;
// the others poll the generation.  Every wait is bounded (GRID_WAIT_NS by
// the global timer): a block that gives up writes 3 into the error word and
// later barriers of the launch no longer wait, so the kernel always ends;
// the host reports the error after the solve (its results are then invalid).
// A fence on both sides of the barrier orders one phase's global writes
// before the next phase's plain loads on every SM.
constexpr unsigned long long GRID_WAIT_NS = 1000000000ull;  // 1 s
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ GridCtl &grid_ctl() {
  __shared__ GridCtl ctl;
  return ctl;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v)
               : "memory");
  return old;
}
__device__ __forceinline__ void grid_barrier(const GridCtl &g) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int *err = g.err;
    if (*err == 0) {
      const unsigned gen0 = ld_acquire_gpu(g.gen);
      // arrive (release this block's writes of the phase)
      const unsigned arrived = atom_add_acq_rel_gpu(g.count, 1u) + 1u;
      if (arrived == gridDim.x) {
        atomicExch(g.count, 0u);
        atom_add_acq_rel_gpu(g.gen, 1u);
      } else {
        // wait (acquire the other blocks' writes); the timer is read only
        // every 256 polls
        unsigned long long t0 = 0;
        for (unsigned it = 0; ld_acquire_gpu(g.gen) == gen0; it++) {
          if ((it & 255u) == 0) {
            if (*err != 0) break;
            const unsigned long long t = global_ns();
            if (it == 0) {
              t0 = t;
            } else if (t - t0 > GRID_WAIT_NS) {
              atomicCAS(g.err, 0, 3);
              break;
            }
          }
        }
      }
    }
  }
  __syncthreads();
}
struct GridTeam {
  __device__ static int rank() { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ static int size() { return gridDim.x * blockDim.x; }
  __device__ static void sync() { grid_barrier(grid_ctl()); }
};

template <typename T, bool H, class Team>
__device__ __forceinline__ void team_smooth(const MGLevel<T> &L, T *x, const T *b, int zero,
                                            int smoother, T w, T *tmp) {
  const int r0 = Team::rank(), rs = Team::size();
  if (smoother == 1) {
    const FastDiv fx = fast_div(L.nx), fy = fast_div(L.ny);
    for (int t = r0; t < (int)L.n; t += rs) {
      int i, j, k;
      split_ijk(t, fx, fy, i, j, k);
      wjacobi_cell<T, H>(L, x, b, tmp, zero, i, j, k);
    }
    Team::sync();
    for (long long c = r0; c < L.n; c += rs) wjacobi_update_cell(x, (const T *)tmp, L.n, w, zero, c);
    Team::sync();
    return;
  }
  const int hx = (L.nx + 1) / 2;
  const int half = hx * L.ny * L.nz;
  const FastDiv fx = fast_div(hx), fy = fast_div(L.ny);
  const int nsweep = smoother == 2 ? 2 : 3;  // non-symmetric: red, black
  for (int sweep = 0; sweep < nsweep; sweep++) {
    const int colour = sweep == 1 ? 1 : 0;
    const int init = (sweep == 0) ? zero : 0;
    for (int t = r0; t < half; t += rs) {
      int q, j, k;
      split_ijk(t, fx, fy, q, j, k);
      rb_cell<T, H>(L, x, b, colour, init, q, j, k);
    }
    Team::sync();
  }
}

// down-leg of one level: pre-smooth (zero guess), residual, restriction to C
template <typename T, bool H, class Team>
__device__ __forceinline__ void team_down(const MGLevel<T> &L, const MGLevel<T> &C,
                                          int smoother, T w, T *tmp) {
  const int r0 = Team::rank(), rs = Team::size();
  team_smooth<T, H, Team>(L, L.x, (const T *)L.b, 1, smoother, w, tmp);
  const FastDiv fx = fast_div(L.nx), fy = fast_div(L.ny);
  for (int t = r0; t < (int)L.n; t += rs) {
    int i, j, k;
    split_ijk(t, fx, fy, i, j, k);
    // the colour swept last (red: (i+j+k) odd) has a zero residual
    if (L.zc >= 0 && (((i + j + k) & 1) == (L.zc == 0 ? 1 : 0)))
      L.t[t] = T(0);
    else
      mg_residual_cell<T, H>(L, (const T *)L.x, (const T *)L.b, L.t, i, j, k);
  }
  Team::sync();
  const FastDiv cx = fast_div(C.nx), cy = fast_div(C.ny);
  for (int t = r0; t < (int)C.n; t += rs) {
    int i, j, k;
    split_ijk(t, cx, cy, i, j, k);
    restrict_cell<T, H>(L, C, (const T *)L.t, C.b, i, j, k);
  }
  Team::sync();
}

// up-leg of one level: prolong C's correction and add it, post-smooth
template <typename T, bool H, class Team>
__device__ __forceinline__ void team_up(const MGLevel<T> &L, const MGLevel<T> &C, int smoother,
                                        T w, T *tmp) {
  const int r0 = Team::rank(), rs = Team::size();
  const FastDiv fx = fast_div(L.nx), fy = fast_div(L.ny);
  for (int t = r0; t < (int)L.n; t += rs) {
    int i, j, k;
    split_ijk(t, fx, fy, i, j, k);
    prolong_add_cell<T, H>(L, C, (const T *)C.x, L.x, i, j, k);
  }
  Team::sync();
  team_smooth<T, H, Team>(L, L.x, (const T *)L.b, 0, smoother, w, tmp);
}

// the tail cycle over levels first .. nl-1 of the table Ls (global or shared)
template <typename T, bool H, class Team = BlockTeam>
__device__ __forceinline__ void tail_cycle(const MGLevel<T> *Ls, int first, int nl,
                                           int smoother, T w, T *tmp) {
  // down: levels first .. nl-2
  for (int l = first; l <= nl - 2; l++) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_down<T, H, Team>(L, C, smoother, w, tmp);
  }
  // coarse solve: red/black Gauss-Seidel
  {
    const MGLevel<T> L = Ls[nl - 1];
    team_smooth<T, H, Team>(L, L.x, (const T *)L.b, 1, 0, T(1), tmp);
  }
  // up: levels nl-2 .. first
  for (int l = nl - 2; l >= first; l--) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_up<T, H, Team>(L, C, smoother, w, tmp);
  }
}

// Tail levels in global memory (used when they do not fit in shared memory).
template <typename T, bool H>
__global__ void __launch_bounds__(512) k_vcycle_tail(const MGLevel<T> *__restrict__ Ls,
                                                      int first, int nl, int smoother, T w,
                                                      T *tmp) {
  pdl_enter();
  tail_cycle<T, H>(Ls, first, nl, smoother, w, tmp);
}

// Tail levels in shared memory: the block copies every tail level's operator
// (C E N U, or the scaled FP16 off-diagonals in H mode), transfer weights and
// the first tail level's right-hand side into shared memory (x and b of the
// coarser levels live there too, plus one scratch vector for residuals and
// Jacobi updates), runs the cycle with each phase waiting on shared-memory
// rather than L2 latency, and writes the first tail level's x back.  The
// copy-in is one flattened loop over all arrays in 32-bit words with eight
// loads in flight per thread (FP16 arrays are allocated with padding, so the
// last word of an odd-length one stays inside its allocation).
struct TailSeg {
  uint32_t *dst;
  const uint32_t *src;
  int start;  // first flattened word of this array
};

__host__ __device__ inline long long pad16(long long bytes) { return (bytes + 15) / 16 * 16; }

template <typename T, bool H>
__device__ __forceinline__ void tail_smem_cycle(const MGLevel<T> *__restrict__ Ls, int first,
                                                int nl, int smoother, T w) {
  extern __shared__ __align__(16) unsigned char tail_raw[];
  __shared__ MGLevel<T> S[TAIL_MAX_LEVELS];
  __shared__ TailSeg seg[7 * TAIL_MAX_LEVELS + 1];
  __shared__ int nseg;
  const int nt = nl - first;
  if ((int)threadIdx.x < nt) S[threadIdx.x] = Ls[first + threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned char *p = tail_raw;
    int ns = 0, e = 0, maxn = 0;
    auto place = [&](auto &ptr, int n, bool load) {
      using E = typename std::remove_pointer<typename std::remove_reference<decltype(ptr)>::type>::type;
      const long long bytes = (long long)n * (long long)sizeof(E);
      if (load) {
        seg[ns].dst = reinterpret_cast<uint32_t *>(p);
        seg[ns].src = reinterpret_cast<const uint32_t *>(ptr);
        seg[ns].start = e;
        ns++;
        e += (int)((bytes + 3) / 4);
      }
      ptr = reinterpret_cast<E *>(p);
      p += pad16(bytes);
    };
    for (int q = 0; q < nt; q++) {
      MGLevel<T> &L = S[q];
      const int n = (int)L.n;
      if constexpr (H) {
        for (int s = 0; s < 4; s++) place(L.h[s], n, true);
      } else {
        for (int s = 0; s < 4; s++) place(L.a[s], n, true);
      }
      place(L.x, n, false);
      place(L.b, n, q == 0);
      if (q < nt - 1) {
        if constexpr (H) {
          place(L.q1, n, true);
          place(L.q2, n, true);
        } else {
          place(L.p1, n, true);
          place(L.p2, n, true);
        }
      }
      maxn = n > maxn ? n : maxn;
    }
    for (int q = 0; q < nt; q++) S[q].t = reinterpret_cast<T *>(p);
    seg[ns].start = e;  // sentinel
    nseg = ns;
  }
  __syncthreads();
  const int E = seg[nseg].start;
  int sg = 0;
  for (int e0 = threadIdx.x; e0 < E; e0 += 8 * blockDim.x) {
    uint32_t v[8];
    uint32_t *d[8];
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
  tail_cycle<T, H>(S, 0, nt, smoother, w, S[0].t);
  T *xo = Ls[first].x;
  for (int c = threadIdx.x; c < (int)S[0].n; c += blockDim.x) xo[c] = S[0].x[c];
}

template <typename T, bool H>
__global__ void __launch_bounds__(TAIL_THREADS) k_vcycle_tail_smem(
    const MGLevel<T> *__restrict__ Ls, int first, int nl, int smoother, T w) {
  pdl_enter();
  tail_smem_cycle<T, H>(Ls, first, nl, smoother, w);
}

// Middle levels on one thread-block cluster: levels mid .. tail-1 hold tens
// of thousands of cells, too few to fill the GPU but enough that one block
// is slow on them.  The cluster's blocks walk their phases together in one
// launch (barrier.cluster between phases, data in global memory / L2), and
// block 0 alone runs the tail levels tail .. nl-1 in between, in shared
// memory when tail_in_smem (as k_vcycle_tail_smem) or from global memory
// (as k_vcycle_tail).  Same phases and per-cell arithmetic as the grid
// kernels, so the V-cycle's result does not depend on where the levels run.
template <typename T, bool H>
__global__ void __launch_bounds__(TAIL_THREADS, 1) k_vcycle_mid(
    const MGLevel<T> *__restrict__ Ls, int mid, int tail, int nl, int smoother, T w, T *tmp,
    int tail_in_smem) {
  pdl_enter();
  for (int l = mid; l < tail; l++) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_down<T, H, ClusterTeam>(L, C, smoother, w, tmp);
  }
  if (cluster_rank() == 0) {
    if (tail_in_smem)
      tail_smem_cycle<T, H>(Ls, tail, nl, smoother, w);
    else
      tail_cycle<T, H, BlockTeam>(Ls, tail, nl, smoother, w, tmp);
  }
  ClusterTeam::sync();
  for (int l = tail - 1; l >= mid; l--) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_up<T, H, ClusterTeam>(L, C, smoother, w, tmp);
  }
}

// Levels mid .. tail-1 of a V-cycle on a grid team (cooperative launch):
// the down leg (pre-smooth, residual, restriction per level) in one launch,
// the up leg (prolongation and correction, post-smooth per level) in
// another, the tail levels in between in their own single-block kernel.
// Same phases and per-cell arithmetic as the per-phase grid kernels, so the
// V-cycle's result does not depend on where the levels run.  A launch whose
// barrier gave up (error word set) stops after the phase it was in.
template <typename T, bool H>
__global__ void __launch_bounds__(GRID_THREADS) k_vcycle_grid_down(
    const MGLevel<T> *__restrict__ Ls, int mid, int tail, int smoother, T w, T *tmp, GridCtl ctl) {
  if (threadIdx.x == 0) grid_ctl() = ctl;
  __syncthreads();
  for (int l = mid; l < tail; l++) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_down<T, H, GridTeam>(L, C, smoother, w, tmp);
    if (*(volatile int *)ctl.err) return;
  }
}
template <typename T, bool H>
__global__ void __launch_bounds__(GRID_THREADS) k_vcycle_grid_up(
    const MGLevel<T> *__restrict__ Ls, int mid, int tail, int smoother, T w, T *tmp, GridCtl ctl) {
  if (threadIdx.x == 0) grid_ctl() = ctl;
  __syncthreads();
  for (int l = tail - 1; l >= mid; l--) {
    const MGLevel<T> L = Ls[l], C = Ls[l + 1];
    team_up<T, H, GridTeam>(L, C, smoother, w, tmp);
    if (*(volatile int *)ctl.err) return;
  }
}

template <typename T>
size_t tail_smem_bytes(const MGLevel<T> *L, int first, int nl, bool h16) {
  if (nl - first > TAIL_MAX_LEVELS) return ~(size_t)0;
  long long bytes = 0, maxn = 0;
  for (int q = first; q < nl; q++) {
    const long long n = L[q].n;
    bytes += h16 ? 4 * pad16(2 * n) : 4 * pad16((long long)sizeof(T) * n);  // operator
    bytes += 2 * pad16((long long)sizeof(T) * n);                          // x, b
    if (q < nl - 1) bytes += 2 * pad16((long long)sizeof(T) * n);          // weights
    maxn = n > maxn ? n : maxn;
  }
  bytes += pad16((long long)sizeof(T) * maxn);
  return (size_t)bytes;
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

// one converted element: (TO) v, or with a scale s (H mode) the FP32
// product (float) v * s (into the V-cycle) / v * s widened (out of it)
template <typename TI, typename TO>
__device__ __forceinline__ TO cvt(TI v, const float *s, long long i) {
  if (!s) return (TO)v;
  return (TO)((float)v * s[i]);
}

// out = (TO) in (times scale when given); with vec set (all pointers 16-byte
// aligned) each thread moves four elements per vector access, which keeps
// enough bytes in flight for a streaming conversion to run at HBM bandwidth
template <typename TI, typename TO>
__global__ void k_convert(const TI *__restrict__ in, TO *__restrict__ out, long long n,
                          int vec, int flip, const float *__restrict__ scale) {
  pdl_enter();
  const long long bx = flip ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
  const long long t = bx * blockDim.x + threadIdx.x;
  const long long n4 = vec ? n / 4 : 0;
  if (t < n4) {
    TI a[4];
    TO b[4];
    ld4(in + 4 * t, a);
    if (scale) {
      float sv[4];
      ld4(scale + 4 * t, sv);
#pragma unroll
      for (int u = 0; u < 4; u++) b[u] = (TO)((float)a[u] * sv[u]);
    } else {
#pragma unroll
      for (int u = 0; u < 4; u++) b[u] = (TO)a[u];
    }
    st4(out + 4 * t, b);
  }
  const long long c = 4 * n4 + t;
  if (c < n && t < (vec ? 4 : n)) out[c] = cvt<TI, TO>(in[c], scale, c);
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
template <typename T, bool H>
static void setup_level_d(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st) {
  Shape3 g = shape3(C.nx, C.ny, C.nz);
  if (F.dir == 0)
    launch_pdl(k_setup_level<T, 0, H>, dim3(g.grid), dim3(g.block), st, F, C);
  else if (F.dir == 1)
    launch_pdl(k_setup_level<T, 1, H>, dim3(g.grid), dim3(g.block), st, F, C);
  else
    launch_pdl(k_setup_level<T, 2, H>, dim3(g.grid), dim3(g.block), st, F, C);
}
template <typename T>
void launch_mg_setup_level(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st,
                           bool h16) {
  if constexpr (kHasH16<T>) {
    if (h16) {
      setup_level_d<T, true>(F, C, st);
      return;
    }
  }
  setup_level_d<T, false>(F, C, st);
}
// the two-cells-per-thread sweep serves this level
template <typename T>
static bool rb_sweep_pairs(const MGLevel<T> &L, bool h16) {
  if constexpr (kHasH16<T>)
    return h16 && L.split && !getenv_flag_one_cell();
  else
    return false;
}
template <typename T>
static void rb_sweep(const MGLevel<T> &L, T *x, const T *b, int colour, int init,
                     cudaStream_t st, int flip, bool h16, int from_b = 0) {
  // two cells per thread on colour-split levels of the FP16 operator (it is
  // bound by instruction issue there; the FP32 and FP64 sweeps, bound by
  // memory, are as fast or faster with one cell per thread and more threads)
  if constexpr (kHasH16<T>) {
    if (rb_sweep_pairs(L, h16)) {
      Shape3 g2 = shape3((L.hx + 1) / 2, L.ny, L.nz);
      if (from_b)
        launch_pdl(k_rb_sweep2<T, true, true>, dim3(g2.grid), dim3(g2.block), st, L, x, b,
                   colour, init, flip);
      else
        launch_pdl(k_rb_sweep2<T, true>, dim3(g2.grid), dim3(g2.block), st, L, x, b, colour,
                   init, flip);
      return;
    }
  }
  Shape3 g = shape3((L.nx + 1) / 2, L.ny, L.nz);
  if constexpr (kHasH16<T>) {
    if (h16) {
      launch_pdl(k_rb_sweep<T, true>, dim3(g.grid), dim3(g.block), st, L, x, b, colour, init,
                 flip);
      return;
    }
  }
  launch_pdl(k_rb_sweep<T, false>, dim3(g.grid), dim3(g.block), st, L, x, b, colour, init, flip);
}
// RedBlackGSPoint, MaxIter 1: red, black, red (Symmetric True, smoother 0)
// or red, black (Symmetric False, smoother 2); a zero initial guess turns the
// first red sweep into x = b / a0 (rb_GS_point.c:107-240).  Smoother 9 is a
// single red sweep (kernel timing).
template <typename T>
int launch_mg_smooth(const MGLevel<T> &L, T *x, const T *b, int zero, int smoother,
                      double weight, T *tmp, cudaStream_t st, int *flip, bool h16) {
  const int f = flip ? *flip : 0, g = flip ? f ^ 1 : 0;
  if (smoother == 1) {
    Shape3 sh = shape3(L.nx, L.ny, L.nz);
    bool done = false;
    if constexpr (kHasH16<T>) {
      if (h16) {
        launch_pdl(k_wjacobi<T, true>, dim3(sh.grid), dim3(sh.block), st, L, x, b, tmp, zero);
        done = true;
      }
    }
    if (!done)
      launch_pdl(k_wjacobi<T, false>, dim3(sh.grid), dim3(sh.block), st, L, x, b, tmp, zero);
    launch_pdl(k_wjacobi_update<T>, dim3(nb(L.n, 256)), dim3(256), st, x, tmp, L.n, (T)weight,
               zero);
    return 2;
  }
  if (smoother == 9) {  // a single red sweep (kernel timing)
    rb_sweep(L, x, b, 0, 0, st, 0, h16);
    return 1;
  }
  if (smoother == 2) {
    rb_sweep(L, x, b, 0, zero, st, f, h16);
    rb_sweep(L, x, b, 1, 0, st, g, h16);
    if (flip) *flip = f;
    return 2;
  }
  if (zero && rb_sweep_pairs(L, h16) && skip_zero_sweep()) {
    // the black sweep reads the zero-guess red values from b; the last red
    // sweep writes x of the red cells
    rb_sweep(L, x, b, 1, 0, st, g, h16, 1);
    rb_sweep(L, x, b, 0, 0, st, f, h16);
    if (flip) *flip = g;
    return 2;
  }
  rb_sweep(L, x, b, 0, zero, st, f, h16);
  rb_sweep(L, x, b, 1, 0, st, g, h16);
  rb_sweep(L, x, b, 0, 0, st, f, h16);
  if (flip) *flip = g;
  return 3;
}
template <typename K>
static cudaError_t mid_prepare(K kern) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TAIL_SMEM_MAX);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

// opt the fused smoother, the shared-memory tails and the cluster kernel into
// their dynamic shared memory (> 48 KB) and cluster sizes above 8; called once
// per device before any launch or graph capture
cudaError_t mg_prepare_kernels() {
  cudaError_t e = rbr_fused_prepare<float>();
  if (e != cudaSuccess) return e;
  e = rbr_fused_prepare<double>();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_vcycle_tail_smem<float, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM_MAX);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_vcycle_tail_smem<float, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM_MAX);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_vcycle_tail_smem<double, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM_MAX);
  if (e != cudaSuccess) return e;
  e = mid_prepare(k_vcycle_mid<float, false>);
  if (e != cudaSuccess) return e;
  e = mid_prepare(k_vcycle_mid<float, true>);
  if (e != cudaSuccess) return e;
  return mid_prepare(k_vcycle_mid<double, false>);
}

template <typename T>
int vcycle_mid_cluster_size(bool h16, size_t smem) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16);
  cfg.blockDim = dim3(TAIL_THREADS);
  cfg.dynamicSmemBytes = smem;
  int cs = 0;
  cudaError_t e;
  if constexpr (kHasH16<T>)
    e = h16 ? cudaOccupancyMaxPotentialClusterSize(&cs, k_vcycle_mid<T, true>, &cfg)
            : cudaOccupancyMaxPotentialClusterSize(&cs, k_vcycle_mid<T, false>, &cfg);
  else
    e = cudaOccupancyMaxPotentialClusterSize(&cs, k_vcycle_mid<T, false>, &cfg);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return cs;
}

template <typename T>
void launch_mg_residual(const MGLevel<T> &L, const T *x, const T *b, T *r, cudaStream_t st,
                        int flip, bool h16, int zero_colour) {
  if (zero_colour >= 0) {
    Shape3 g = shape3((L.nx + 1) / 2, L.ny, L.nz);
    if constexpr (kHasH16<T>) {
      if (h16) {
        launch_pdl(k_mg_residual_pair<T, true>, dim3(g.grid), dim3(g.block), st, L, x, b, r,
                   flip, zero_colour);
        return;
      }
    }
    launch_pdl(k_mg_residual_pair<T, false>, dim3(g.grid), dim3(g.block), st, L, x, b, r, flip,
               zero_colour);
    return;
  }
  Shape3 g = shape3(L.nx, L.ny, L.nz);
  if constexpr (kHasH16<T>) {
    if (h16) {
      launch_pdl(k_mg_residual<T, true>, dim3(g.grid), dim3(g.block), st, L, x, b, r, flip);
      return;
    }
  }
  launch_pdl(k_mg_residual<T, false>, dim3(g.grid), dim3(g.block), st, L, x, b, r, flip);
}
template <typename T, bool H>
static void restrict_d(const MGLevel<T> &F, const MGLevel<T> &C, const T *rf, T *rc,
                       cudaStream_t st, int flip) {
  Shape3 g = shape3(C.nx, C.ny, C.nz);
  if (F.dir == 0)
    launch_pdl(k_restrict<T, H, 0>, dim3(g.grid), dim3(g.block), st, F, C, rf, rc, flip);
  else if (F.dir == 1)
    launch_pdl(k_restrict<T, H, 1>, dim3(g.grid), dim3(g.block), st, F, C, rf, rc, flip);
  else
    launch_pdl(k_restrict<T, H, 2>, dim3(g.grid), dim3(g.block), st, F, C, rf, rc, flip);
}
template <typename T, bool H>
static void prolong_d(const MGLevel<T> &F, const MGLevel<T> &C, const T *ec, T *xf,
                      cudaStream_t st, int flip, int skip_red) {
  Shape3 g = shape3(F.nx, F.ny, F.nz);
  if (F.dir == 0)
    launch_pdl(k_prolong_add<T, H, 0>, dim3(g.grid), dim3(g.block), st, F, C, ec, xf, flip,
               skip_red);
  else if (F.dir == 1)
    launch_pdl(k_prolong_add<T, H, 1>, dim3(g.grid), dim3(g.block), st, F, C, ec, xf, flip,
               skip_red);
  else
    launch_pdl(k_prolong_add<T, H, 2>, dim3(g.grid), dim3(g.block), st, F, C, ec, xf, flip,
               skip_red);
}
template <typename T>
void launch_mg_restrict(const MGLevel<T> &F, const MGLevel<T> &C, const T *rf, T *rc,
                        cudaStream_t st, int flip, bool h16) {
  if constexpr (kHasH16<T>) {
    if (h16) {
      restrict_d<T, true>(F, C, rf, rc, st, flip);
      return;
    }
  }
  restrict_d<T, false>(F, C, rf, rc, st, flip);
}
template <typename T>
void launch_mg_prolong_add(const MGLevel<T> &F, const MGLevel<T> &C, const T *ec, T *xf,
                           cudaStream_t st, int flip, bool h16, int skip_red) {
  if constexpr (kHasH16<T>) {
    if (h16) {
      prolong_d<T, true>(F, C, ec, xf, st, flip, skip_red);
      return;
    }
  }
  prolong_d<T, false>(F, C, ec, xf, st, flip, skip_red);
}
template <typename T>
void launch_vcycle_tail(const MGLevel<T> *levels_dev, int first, int nl, int smoother,
                        double weight, T *tmp, size_t smem, cudaStream_t st, bool h16) {
  if constexpr (kHasH16<T>) {
    if (h16) {
      if (smem > 0)
        launch_pdl_smem(k_vcycle_tail_smem<T, true>, dim3(1), dim3(TAIL_THREADS), smem, st,
                        levels_dev, first, nl, smoother, (T)weight);
      else
        launch_pdl(k_vcycle_tail<T, true>, dim3(1), dim3(512), st, levels_dev, first, nl,
                   smoother, (T)weight, tmp);
      return;
    }
  }
  if (smem > 0)
    launch_pdl_smem(k_vcycle_tail_smem<T, false>, dim3(1), dim3(TAIL_THREADS), smem, st,
                    levels_dev, first, nl, smoother, (T)weight);
  else
    launch_pdl(k_vcycle_tail<T, false>, dim3(1), dim3(512), st, levels_dev, first, nl, smoother,
               (T)weight, tmp);
}
template <typename T>
void launch_vcycle_mid(const MGLevel<T> *levels_dev, int mid, int tail, int nl, int smoother,
                       double weight, T *tmp, size_t smem, int cs, cudaStream_t st, bool h16) {
  const int in_smem = smem > 0 ? 1 : 0;
  if constexpr (kHasH16<T>) {
    if (h16) {
      launch_pdl_cluster(k_vcycle_mid<T, true>, cs, dim3(TAIL_THREADS), smem, st, levels_dev,
                         mid, tail, nl, smoother, (T)weight, tmp, in_smem);
      return;
    }
  }
  launch_pdl_cluster(k_vcycle_mid<T, false>, cs, dim3(TAIL_THREADS), smem, st, levels_dev, mid,
                     tail, nl, smoother, (T)weight, tmp, in_smem);
}
// blocks of the cooperative V-cycle kernels: as many as the device keeps
// resident at once, at most per_sm per SM (cooperative-launch limit)
template <typename T>
int vcycle_grid_blocks(bool h16, int per_sm) {
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  cudaError_t e;
  if constexpr (kHasH16<T>) {
    if (h16)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_vcycle_grid_down<T, true>,
                                                        GRID_THREADS, 0);
    else
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_vcycle_grid_down<T, false>,
                                                        GRID_THREADS, 0);
  } else {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_vcycle_grid_down<T, false>,
                                                      GRID_THREADS, 0);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int up = 0;
  if constexpr (kHasH16<T>) {
    if (h16)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up, k_vcycle_grid_up<T, true>,
                                                        GRID_THREADS, 0);
    else
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up, k_vcycle_grid_up<T, false>,
                                                        GRID_THREADS, 0);
  } else {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up, k_vcycle_grid_up<T, false>,
                                                      GRID_THREADS, 0);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  occ = occ < up ? occ : up;
  if (occ > per_sm) occ = per_sm;
  return occ * sms;
}

template <typename K, typename... Args>
static cudaError_t launch_coop(K kern, int blocks, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(GRID_THREADS);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename T>
cudaError_t launch_vcycle_grid(const MGLevel<T> *levels_dev, int mid, int tail, int up,
                               int smoother, double weight, T *tmp, int blocks, GridCtl ctl,
                               cudaStream_t st, bool h16) {
  // a counter left by a launch whose barrier gave up starts from zero again
  cudaError_t e = cudaMemsetAsync(ctl.count, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  const T w = (T)weight;
  if constexpr (kHasH16<T>) {
    if (h16)
      return up ? launch_coop(k_vcycle_grid_up<T, true>, blocks, st, levels_dev, mid, tail,
                              smoother, w, tmp, ctl)
                : launch_coop(k_vcycle_grid_down<T, true>, blocks, st, levels_dev, mid, tail,
                              smoother, w, tmp, ctl);
  }
  return up ? launch_coop(k_vcycle_grid_up<T, false>, blocks, st, levels_dev, mid, tail,
                          smoother, w, tmp, ctl)
            : launch_coop(k_vcycle_grid_down<T, false>, blocks, st, levels_dev, mid, tail,
                          smoother, w, tmp, ctl);
}

template <typename T>
void launch_setup_tail(const MGLevel<T> *levels_dev, int first, int nl, cudaStream_t st) {
  launch_pdl(k_setup_tail<T>, dim3(1), dim3(512), st, levels_dev, first, nl);
}

// ---------------------------------------------------------------------------
// Scaled FP16 operator (H mode): from the plain FP32 operator of level F (and
// the diagonal of the next coarser level C) build h = off-diagonals over
// S_i S_j and the diagonal C / S^2, the scaled transfer weights q1/q2 and, on
// level 0, sinv = 1/S, with S = sqrt(|C|) (1 where C is 0 or not finite).
// 1/S comes from the hardware reciprocal square root (a few ulp): the
// results are stored as 11-bit FP16 significands, the +-1 diagonal rounds
// exactly, and sinv is used consistently on the way into and out of the cycle.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void h16_scale_cell(const MGLevel<float> &F, const MGLevel<float> &C,
                                               int has_coarse, int i, int j, int k) {
  if (i >= F.nx || j >= F.ny || k >= F.nz) return;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int sy = nx, sz = nx * ny;
  const int c = i + sy * j + sz * k;
  const float *a0 = F.a[0];
  // every operand first (predicated loads, one round trip per thread)
  const float cd = a0[c];
  const float ce = i + 1 < nx ? a0[c + 1] : 0.0f;
  const float cn = j + 1 < ny ? a0[c + sy] : 0.0f;
  const float cu = k + 1 < nz ? a0[c + sz] : 0.0f;
  const float e = F.a[1][c], n = F.a[2][c], u = F.a[3][c];
  const int d = F.dir;
  const int ci = d == 0 ? i : d == 1 ? j : k;
  const int nd = d == 0 ? nx : d == 1 ? ny : nz;
  const int ncd = d == 0 ? C.nx : d == 1 ? C.ny : C.nz;
  float w1 = 0.0f, w2 = 0.0f, clo = 0.0f, chi = 0.0f;
  if (has_coarse) {
    // p1/p2 are zero at coarse points (written at fine points only)
    w1 = F.p1[c];
    w2 = F.p2[c];
    const int lo = ci >> 1, hi = (ci + 1) >> 1;  // coarse point at/below, at/above
    const int il = d == 0 ? lo : i, jl = d == 1 ? lo : j, kl = d == 2 ? lo : k;
    clo = C.a[0][il + C.nx * (jl + C.ny * kl)];
    if (hi < ncd) {
      const int ih = d == 0 ? hi : i, jh = d == 1 ? hi : j, kh = d == 2 ? hi : k;
      chi = C.a[0][ih + C.nx * (jh + C.ny * kh)];
    }
  }
  const float ic = h16_store(F, c, cd, e, n, u, i + 1 < nx, ce, j + 1 < ny, cn, k + 1 < nz, cu);
  if (!has_coarse) return;
  const float sf = scale_from(cd, ic);
  if (!(ci & 1)) {
    F.q1[c] = sf * inv_scale_of(clo);
    F.q2[c] = 0.0f;
  } else {
    F.q1[c] = w1 * sf * inv_scale_of(clo);
    F.q2[c] = ci + 1 < nd ? w2 * sf * inv_scale_of(chi) : 0.0f;
  }
}

__global__ void k_h16_scale(MGLevel<float> F, MGLevel<float> C, int has_coarse) {
  pdl_enter();
  int i, j, k;
  thread_ijk(i, j, k);
  h16_scale_cell(F, C, has_coarse, i, j, k);
}

__global__ void __launch_bounds__(512) k_h16_scale_tail(const MGLevel<float> *__restrict__ Ls,
                                                        int first, int nl) {
  pdl_enter();
  for (int l = first; l < nl; l++) {
    const MGLevel<float> F = Ls[l];
    const MGLevel<float> C = Ls[l + 1 < nl ? l + 1 : l];
    for (int t = threadIdx.x; t < (int)F.n; t += blockDim.x) {
      int i, j, k;
      split_ijk(t, F.nx, F.ny, i, j, k);
      h16_scale_cell(F, C, l + 1 < nl, i, j, k);
    }
  }
}

void launch_h16_scale(const MGLevel<float> &F, const MGLevel<float> *C, cudaStream_t st) {
  Shape3 g = shape3(F.nx, F.ny, F.nz);
  launch_pdl(k_h16_scale, dim3(g.grid), dim3(g.block), st, F, C ? *C : F, C ? 1 : 0);
}
void launch_h16_scale_tail(const MGLevel<float> *levels_dev, int first, int nl,
                           cudaStream_t st) {
  launch_pdl(k_h16_scale_tail, dim3(1), dim3(512), st, levels_dev, first, nl);
}

// level-0 transfers of the preconditioner: a natural-layout FP64 vector into
// b of level 0 (its storage type and layout, times the FP16 scaling when
// given), and x of level 0 back out
// Each thread moves one cell in each of four consecutive planes: accesses
// stay contiguous across a warp (in the natural vector and within each
// colour block) and four loads are in flight per thread.
constexpr int LEVEL_PLANES = 4;

template <typename TO>
__global__ void k_level_in(MGLevel<TO> L, const double *__restrict__ in, TO *__restrict__ out,
                           const float *__restrict__ scale) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k0 = LEVEL_PLANES * blockIdx.z;
  if (i >= L.nx || j >= L.ny) return;
  const int sz = L.nx * L.ny, c0 = i + L.nx * j + sz * k0;
  double v[LEVEL_PLANES];
#pragma unroll
  for (int u = 0; u < LEVEL_PLANES; u++) v[u] = k0 + u < L.nz ? in[c0 + u * sz] : 0.0;
#pragma unroll
  for (int u = 0; u < LEVEL_PLANES; u++)
    if (k0 + u < L.nz)
      out[xb_index(L, i, j, k0 + u)] = cvt<double, TO>(v[u], scale, c0 + u * sz);
}
template <typename TI>
__global__ void k_level_out(MGLevel<TI> L, const TI *__restrict__ in, double *__restrict__ out,
                            const float *__restrict__ scale, int flip) {
  pdl_enter();
  const int by = flip ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k0 = LEVEL_PLANES * (flip ? gridDim.z - 1 - blockIdx.z : blockIdx.z);
  if (i >= L.nx || j >= L.ny) return;
  const int sz = L.nx * L.ny, c0 = i + L.nx * j + sz * k0;
  TI v[LEVEL_PLANES];
#pragma unroll
  for (int u = 0; u < LEVEL_PLANES; u++)
    v[u] = k0 + u < L.nz ? in[xb_index(L, i, j, k0 + u)] : TI(0);
#pragma unroll
  for (int u = 0; u < LEVEL_PLANES; u++)
    if (k0 + u < L.nz) out[c0 + u * sz] = cvt<TI, double>(v[u], scale, c0 + u * sz);
}

template <typename T>
int launch_level_in(const MGLevel<T> &L, const double *r, const float *scale, cudaStream_t st) {
  if (L.split) {
    Shape3 g = shape3(L.nx, L.ny, (L.nz + LEVEL_PLANES - 1) / LEVEL_PLANES);
    launch_pdl(k_level_in<T>, dim3(g.grid), dim3(g.block), st, L, r, L.b, scale);
    return 1;
  }
  if (std::is_same<T, double>::value && !scale) {
    cudaMemcpyAsync(L.b, r, L.n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    return 0;
  }
  launch_convert<double, T>(r, L.b, L.n, st, 0, scale);
  return 1;
}
template <typename T>
int launch_level_out(const MGLevel<T> &L, const T *x, double *z, const float *scale, int flip,
                     cudaStream_t st) {
  if (L.split) {
    Shape3 g = shape3(L.nx, L.ny, (L.nz + LEVEL_PLANES - 1) / LEVEL_PLANES);
    launch_pdl(k_level_out<T>, dim3(g.grid), dim3(g.block), st, L, x, z, scale, flip);
    return 1;
  }
  if (std::is_same<T, double>::value && !scale) {
    cudaMemcpyAsync(z, x, L.n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    return 0;
  }
  launch_convert<T, double>(x, z, L.n, st, flip, scale);
  return 1;
}
template int launch_level_in<float>(const MGLevel<float> &, const double *, const float *,
                                    cudaStream_t);
template int launch_level_in<double>(const MGLevel<double> &, const double *, const float *,
                                     cudaStream_t);
template int launch_level_out<float>(const MGLevel<float> &, const float *, double *,
                                     const float *, int, cudaStream_t);
template int launch_level_out<double>(const MGLevel<double> &, const double *, double *,
                                      const float *, int, cudaStream_t);

template <typename TI, typename TO>
void launch_convert(const TI *in, TO *out, long long n, cudaStream_t st, int flip,
                    const float *scale) {
  const int vec = (((uintptr_t)in | (uintptr_t)out | (uintptr_t)scale) & 15) == 0;
  const long long threads = vec ? (n / 4 > 4 ? n / 4 : 4) : (n > 1 ? n : 1);
  launch_pdl(k_convert<TI, TO>, dim3(nb(threads, 256)), dim3(256), st, in, out, n, vec, flip,
             scale);
}

#define INST(T)                                                                              \
  template void launch_mg_prolong_weights<T>(const MGLevel<T> &, cudaStream_t);               \
  template void launch_mg_coarse_op<T>(const MGLevel<T> &, const MGLevel<T> &, cudaStream_t); \
  template void launch_mg_setup_level<T>(const MGLevel<T> &, const MGLevel<T> &, cudaStream_t, \
                                         bool);                                               \
  template int launch_mg_smooth<T>(const MGLevel<T> &, T *, const T *, int, int, double, T *,  \
                                    cudaStream_t, int *, bool);                               \
  template void launch_mg_residual<T>(const MGLevel<T> &, const T *, const T *, T *,          \
                                      cudaStream_t, int, bool, int);                          \
  template void launch_mg_restrict<T>(const MGLevel<T> &, const MGLevel<T> &, const T *, T *, \
                                      cudaStream_t, int, bool);                               \
  template void launch_mg_prolong_add<T>(const MGLevel<T> &, const MGLevel<T> &, const T *,   \
                                         T *, cudaStream_t, int, bool, int);                  \
  template void launch_vcycle_mid<T>(const MGLevel<T> *, int, int, int, int, double, T *,       \
                                     size_t, int, cudaStream_t, bool);                         \
  template int vcycle_mid_cluster_size<T>(bool, size_t);                                       \
  template int vcycle_grid_blocks<T>(bool, int);                                               \
  template cudaError_t launch_vcycle_grid<T>(const MGLevel<T> *, int, int, int, int, double, T *, \
                                             int, GridCtl, cudaStream_t, bool);                \
  template void launch_vcycle_tail<T>(const MGLevel<T> *, int, int, int, double, T *, size_t, \
                                      cudaStream_t, bool);                                    \
  template size_t tail_smem_bytes<T>(const MGLevel<T> *, int, int, bool);                    \
  template void launch_setup_tail<T>(const MGLevel<T> *, int, int, cudaStream_t);
INST(double)
INST(float)
template void launch_convert<double, float>(const double *, float *, long long, cudaStream_t, int,
                                            const float *);
template void launch_convert<float, double>(const float *, double *, long long, cudaStream_t, int,
                                            const float *);
template void launch_convert<double, double>(const double *, double *, long long, cudaStream_t,
                                             int, const float *);

}  // namespace pfgpu
