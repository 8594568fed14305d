// Grid vectors, deterministic reductions and the scalar side of GMRES.
//
// Reductions: a fixed grid of blocks writes one partial per block; the last
// block to finish (ticket counter) sums the partials in index order, so every
// result is bitwise reproducible run to run.  Results stay in device memory.
// The scalar GMRES steps (modified Gram-Schmidt bookkeeping, Givens QR,
// back substitution) run in one thread on device-resident scalars and follow
// pfsimulator/kinsol/iterativ.c:30-286 and spgmr.c:168-450.
#include "pdl.cuh"
#include "pfgpu_kernels.h"
#include "nk_control.h"

namespace pfgpu {

static const int RED_THREADS = 256;
static const int RED_BLOCKS = 592;  // 4 x 148 SMs

int reduce_blocks() { return RED_BLOCKS; }


struct OpDot {
  const double *a, *b;
  __device__ double operator()(long long i) const { return a[i] * b[i]; }
  __device__ static double comb(double x, double y) { return x + y; }
  __device__ static double init() { return 0.0; }
};
struct OpMaxAbs {
  const double *a;
  __device__ double operator()(long long i) const { return fabs(a[i]); }
  __device__ static double comb(double x, double y) { return x > y ? x : y; }
  __device__ static double init() { return 0.0; }
};
struct OpStep {  // |s| / (1/1 + |u|)  (KINScSteplength, kinsol.c:1490-1505)
  const double *s, *u;
  __device__ double operator()(long long i) const { return fabs(s[i] / (1.0 / 1.0 + fabs(u[i]))); }
  __device__ static double comb(double x, double y) { return x > y ? x : y; }
  __device__ static double init() { return 0.0; }
};
struct OpStepDiff {  // |a - b| / (1 + |a|)  (KINStop, kinsol.c:1541-1544)
  const double *a, *b;
  __device__ double operator()(long long i) const {
    return fabs((a[i] - b[i]) / (1.0 / 1.0 + fabs(a[i])));
  }
  __device__ static double comb(double x, double y) { return x > y ? x : y; }
  __device__ static double init() { return 0.0; }
};

template <typename Op>
__global__ void __launch_bounds__(RED_THREADS) k_reduce(Op op, long long n, double *partial,
                                                        double *dst, unsigned int *ticket,
                                                        const double *gate) {
  pdl_enter();
  __shared__ double sh[RED_THREADS / 32];
  __shared__ bool last;
  if (gate && *gate == 0.0) return;  // reduction not needed this time
  double acc = Op::init();
  for (long long i = blockIdx.x * (long long)RED_THREADS + threadIdx.x; i < n;
       i += (long long)gridDim.x * RED_THREADS)
    acc = Op::comb(acc, op(i));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc = Op::comb(acc, __shfl_down_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = sh[0];
    for (int w = 1; w < RED_THREADS / 32; w++) b = Op::comb(b, sh[w]);
    partial[blockIdx.x] = b;
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  // last block: ordered final sum
  __threadfence();
  double v = Op::init();
  for (int i = threadIdx.x; i < (int)gridDim.x; i += RED_THREADS) {
    double pv = ((volatile double *)partial)[i];
    v = (i == (int)threadIdx.x) ? pv : Op::comb(v, pv);
  }
  // fixed-order tree over threads
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Op::comb(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sh[0];
    for (int w = 1; w < RED_THREADS / 32; w++) r = Op::comb(r, sh[w]);
    *dst = r;
    *ticket = 0u;
  }
}

template <typename Op>
static void reduce(Op op, long long n, double *dst, ReduceBuf rb, cudaStream_t st,
                   const double *gate = nullptr) {
  long long need = (n + RED_THREADS - 1) / RED_THREADS;
  int blocks = (int)(need < rb.blocks ? need : rb.blocks);
  if (blocks < 1) blocks = 1;
  launch_pdl(k_reduce<Op>, dim3(blocks), dim3(RED_THREADS), st, op, n, rb.partial, dst, rb.ticket, gate);
}

void launch_dot(const double *a, const double *b, long long n, double *dst, ReduceBuf rb,
                cudaStream_t st) {
  OpDot op{a, b};
  reduce(op, n, dst, rb, st);
}
void launch_dot_gated(const double *a, const double *b, long long n, double *dst,
                      const double *gate, ReduceBuf rb, cudaStream_t st) {
  OpDot op{a, b};
  reduce(op, n, dst, rb, st, gate);
}
void launch_maxabs(const double *a, long long n, double *dst, ReduceBuf rb, cudaStream_t st) {
  OpMaxAbs op{a};
  reduce(op, n, dst, rb, st);
}
void launch_steplen(const double *s, const double *u, long long n, double *dst, ReduceBuf rb,
                    cudaStream_t st) {
  OpStep op{s, u};
  reduce(op, n, dst, rb, st);
}
void launch_steplen_diff(const double *a, const double *b, long long n, double *dst,
                         ReduceBuf rb, cudaStream_t st) {
  OpStepDiff op{a, b};
  reduce(op, n, dst, rb, st);
}

// ---- fused multi-value reductions ------------------------------------------
// One pass over the vectors for several sums / maxima that the solver needs
// together; each value is reduced exactly like k_reduce (per-thread grid-
// stride accumulation, fixed-order block and final combination).  An op
// may also update a vector element-wise in the same pass (MGS axpy).
static const int RED_MAX_K = 4;

template <typename Op>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_multi(Op op, long long n,
                                                              double *partial,
                                                              unsigned int *ticket) {
  constexpr int K = Op::K;
  pdl_enter();
  __shared__ double sh[K][RED_THREADS / 32];
  __shared__ bool last;
  Op o = op;
  o.setup();
  double acc[K];
#pragma unroll
  for (int q = 0; q < K; q++) acc[q] = 0.0;
  for (long long i = blockIdx.x * (long long)RED_THREADS + threadIdx.x; i < n;
       i += (long long)gridDim.x * RED_THREADS)
    o.acc(i, acc);
#pragma unroll
  for (int q = 0; q < K; q++) {
    double a = acc[q];
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) a = Op::comb(q, a, __shfl_down_sync(0xffffffffu, a, w));
    if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; q++) {
      double b = sh[q][0];
      for (int w = 1; w < RED_THREADS / 32; w++) b = Op::comb(q, b, sh[q][w]);
      partial[q * gridDim.x + blockIdx.x] = b;
    }
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int q = 0; q < K; q++) {
    double v = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += RED_THREADS) {
      double pv = ((volatile double *)partial)[q * gridDim.x + i];
      v = (i == (int)threadIdx.x) ? pv : Op::comb(q, v, pv);
    }
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) v = Op::comb(q, v, __shfl_down_sync(0xffffffffu, v, w));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; q++) {
      double r = sh[q][0];
      for (int w = 1; w < RED_THREADS / 32; w++) r = Op::comb(q, r, sh[q][w]);
      *o.dst[q] = r;
    }
    *ticket = 0u;
  }
}

__device__ __forceinline__ double comb_sum(double x, double y) { return x + y; }
__device__ __forceinline__ double comb_max(double x, double y) { return x > y ? x : y; }

// <vk, vk> and <v0, vk> (the first two dot products of ModifiedGS)
struct OpMgsFirst {
  static constexpr int K = 2;
  const double *vk, *v0;
  double *dst[K];
  __device__ void setup() {}
  __device__ void acc(long long i, double *v) const {
    const double a = vk[i];
    v[0] = v[0] + a * a;
    v[1] = v[1] + v0[i] * a;
  }
  __device__ static double comb(int, double x, double y) { return comb_sum(x, y); }
};
// y = y + sign * (*s) x, then <z, y> with the updated y (z = y when null):
// one ModifiedGS projection fused with the next dot product
struct OpAxpyDot {
  static constexpr int K = 1;
  double *y;
  const double *x, *s, *z;
  double sign, a;
  double *dst[K];
  __device__ void setup() { a = sign * (*s); }
  __device__ void acc(long long i, double *v) {
    const double yn = y[i] + a * x[i];
    y[i] = yn;
    const double zi = z ? z[i] : yn;
    v[0] = v[0] + zi * yn;
  }
  __device__ static double comb(int, double x, double y) { return comb_sum(x, y); }
};
// line-search inputs after the Newton direction p: <Jp, Jp>, <f, Jp>, <p, p>
// and max |p| / (1 + |u|)
struct OpLineSearchIn {
  static constexpr int K = 4;
  const double *jp, *f, *p, *u;
  double *dst[K];
  __device__ void setup() {}
  __device__ void acc(long long i, double *v) const {
    const double j = jp[i], pi = p[i];
    v[0] = v[0] + j * j;
    v[1] = v[1] + f[i] * j;
    v[2] = v[2] + pi * pi;
    v[3] = comb_max(v[3], fabs(pi / (1.0 / 1.0 + fabs(u[i]))));
  }
  __device__ static double comb(int q, double x, double y) {
    return q == 3 ? comb_max(x, y) : comb_sum(x, y);
  }
};
// after a trial step: <f, f>, max |f| and max |unew - u| / (1 + |unew|)
struct OpStepNorms {
  static constexpr int K = 2;
  const double *f;
  double *dst[K];
  __device__ void setup() {}
  __device__ void acc(long long i, double *v) const {
    const double fi = f[i];
    v[0] = v[0] + fi * fi;
    v[1] = comb_max(v[1], fabs(fi));
  }
  __device__ static double comb(int q, double x, double y) {
    return q == 0 ? comb_sum(x, y) : comb_max(x, y);
  }
};
// at KINSol's start: <u, u>, max |f|, <f, f>
struct OpInitNorms {
  static constexpr int K = 3;
  const double *u, *f;
  double *dst[K];
  __device__ void setup() {}
  __device__ void acc(long long i, double *v) const {
    const double ui = u[i], fi = f[i];
    v[0] = v[0] + ui * ui;
    v[1] = comb_max(v[1], fabs(fi));
    v[2] = v[2] + fi * fi;
  }
  __device__ static double comb(int q, double x, double y) {
    return q == 1 ? comb_max(x, y) : comb_sum(x, y);
  }
};

// <u, v>, <v, v> and sum |v| of a difference-quotient product (KINSpgmrAtimesDQ)
struct OpDQ {
  static constexpr int K = 3;
  const double *u, *v;
  double *dst[K];
  __device__ void setup() {}
  __device__ void acc(long long i, double *s) const {
    const double ui = u[i], vi = v[i];
    s[0] = s[0] + ui * vi;
    s[1] = s[1] + vi * vi;
    s[2] = s[2] + fabs(vi);
  }
  __device__ static double comb(int, double x, double y) { return comb_sum(x, y); }
};

template <typename Op>
static void reduce_multi(Op op, long long n, ReduceBuf rb, cudaStream_t st) {
  long long need = (n + RED_THREADS - 1) / RED_THREADS;
  int blocks = (int)(need < rb.blocks ? need : rb.blocks);
  if (blocks < 1) blocks = 1;
  launch_pdl(k_reduce_multi<Op>, dim3(blocks), dim3(RED_THREADS), st, op, n, rb.partial,
             rb.ticket);
}

int reduce_partials() { return RED_BLOCKS * RED_MAX_K; }

void launch_mgs_first(const double *vk, const double *v0, long long n, double *d_vk2,
                      double *d_h0, ReduceBuf rb, cudaStream_t st) {
  OpMgsFirst op{vk, v0, {d_vk2, d_h0}};
  reduce_multi(op, n, rb, st);
}
void launch_axpy_dot(double *y, const double *x, const double *s, double sign, const double *z,
                     long long n, double *dst, ReduceBuf rb, cudaStream_t st) {
  OpAxpyDot op{y, x, s, z, sign, 0.0, {dst}};
  reduce_multi(op, n, rb, st);
}
void launch_linesearch_inputs(const double *jp, const double *f, const double *p,
                              const double *u, long long n, double *d_jp2, double *d_fjp,
                              double *d_p2, double *d_plen, ReduceBuf rb, cudaStream_t st) {
  OpLineSearchIn op{jp, f, p, u, {d_jp2, d_fjp, d_p2, d_plen}};
  reduce_multi(op, n, rb, st);
}
void launch_step_norms(const double *f, long long n, double *d_f2, double *d_fmax, ReduceBuf rb,
                       cudaStream_t st) {
  OpStepNorms op{f, {d_f2, d_fmax}};
  reduce_multi(op, n, rb, st);
}
void launch_init_norms(const double *u, const double *f, long long n, double *d_u2,
                       double *d_fmax, double *d_f2, ReduceBuf rb, cudaStream_t st) {
  OpInitNorms op{u, f, {d_u2, d_fmax, d_f2}};
  reduce_multi(op, n, rb, st);
}

// ---- difference-quotient J v (kinspgmr.c:481-518, uscale = 1) ---------------
// d[0..2] = <u, v>, <v, v>, |v|_1 from OpDQ; writes sigma to d[3] and 1/sigma
// to d[4]: sigma = sign(<u, v>) sqrt_relfunc max(|<u, v>|, |v|_1) / <v, v>
__global__ void k_dq_sigma(double *d, double sqrt_relfunc) {
  pdl_enter();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double sutsv = d[0], vtv = d[1], sq1norm = d[2];
    const double sign = (sutsv >= 0.0) ? 1.0 : -1.0;
    const double a = fabs(sutsv);
    const double sigma = sign * sqrt_relfunc * (a > sq1norm ? a : sq1norm) / vtv;
    d[3] = sigma;
    d[4] = 1.0 / sigma;
  }
}
// w = sigma v + u
__global__ void k_dq_point(double *__restrict__ w, const double *__restrict__ u,
                           const double *__restrict__ v, const double *__restrict__ d,
                           long long n) {
  pdl_enter();
  const double sigma = d[3];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    w[i] = sigma * v[i] + u[i];
}
// z = (1/sigma) (fw - f)
__global__ void k_dq_finish(double *__restrict__ z, const double *__restrict__ fw,
                            const double *__restrict__ f, const double *__restrict__ d,
                            long long n) {
  pdl_enter();
  const double sigma_inv = d[4];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = sigma_inv * (fw[i] - f[i]);
}
static inline int grid_for(long long n);
void launch_dq_prepare(const double *u, const double *v, long long n, double *d,
                       double sqrt_relfunc, ReduceBuf rb, cudaStream_t st) {
  OpDQ op{u, v, {d, d + 1, d + 2}};
  reduce_multi(op, n, rb, st);
  launch_pdl(k_dq_sigma, dim3(1), dim3(32), st, d, sqrt_relfunc);
}
void launch_dq_point(double *w, const double *u, const double *v, const double *d, long long n,
                     cudaStream_t st) {
  launch_pdl(k_dq_point, dim3(grid_for(n)), dim3(256), st, w, u, v, d, n);
}
void launch_dq_finish(double *z, const double *fw, const double *f, const double *d,
                      long long n, cudaStream_t st) {
  launch_pdl(k_dq_finish, dim3(grid_for(n)), dim3(256), st, z, fw, f, d, n);
}

// ---- element-wise ---------------------------------------------------------
__global__ void k_axpy_dev(double *__restrict__ y, const double *__restrict__ x,
                           const double *__restrict__ s, double sign, long long n) {
  pdl_enter();
  double a = sign * (*s);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}
__global__ void k_axpby(double *__restrict__ y, const double *__restrict__ x, double a, double b,
                        long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = (b == 0.0) ? a * x[i] : a * x[i] + b * y[i];
}
__global__ void k_xpay(double *__restrict__ z, const double *__restrict__ x, double a,
                       const double *__restrict__ y, long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = x[i] + a * y[i];
}
__global__ void k_scale_inv_dev(double *__restrict__ x, const double *__restrict__ s,
                                long long n) {
  pdl_enter();
  double a = 1.0 / (*s);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_scale(double *__restrict__ x, double a, long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_fill(double *__restrict__ x, double v, long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}
struct VecList {
  const double *v[NK_MAX_KRYLOV + 1];
};
// xcor = yg[0] V0 + 0, then xcor = yg[k] Vk + xcor (sequential N_VLinearSum order)
// xcor = sum_k yg[k] V_k, accumulated in k order onto 0 (accumulate = 0) or
// onto xcor itself (accumulate = 1: a GMRES restart cycle adds to the
// correction of the earlier cycles, spgmr.c:357-358)
__global__ void k_combine(double *__restrict__ xcor, VecList V, const double *__restrict__ yg,
                          int kdim, long long n, int accumulate) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = accumulate ? xcor[i] : 0.0;
    for (int k = 0; k < kdim; k++) acc = yg[k] * V.v[k][i] + 1.0 * acc;
    xcor[i] = acc;
  }
}

// restart direction V_0 = yg[0] V_0 + sum_{k=1..kdim} yg[k] V_k, in place
// (spgmr.c:405-409): every element reads only its own index
__global__ void k_restart_v0(double *v0, VecList V, const double *__restrict__ yg, int kdim,
                             long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = yg[0] * v0[i];
    for (int k = 1; k <= kdim; k++) acc = yg[k] * V.v[k][i] + 1.0 * acc;
    v0[i] = acc;
  }
}

static inline int grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

void launch_axpy_dev(double *y, const double *x, const double *s, double sign, long long n,
                     cudaStream_t st) {
  launch_pdl(k_axpy_dev, dim3(grid_for(n)), dim3(256), st, y, x, s, sign, n);
}
void launch_axpby(double *y, const double *x, double a, double b, long long n, cudaStream_t st) {
  launch_pdl(k_axpby, dim3(grid_for(n)), dim3(256), st, y, x, a, b, n);
}
void launch_xpay(double *z, const double *x, double a, const double *y, long long n,
                 cudaStream_t st) {
  launch_pdl(k_xpay, dim3(grid_for(n)), dim3(256), st, z, x, a, y, n);
}
void launch_scale_inv_dev(double *x, const double *s, long long n, cudaStream_t st) {
  launch_pdl(k_scale_inv_dev, dim3(grid_for(n)), dim3(256), st, x, s, n);
}
void launch_scale(double *x, double a, long long n, cudaStream_t st) {
  launch_pdl(k_scale, dim3(grid_for(n)), dim3(256), st, x, a, n);
}
void launch_fill(double *x, double v, long long n, cudaStream_t st) {
  launch_pdl(k_fill, dim3(grid_for(n)), dim3(256), st, x, v, n);
}
void launch_combine(double *xcor, double *const *V, const double *yg, int kdim, long long n,
                    cudaStream_t st, int accumulate) {
  VecList L;
  for (int k = 0; k < kdim && k <= NK_MAX_KRYLOV; k++) L.v[k] = V[k];
  launch_pdl(k_combine, dim3(grid_for(n)), dim3(256), st, xcor, L, yg, kdim, n, accumulate);
}
void launch_restart_v0(double *const *V, const double *yg, int kdim, long long n,
                       cudaStream_t st) {
  VecList L;
  for (int k = 0; k <= kdim && k <= NK_MAX_KRYLOV; k++) L.v[k] = V[k];
  launch_pdl(k_restart_v0, dim3(grid_for(n)), dim3(256), st, V[0], L, yg, kdim, n);
}

// ---- the same steps with their scalars on the device (graph solve) ---------
// V0 of a GMRES cycle: b / ||b|| = src * (bsign / r_norm) on the first cycle
// (as launch_axpby with b = 0), the restart direction / its norm after
__global__ void k_v0_init(double *__restrict__ v0, const double *__restrict__ src,
                          const NkState *S, const double *__restrict__ sc, long long n) {
  pdl_enter();
  const bool first = S->ntries == 0;
  const double a = first ? S->k.bsign * (1.0 / S->r_norm) : 1.0 / sc[SCI_RNORM];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (first)
      v0[i] = a * src[i];
    else
      v0[i] *= a;
  }
}
__global__ void k_combine_dev(double *__restrict__ xcor, VecList V, const double *__restrict__ yg,
                              const int *kdim_p, const int *acc_p, long long n) {
  pdl_enter();
  const int kdim = *kdim_p, accumulate = *acc_p;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = accumulate ? xcor[i] : 0.0;
    for (int k = 0; k < kdim; k++) acc = yg[k] * V.v[k][i] + 1.0 * acc;
    xcor[i] = acc;
  }
}
__global__ void k_restart_v0_dev(double *v0, VecList V, const double *__restrict__ yg,
                                 const int *kdim_p, long long n) {
  pdl_enter();
  const int kdim = *kdim_p;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = yg[0] * v0[i];
    for (int k = 1; k <= kdim; k++) acc = yg[k] * V.v[k][i] + 1.0 * acc;
    v0[i] = acc;
  }
}
__global__ void k_scale_inv_dev_unless(double *__restrict__ x, const double *__restrict__ s,
                                       const int *skip, long long n) {
  pdl_enter();
  if (*skip) return;
  double a = 1.0 / (*s);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_fill_if(double *__restrict__ x, double v, const int *flag, long long n) {
  pdl_enter();
  if (!*flag) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}
// a trial step: z = x + lam y, or z = x when lam == 0 (the copy of KINSOL's
// N_VScale(ONE, uu, unew))
__global__ void k_xpay_lam(double *__restrict__ z, const double *__restrict__ x,
                           const double *lam, const double *__restrict__ y, long long n) {
  pdl_enter();
  const double a = *lam;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = (a == 0.0) ? x[i] : x[i] + a * y[i];
}
__global__ void k_scale_by(double *__restrict__ x, const double *a_p, long long n) {
  pdl_enter();
  const double a = *a_p;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_copy_if(double *__restrict__ dst, const double *__restrict__ src,
                          const int *flag, long long n) {
  pdl_enter();
  if (!*flag) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

void launch_v0_init(double *v0, const double *src, const NkState *S, const double *sc,
                    long long n, cudaStream_t st) {
  launch_pdl(k_v0_init, dim3(grid_for(n)), dim3(256), st, v0, src, S, sc, n);
}
void launch_combine_dev(double *xcor, double *const *V, int nv, const double *yg, const int *kdim,
                        const int *accumulate, long long n, cudaStream_t st) {
  VecList L{};
  for (int k = 0; k < nv && k <= NK_MAX_KRYLOV; k++) L.v[k] = V[k];
  launch_pdl(k_combine_dev, dim3(grid_for(n)), dim3(256), st, xcor, L, yg, kdim, accumulate, n);
}
void launch_restart_v0_dev(double *const *V, int nv, const double *yg, const int *kdim,
                           long long n, cudaStream_t st) {
  VecList L{};
  for (int k = 0; k < nv && k <= NK_MAX_KRYLOV; k++) L.v[k] = V[k];
  launch_pdl(k_restart_v0_dev, dim3(grid_for(n)), dim3(256), st, V[0], L, yg, kdim, n);
}
void launch_scale_inv_dev_unless(double *x, const double *s, const int *skip, long long n,
                                 cudaStream_t st) {
  launch_pdl(k_scale_inv_dev_unless, dim3(grid_for(n)), dim3(256), st, x, s, skip, n);
}
void launch_fill_if(double *x, double v, const int *flag, long long n, cudaStream_t st) {
  launch_pdl(k_fill_if, dim3(grid_for(n)), dim3(256), st, x, v, flag, n);
}
void launch_xpay_lam(double *z, const double *x, const double *lam, const double *y, long long n,
                     cudaStream_t st) {
  launch_pdl(k_xpay_lam, dim3(grid_for(n)), dim3(256), st, z, x, lam, y, n);
}
void launch_scale_by(double *x, const double *a, long long n, cudaStream_t st) {
  launch_pdl(k_scale_by, dim3(grid_for(n)), dim3(256), st, x, a, n);
}
void launch_copy_if(double *dst, const double *src, const int *flag, long long n,
                    cudaStream_t st) {
  launch_pdl(k_copy_if, dim3(grid_for(n)), dim3(256), st, dst, src, flag, n);
}

// ---- GMRES scalars ----------------------------------------------------------
// S layout: [0, (lmax+1)*lmax) Hessenberg H(i,j) at i*lmax+j; then givens
// (2*lmax), yg (lmax+1), then named scalars.
struct GS {
  double *H, *giv, *yg, *sc;
  int lmax;
  __device__ double &h(int i, int j) { return H[i * lmax + j]; }
};
enum { SC_RNORM = 0, SC_ROT, SC_RHO, SC_VKNORM2, SC_NEWNORM2, SC_FLAG, SC_NN2, SC_NP, SC_GATE,
       SC_COEF, SC_HLL, SC_BETA, SC_QRFAIL };

__device__ GS gs_view(double *S, int lmax) {
  GS g;
  g.lmax = lmax;
  g.H = S;
  g.giv = S + (lmax + 1) * lmax;
  g.yg = g.giv + 2 * lmax;
  g.sc = g.yg + lmax + 1;
  return g;
}

__device__ void givens(double t1, double t2, double &c, double &s) {
  if (t2 == 0.0) {
    c = 1.0;
    s = 0.0;
  } else if (fabs(t2) >= fabs(t1)) {
    double t3 = t1 / t2;
    s = -1.0 / sqrt(1.0 + t3 * t3);
    c = -s * t3;
  } else {
    double t3 = t2 / t1;
    c = 1.0 / sqrt(1.0 + t3 * t3);
    s = -c * t3;
  }
}

__device__ __forceinline__ void gmres_scalar_op(int op, double *S, int l, int lmax) {
  GS g = gs_view(S, lmax);
  double *sc = g.sc;
  switch (op) {
    case 0: {  // start: r_norm = sqrt(<V0,V0>) already in SC_RNORM as squared
      double r = sqrt(sc[SC_RNORM]);
      sc[SC_RNORM] = r;
      sc[SC_BETA] = r;
      sc[SC_ROT] = 1.0;
      sc[SC_RHO] = r;
      for (int i = 0; i < (lmax + 1) * lmax; i++) g.H[i] = 0.0;
      break;
    }
    case 1: {  // after GS: H(i, k-1) stored by dots; compute new norm & reorth flag
      int k = l + 1;
      double vk_norm = sqrt(sc[SC_VKNORM2]);
      double new_norm = sqrt(sc[SC_NEWNORM2]);
      double temp = 1000.0 * vk_norm;
      sc[SC_FLAG] = ((temp + new_norm) != temp) ? 0.0 : 1.0;
      sc[SC_NN2] = 0.0;
      g.h(k, k - 1) = new_norm;
      break;
    }
    case 3: {  // QR update for column l and residual estimate (iterativ.c:205-250)
      int n = l + 1;
      if (l == 0) {
        double t1 = g.h(0, 0), t2 = g.h(1, 0), c, s;
        givens(t1, t2, c, s);
        g.giv[0] = c;
        g.giv[1] = s;
        g.h(0, 0) = c * t1 - s * t2;
      } else {
        int nm1 = n - 1;
        for (int k = 0; k < nm1; k++) {
          double t1 = g.h(k, nm1), t2 = g.h(k + 1, nm1);
          double c = g.giv[2 * k], s = g.giv[2 * k + 1];
          g.h(k, nm1) = c * t1 - s * t2;
          g.h(k + 1, nm1) = s * t1 + c * t2;
        }
        double t1 = g.h(nm1, nm1), t2 = g.h(n, nm1), c, s;
        givens(t1, t2, c, s);
        g.giv[2 * nm1] = c;
        g.giv[2 * nm1 + 1] = s;
        g.h(nm1, nm1) = c * t1 - s * t2;
      }
      sc[SC_ROT] *= g.giv[2 * l + 1];
      sc[SC_RHO] = fabs(sc[SC_ROT] * sc[SC_RNORM]);
      sc[SC_HLL] = g.h(l + 1, l);
      break;
    }
    case 4: {  // QRsol with krydim = l (iterativ.c:253-286)
      int kd = l;
      g.yg[0] = sc[SC_RNORM];
      for (int i = 1; i <= kd; i++) g.yg[i] = 0.0;
      for (int k = 0; k < kd; k++) {
        double c = g.giv[2 * k], s = g.giv[2 * k + 1];
        double t1 = g.yg[k], t2 = g.yg[k + 1];
        g.yg[k] = c * t1 - s * t2;
        g.yg[k + 1] = s * t1 + c * t2;
      }
      sc[SC_QRFAIL] = 0.0;
      for (int k = kd - 1; k >= 0; k--) {
        if (g.h(k, k) == 0.0) {
          sc[SC_QRFAIL] = 1.0;
          break;
        }
        g.yg[k] /= g.h(k, k);
        for (int i = 0; i < k; i++) g.yg[i] -= g.yg[k] * g.h(i, k);
      }
      break;
    }
    case 6: {  // restart (spgmr.c:390-404), krydim = l: the residual direction's
               // coefficients yg and the new r_norm
      int kd = l;
      double s_product = 1.0;
      for (int i = kd; i > 0; i--) {
        g.yg[i] = s_product * g.giv[2 * i - 2];
        s_product *= g.giv[2 * i - 1];
      }
      g.yg[0] = s_product;
      double r_norm = sc[SC_RNORM] * s_product;
      for (int i = 0; i <= kd; i++) g.yg[i] *= r_norm;
      sc[SC_RNORM] = fabs(r_norm);
      break;
    }
    case 7: {  // next restart cycle: Hessenberg cleared, rotation product 1
      sc[SC_ROT] = 1.0;
      for (int i = 0; i < (lmax + 1) * lmax; i++) g.H[i] = 0.0;
      break;
    }
    case 5: {  // finish reorthogonalisation: corrected new norm (iterativ.c:79-84)
      int k = l + 1;
      if (sc[SC_FLAG] != 0.0 && sc[SC_NN2] != 0.0) {
        double nn = g.h(k, k - 1);
        double np2 = nn * nn - sc[SC_NN2];
        g.h(k, k - 1) = (np2 > 0.0) ? sqrt(np2) : 0.0;
      }
      sc[SC_HLL] = g.h(k, k - 1);
      break;
    }
  }
}
__global__ void k_gmres_scalar(int op, double *S, int l, int lmax) {
  pdl_enter();
  gmres_scalar_op(op, S, l, lmax);
}
// the same step with its column / Krylov dimension read from the device
__global__ void k_gmres_scalar_dev(int op, double *S, const int *l, int lmax) {
  pdl_enter();
  gmres_scalar_op(op, S, *l, lmax);
}

// Reorthogonalisation decision for basis vector i against V_k
// (iterativ.c:68-77): dot result in SC_NP; sets SC_GATE (apply?) and SC_COEF.
__global__ void k_reorth_decide(double *S, int i, int l, int lmax) {
  pdl_enter();
  GS g = gs_view(S, lmax);
  double *sc = g.sc;
  int k = l + 1;
  sc[SC_GATE] = 0.0;
  if (sc[SC_FLAG] == 0.0) return;
  double new_product = sc[SC_NP];
  double temp = 1000.0 * g.h(i, k - 1);
  if ((temp + new_product) == temp) return;
  g.h(i, k - 1) += new_product;
  sc[SC_COEF] = -new_product;
  sc[SC_NN2] += new_product * new_product;
  sc[SC_GATE] = 1.0;
}

// y = y + (*coef) * x when *gate != 0
__global__ void k_axpy_gated(double *__restrict__ y, const double *__restrict__ x,
                             const double *__restrict__ coef, const double *__restrict__ gate,
                             long long n) {
  pdl_enter();
  if (*gate == 0.0) return;
  double a = *coef;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}

void launch_gmres_scalar(int op, double *S, int l, int lmax, cudaStream_t st) {
  launch_pdl(k_gmres_scalar, dim3(1), dim3(1), st, op, S, l, lmax);
}
void launch_gmres_scalar_dev(int op, double *S, const int *l, int lmax, cudaStream_t st) {
  launch_pdl(k_gmres_scalar_dev, dim3(1), dim3(1), st, op, S, l, lmax);
}
void launch_reorth_decide(double *S, int i, int l, int lmax, cudaStream_t st) {
  launch_pdl(k_reorth_decide, dim3(1), dim3(1), st, S, i, l, lmax);
}
void launch_axpy_gated(double *y, const double *x, const double *coef, const double *gate,
                       long long n, cudaStream_t st) {
  launch_pdl(k_axpy_gated, dim3(grid_for(n)), dim3(256), st, y, x, coef, gate, n);
}

// ---- ParFlow layout <-> dense ------------------------------------------------
__global__ void k_unpad(const double *__restrict__ pad, double *__restrict__ dense, int nx,
                        int ny, int nz) {
  pdl_enter();
  long long n = (long long)nx * ny * nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c % nx);
    long long r = c / nx;
    int j = (int)(r % ny), k = (int)(r / ny);
    dense[c] = pad[(i + 1) + (long long)(nx + 2) * ((j + 1) + (long long)(ny + 2) * (k + 1))];
  }
}
__global__ void k_pad(const double *__restrict__ dense, double *__restrict__ pad, int nx, int ny,
                      int nz) {
  pdl_enter();
  long long n = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c % (nx + 2)) - 1;
    long long r = c / (nx + 2);
    int j = (int)(r % (ny + 2)) - 1, k = (int)(r / (ny + 2)) - 1;
    bool in = i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
    pad[c] = in ? dense[i + (long long)nx * (j + (long long)ny * k)] : 0.0;
  }
}
// dense -> a frame of g ghost layers on every side (ghosts written as 0)
__global__ void k_pad_ghost(const double *__restrict__ dense, double *__restrict__ pad, int nx,
                            int ny, int nz, int g) {
  pdl_enter();
  const int px = nx + 2 * g, py = ny + 2 * g;
  long long n = (long long)px * py * (nz + 2 * g);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c % px) - g;
    long long r = c / px;
    int j = (int)(r % py) - g, k = (int)(r / py) - g;
    bool in = i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
    pad[c] = in ? dense[i + (long long)nx * (j + (long long)ny * k)] : 0.0;
  }
}
void launch_pad_ghost(const double *dense, double *pad, int nx, int ny, int nz, int g,
                      cudaStream_t st) {
  const long long n = (long long)(nx + 2 * g) * (ny + 2 * g) * (nz + 2 * g);
  launch_pdl(k_pad_ghost, dim3(grid_for(n)), dim3(256), st, dense, pad, nx, ny, nz, g);
}
void launch_unpad(const double *pad, double *dense, int nx, int ny, int nz, cudaStream_t st) {
  launch_pdl(k_unpad, dim3(grid_for((long long)nx * ny * nz)), dim3(256), st, pad, dense, nx, ny, nz);
}
void launch_pad(const double *dense, double *pad, int nx, int ny, int nz, cudaStream_t st) {
  launch_pdl(k_pad, dim3(grid_for((long long)(nx + 2) * (ny + 2) * (nz + 2))), dim3(256), st, dense, pad, nx, ny,
                                                                             nz);
}

}  // namespace pfgpu
