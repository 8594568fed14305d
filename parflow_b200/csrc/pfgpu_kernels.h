// Kernel launch interfaces shared between the library's translation units.
#pragma once

#include <vector>

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "pfgpu_device.cuh"

namespace pfgpu {

// Full 7-point Jacobian, stencil order of jacobian_stencil_shape
// (pfsimulator/parflow_lib/richards_jacobian_eval.c:126-132): C W E S N L U.
template <typename T>
struct JacOut {
  T *c, *w, *e, *s, *n, *l, *u;
};
template <typename T>
struct JacIn {
  const T *c, *w, *e, *s, *n, *l, *u;
};
// Symmetric operator: C and the upper entries E N U; W(i) = E(i-1),
// S(i) = N(i-nx), L(i) = U(i-nx*ny) (pfsimulator/parflow_lib/matrix.c:258-310).
// wg (ny*nz, optional): W of the i = 0 cells, i.e. the x_lower ghost column
// of E, which only the diffusive overland terms make nonzero.
// fd: the launch builds the preconditioner of Solver.Nonlinear.UseJacobian
// False (into M, or into J for PCMatrixType FullJacobian), which the
// reference assembles without the overland surface terms and with the
// diagonal term of its "simple" case on ponded OverlandFlow cells
// (richards_jacobian_eval.c:1241-1254, 1863, 2476-2484)
template <typename T>
struct PCOut {
  T *c, *e, *n, *u;
  T *wg;
  int fd;
};

void launch_vg_all(const DevProblem &P, const double *p, double *kr, double *dkr, double *sat,
                   double *dsat, cudaStream_t st);
void launch_saturation(const DevProblem &P, const double *p, double *s, cudaStream_t st);
// vel: also write the face velocities and overland fluxes (null: F only)
void launch_residual(const DevProblem &P, const double *p, const double *p_old,
                     const double *s_old, const double *kr, const double *sat, double dt,
                     double *f, cudaStream_t st, const VelOut *vel = nullptr);
template <typename TJ, typename TP>
void launch_jacobian(const DevProblem &P, const double *p, const double *kr, const double *dkr,
                     const double *sat, const double *dsat, double dt, JacOut<TJ> J,
                     PCOut<TP> M, cudaStream_t st);
// tile: a tuned thread-block shape (bx, by) or null for the heuristic
template <typename TJ>
void launch_matvec7(int nx, int ny, int nz, JacIn<TJ> J, const double *x, double *y,
                    cudaStream_t st, const int *tile = nullptr);

// ---- multigrid (mg_kernels.cu) --------------------------------------------
template <typename T>
struct MGLevel {
  int nx, ny, nz;
  long long n;
  int dir;          // coarsening direction to the next level (-1 on the coarsest)
  T *a[4];          // C E N U
  T *x, *b, *t;
  T *x2;            // output of the fused post-smoother (levels it runs on)
  T *p1, *p2;       // prolongation weights (fine points of this level)
  // (ny*nz) W entries of the i = 0 cells: the x_lower ghost column of E in
  // the reference's symmetric storage, which its setup reads (transverse sums
  // and coarse entries, mg_semi.c:563, 671-682) and which stays in the ghost
  // column of the coarser levels until a coarsening along x; zero unless the
  // finest operator has diffusive overland terms.  The smoothers and
  // residuals multiply it by a zero ghost iterate, so only the setup reads it.
  T *wg;
  // scaled FP16 operator (PFGPU_PREC_MIXED_H16): with S = sqrt(|C|) (1 where
  // C is 0 or not finite) the V-cycle runs on y = S x, b^ = b / S and
  // A^ = S^-1 A S^-1, whose off-diagonals A_ij / (S_i S_j) are h[0..2] =
  // E^ N^ U^ and whose diagonal C / S^2 is h[3]: +1 wherever C > 0, which
  // the kernels assume unless *hflag (set by the scaling pass when some
  // diagonal on some level is not +1) tells them to read h[3].  The transfer
  // weights absorb the scaling: q1 holds S_f / S_c at coarse points (even
  // indices along dir) and p1 S_f / S_c(below) at fine points, q2 holds
  // p2 S_f / S_c(above); sinv = 1 / S on level 0 only.
  __half *h[4];
  T *q1, *q2;
  T *sinv;
  const int *hflag;
  // colour-split storage of x and b (grid levels with the red/black smoother):
  // cell (i,j,k) of parity p = (i+j+k) & 1 lives at
  // p * hx*ny*nz + (i >> 1) + hx * (j + ny * k), hx = (nx + 1) / 2, so that a
  // colour sweep reads and writes whole lines of one colour only
  int split;
  int hx;
  // colour whose residual is written as zero right after the pre-smoother
  // (the colour it swept last: 0 red for red/black/red, 1 black for
  // red/black), or -1: every cell's residual is computed
  int zc;
  // PCMatrixType FullJacobian (mg_full.cu): W S L of the non-symmetric
  // finest operator (level 0 only, else null), and on every level the S of
  // the j = 0 cells (nx*nz) and the L of the k = 0 cells (nx*ny), the
  // y_lower / z_lower ghost planes of N and U that the setup of a coarse
  // operator writes (the companions of wg); null in the symmetric mode
  T *lo[3];
  T *sg, *lg;
};

// storage index of cell (i,j,k) in a level's x / b arrays
template <typename T>
__host__ __device__ __forceinline__ int xb_index(const MGLevel<T> &L, int i, int j, int k) {
  if (!L.split) return i + L.nx * (j + L.ny * k);
  return ((i + j + k) & 1) * (L.hx * L.ny * L.nz) + (i >> 1) + L.hx * (j + L.ny * k);
}

// One Gauss-Seidel point update x = (b - sum_nb a_nb x_nb) / a0, the six
// neighbour products accumulated in the order W E S N L U with explicit fused
// multiply-adds, so that every smoother kernel rounds identically.
template <typename T>
__device__ __forceinline__ T rb_update(T c, T b, T w, T xw, T e, T xe, T s, T xs, T n, T xn,
                                       T l, T xl, T u, T xu) {
  T acc = w * xw;
  acc = fma(e, xe, acc);
  acc = fma(s, xs, acc);
  acc = fma(n, xn, acc);
  acc = fma(l, xl, acc);
  acc = fma(u, xu, acc);
  return (b - acc) / c;
}

// Fused red/black/red smoother (mg_rbr.cu, TMA pipeline): tile, ring size
// and threads per storage type, box halo (x rounded up to the 16-byte rule)
// and the six tensor maps C E N U b x of one level.  The float tile is a
// compile-time tuning knob (PFGPU_RBR_F32_TY / _NS / _NTH).
template <typename T>
struct RbrTile;
#ifndef PFGPU_RBR_F32_TY
#define PFGPU_RBR_F32_TY 16
#define PFGPU_RBR_F32_NS 10
#define PFGPU_RBR_F32_NTH 1024
#endif
template <>
struct RbrTile<float> {
  static constexpr int TX = 32, TY = PFGPU_RBR_F32_TY, NS = PFGPU_RBR_F32_NS,
                       NTH = PFGPU_RBR_F32_NTH;
};
template <>
struct RbrTile<double> {
  static constexpr int TX = 32, TY = 8, NS = 8, NTH = 512;
};
constexpr int RBR_HX = 4, RBR_HY = 3;
struct RbrMaps {
  CUtensorMap m[6];
};
// level storage the TMA smoother can address (row pitch a multiple of 16 B)
template <typename T>
bool rbr_fused_eligible(const MGLevel<T> &L);
// tensor maps of level L with input iterate xin; 0 on success
template <typename T>
int make_rbr_maps(const MGLevel<T> &L, const T *xin, RbrMaps *out);
template <typename T>
cudaError_t rbr_fused_prepare();
// red, black, red on level L: b and the coefficients from the maps, the input
// iterate from maps.m[5] (not read when zero != 0), the result to xout, which
// must not be the input iterate; *err is set if a pipeline wait expires
template <typename T>
void launch_rbr_fused(const MGLevel<T> &L, const RbrMaps &maps, T *xout, int zero, int *err,
                      cudaStream_t st);

// Wavefront red/black/red smoother (mg_wave.cu): per-level control words,
// the (sweep, plane) order and the launch shape
struct WaveLevel {
  int *ctl = nullptr;   // item counter, abort flag, exit counter, per-(sweep, plane) counts
  int *plan = nullptr;  // (sweep, plane) tasks in wavefront order
  int rows = 0, nchunks = 0, grid = 0;
};
// lag: planes by which each sweep trails the one before (>= 2); chunk_cells:
// cells of one colour per work item
template <typename T>
int wave_setup(const MGLevel<T> &L, int ctas_per_sm, int lag, int chunk_cells, WaveLevel *w);
void wave_free(WaveLevel *w);
// red, black, red on level L in place (x not read when zero != 0); *err = 2
// if a dependency wait expires
template <typename T>
void launch_rbr_wave(const MGLevel<T> &L, const WaveLevel &w, T *x, const T *b, int zero,
                     int *err, cudaStream_t st);

template <typename T>
void launch_mg_prolong_weights(const MGLevel<T> &F, cudaStream_t st);
template <typename T>
void launch_mg_coarse_op(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st);
// prolongation weights of F and the coarse operator C in one launch
// (h16: also the scaled FP16 operator of F and its scaled transfer weights)
template <typename T>
void launch_mg_setup_level(const MGLevel<T> &F, const MGLevel<T> &C, cudaStream_t st,
                           bool h16 = false);
// flip (optional): block order of the first sweep (0 forward, 1 reversed);
// sweeps alternate and *flip returns the order the next launch should use;
// returns the number of kernels launched
// PCMatrixType FullJacobian (mg_full.cu): prolongation weights and coarse
// operators of all levels from a non-symmetric level 0; red/black sweeps
// (red, black and, when symmetric, red again; zero: zero initial guess) and
// the residual on the non-symmetric level 0.  Each returns its launches.
template <typename T>
int launch_mg_full_setup(const MGLevel<T> *L, int nl, cudaStream_t st);
template <typename T>
int launch_mg_full_smooth(const MGLevel<T> &L, T *x, const T *b, int zero, int symmetric,
                          cudaStream_t st);
template <typename T>
void launch_mg_full_residual(const MGLevel<T> &L, const T *x, const T *b, T *r,
                             cudaStream_t st);

template <typename T>
int launch_mg_smooth(const MGLevel<T> &L, T *x, const T *b, int zero, int smoother,
                      double weight, T *tmp, cudaStream_t st, int *flip = nullptr,
                      bool h16 = false);
cudaError_t mg_prepare_kernels();
// h16: the level's scaled FP16 operator and weights (float levels only)
template <typename T>
// r = b - A x; zero_colour >= 0: right after a sweep of that colour, whose
// cells' residual is written as zero
void launch_mg_residual(const MGLevel<T> &L, const T *x, const T *b, T *r, cudaStream_t st,
                        int flip = 0, bool h16 = false, int zero_colour = -1);
template <typename T>
void launch_mg_restrict(const MGLevel<T> &F, const MGLevel<T> &C, const T *rf, T *rc,
                        cudaStream_t st, int flip = 0, bool h16 = false);
template <typename T>
// xf += P ec; skip_red: only the black cells (the next sweep is a red one)
void launch_mg_prolong_add(const MGLevel<T> &F, const MGLevel<T> &C, const T *ec, T *xf,
                           cudaStream_t st, int flip = 0, bool h16 = false, int skip_red = 0);
// scaled FP16 operator of level F from its FP32 operator and the diagonal of
// the next coarser level C (null on the coarsest); sets *F.hflag when a
// scaled diagonal is not +1 (the flag is cleared before the first level)
void launch_h16_scale(const MGLevel<float> &F, const MGLevel<float> *C, cudaStream_t st);
void launch_h16_scale_tail(const MGLevel<float> *levels_dev, int first, int nl,
                           cudaStream_t st);
// levels `first` .. nl-1 of a V-cycle / of the setup in one single-block
// kernel; levels_dev is a device copy of the level table.  With smem > 0
// (tail_smem_bytes of those levels, at most TAIL_SMEM_MAX) the V-cycle tail
// runs out of shared memory, otherwise in global memory with tmp as scratch.
constexpr int TAIL_MAX_LEVELS = 32;
constexpr int TAIL_THREADS = 1024;
constexpr size_t TAIL_SMEM_MAX = 200 * 1024;
template <typename T>
size_t tail_smem_bytes(const MGLevel<T> *levels_host, int first, int nl, bool h16 = false);
template <typename T>
void launch_vcycle_tail(const MGLevel<T> *levels_dev, int first, int nl, int smoother,
                        double weight, T *tmp, size_t smem, cudaStream_t st, bool h16 = false);
// levels mid .. tail-1 of a V-cycle on one thread-block cluster of cs blocks
// (TAIL_THREADS threads each), block 0 of which runs the tail levels tail ..
// nl-1 in between (from shared memory when smem > 0, as launch_vcycle_tail)
template <typename T>
void launch_vcycle_mid(const MGLevel<T> *levels_dev, int mid, int tail, int nl, int smoother,
                       double weight, T *tmp, size_t smem, int cs, cudaStream_t st,
                       bool h16 = false);
// largest cluster the device co-schedules for that kernel (0 if none)
template <typename T>
int vcycle_mid_cluster_size(bool h16, size_t smem);
// levels mid .. tail-1 of a V-cycle on every block of a cooperative launch
// (blocks of GRID_THREADS threads, all resident at once): the down leg
// (up = 0) or the up leg (up = 1); the tail levels run in between in their
// own kernel.  ctl: the barrier's counter and generation words (device
// memory, the counter is cleared by this call) and the error word a barrier
// that gave up after one second sets to 3.
constexpr int GRID_THREADS = 512;
struct GridCtl {
  unsigned *count, *gen;
  int *err;
};
template <typename T>
cudaError_t launch_vcycle_grid(const MGLevel<T> *levels_dev, int mid, int tail, int up,
                               int smoother, double weight, T *tmp, int blocks, GridCtl ctl,
                               cudaStream_t st, bool h16 = false);
// blocks of those launches the device keeps resident at once, at most per_sm
// per SM (0 if the kernels cannot be launched cooperatively)
template <typename T>
int vcycle_grid_blocks(bool h16, int per_sm);
template <typename T>
void launch_setup_tail(const MGLevel<T> *levels_dev, int first, int nl, cudaStream_t st);
// a natural-layout FP64 vector r into b of level 0 / x of level 0 back into a
// natural FP64 vector z, in the level's type and layout (times the FP16
// scaling when scale is given); return the number of kernels launched
template <typename T>
int launch_level_in(const MGLevel<T> &L, const double *r, const float *scale, cudaStream_t st);
template <typename T>
int launch_level_out(const MGLevel<T> &L, const T *x, double *z, const float *scale, int flip,
                     cudaStream_t st);
// out = (TO) in, or (TO)((float) in * scale) when scale is given
template <typename TI, typename TO>
void launch_convert(const TI *in, TO *out, long long n, cudaStream_t st, int flip = 0,
                    const float *scale = nullptr);

// ---- PFB values (pfb_kernels.cu) --------------------------------------------
// out = big-endian bytes of dense[0..n)
void launch_pfb_pack(const double *dense, unsigned long long *out, long long n, cudaStream_t st);
// raw big-endian values of the subgrid box (ix..ix+snx) x (iy..) x (iz..) into
// the dense nx x ny x nz field
void launch_pfb_scatter(const unsigned long long *raw, double *dense, int nx, int ny, int ix,
                        int iy, int iz, int snx, int sny, int snz, cudaStream_t st);

// ---- vectors and reductions (krylov_kernels.cu) ----------------------------
struct ReduceBuf {
  double *partial;        // >= reduce_blocks() doubles
  unsigned int *ticket;   // one counter, zero between reductions
  int blocks;
};
int reduce_blocks();
int reduce_partials();  // doubles the partial buffer must hold (multi-value reductions)
// dst = sum(a .* b); deterministic (fixed grid, fixed order)
void launch_dot(const double *a, const double *b, long long n, double *dst, ReduceBuf rb,
                cudaStream_t st);
// as launch_dot, skipped entirely when *gate == 0
void launch_dot_gated(const double *a, const double *b, long long n, double *dst,
                      const double *gate, ReduceBuf rb, cudaStream_t st);
// dst = max |a|
void launch_maxabs(const double *a, long long n, double *dst, ReduceBuf rb, cudaStream_t st);
// dst = max |s| / (1 + |u|)
void launch_steplen(const double *s, const double *u, long long n, double *dst, ReduceBuf rb,
                    cudaStream_t st);
// dst = max |a - b| / (1 + |a|)
void launch_steplen_diff(const double *a, const double *b, long long n, double *dst,
                         ReduceBuf rb, cudaStream_t st);
// fused reductions (one pass each)
void launch_mgs_first(const double *vk, const double *v0, long long n, double *d_vk2,
                      double *d_h0, ReduceBuf rb, cudaStream_t st);
// y += sign * (*s) x, then dst = <z, y> (z null: <y, y>)
void launch_axpy_dot(double *y, const double *x, const double *s, double sign, const double *z,
                     long long n, double *dst, ReduceBuf rb, cudaStream_t st);
void launch_linesearch_inputs(const double *jp, const double *f, const double *p,
                              const double *u, long long n, double *d_jp2, double *d_fjp,
                              double *d_p2, double *d_plen, ReduceBuf rb, cudaStream_t st);
void launch_step_norms(const double *f, long long n, double *d_f2, double *d_fmax, ReduceBuf rb,
                       cudaStream_t st);
void launch_init_norms(const double *u, const double *f, long long n, double *d_u2,
                       double *d_fmax, double *d_f2, ReduceBuf rb, cudaStream_t st);
// y = y + (sign * (*s)) * x
void launch_axpy_dev(double *y, const double *x, const double *s, double sign, long long n,
                     cudaStream_t st);
// y = a*x + b*y (host scalars)
void launch_axpby(double *y, const double *x, double a, double b, long long n, cudaStream_t st);
// difference-quotient J v (KINSpgmrAtimesDQ): the sums and sigma into d[0..4],
// the point u + sigma v, and (F(u + sigma v) - F(u)) / sigma
void launch_dq_prepare(const double *u, const double *v, long long n, double *d,
                       double sqrt_relfunc, ReduceBuf rb, cudaStream_t st);
void launch_dq_point(double *w, const double *u, const double *v, const double *d, long long n,
                     cudaStream_t st);
void launch_dq_finish(double *z, const double *fw, const double *f, const double *d,
                      long long n, cudaStream_t st);
// z = x + a*y
void launch_xpay(double *z, const double *x, double a, const double *y, long long n,
                 cudaStream_t st);
// x *= 1 / (*s)
void launch_scale_inv_dev(double *x, const double *s, long long n, cudaStream_t st);
// x *= a
void launch_scale(double *x, double a, long long n, cudaStream_t st);
// xcor = sum_k yg[k] * V[k] (sequential axpy order)
// xcor = sum_k yg[k] V_k (onto xcor when accumulate)
void launch_combine(double *xcor, double *const *V, const double *yg, int kdim, long long n,
                    cudaStream_t st, int accumulate = 0);
// V_0 = yg[0] V_0 + sum_{k=1..kdim} yg[k] V_k (GMRES restart direction)
void launch_restart_v0(double *const *V, const double *yg, int kdim, long long n,
                       cudaStream_t st);
void launch_fill(double *x, double v, long long n, cudaStream_t st);

// GMRES scalar kernels (single thread); S layout and ops in krylov_kernels.cu
enum { GM_START = 0, GM_AFTER_GS = 1, GM_QR = 3, GM_QRSOL = 4, GM_REORTH_DONE = 5,
       GM_RESTART = 6, GM_RESTART_INIT = 7 };
enum { SCI_RNORM = 0, SCI_ROT, SCI_RHO, SCI_VKNORM2, SCI_NEWNORM2, SCI_FLAG, SCI_NN2, SCI_NP,
       SCI_GATE, SCI_COEF, SCI_HLL, SCI_BETA, SCI_QRFAIL, SCI_COUNT };
inline long long gs_size(int lmax) { return (long long)(lmax + 1) * lmax + 2 * lmax + lmax + 1 + SCI_COUNT; }
inline long long gs_sc_offset(int lmax) { return (long long)(lmax + 1) * lmax + 2 * lmax + lmax + 1; }
inline long long gs_yg_offset(int lmax) { return (long long)(lmax + 1) * lmax + 2 * lmax; }
void launch_gmres_scalar(int op, double *S, int l, int lmax, cudaStream_t st);
void launch_reorth_decide(double *S, int i, int l, int lmax, cudaStream_t st);
void launch_axpy_gated(double *y, const double *x, const double *coef, const double *gate,
                       long long n, cudaStream_t st);

// ParFlow layout (ghost frame 1) <-> dense interior
void launch_unpad(const double *pad, double *dense, int nx, int ny, int nz, cudaStream_t st);
void launch_pad(const double *dense, double *pad, int nx, int ny, int nz, cudaStream_t st);
// dense (nx, ny, nz) -> a frame of g ghost layers (ghosts 0)
void launch_pad_ghost(const double *dense, double *pad, int nx, int ny, int nz, int g,
                      cudaStream_t st);

// ---- discrete adjoint (adjoint.cu) ------------------------------------------
template <typename TJ>
void launch_matvec7_t(int nx, int ny, int nz, JacIn<TJ> J, const double *x, double *y,
                      cudaStream_t st);
void launch_adj_rhs(const DevProblem &P, const double *p, const double *sat, const double *dsat,
                    const double *lam_next, double *rhs, cudaStream_t st);
void launch_gather(int n, const long long *idx, const double *src, double *dst, cudaStream_t st);
void launch_adj_obs(int nobs, const long long *cells, const double *obs, const double *p,
                    double *rhs, cudaStream_t st);
void launch_adj_grad(const DevProblem &P, const double *p, const double *p_prev,
                     const double *lam, const double *kr, double dt, double *g_lnk, double *g_a,
                     double *g_n, cudaStream_t st);

// sets the message pfgpu_last_error returns on this thread
void record_error(const char *msg);


}  // namespace pfgpu
