// Device-side control of one Newton-Krylov solve (KINSOL with line search,
// pfsimulator/kinsol/kinsol.c:363-910, 1054-1589, and SPGMR,
// pfsimulator/kinsol/spgmr.c:168-450) for the solve captured as one CUDA
// graph: every decision the host makes between launches in the host-driven
// solver (GMRES stop test and restarts, line-search backtracking and
// refinement, forcing term, KINStop) is made by a single-thread kernel on
// device-resident scalars, which steers the graph's conditional nodes.
//
// The control kernels are compiled without floating-point contraction, so
// every scalar comes out as the host's plain IEEE double arithmetic gives it:
// the graph solve and the host-driven solve take the same steps bit for bit.
#pragma once

#include <cuda_runtime.h>

namespace pfgpu {

// device scalar slots of the solver (results of the fused reductions)
enum {
  D_F2 = 0,  // <f, f>
  D_FMAX,    // max |f|
  D_FREE,    // unused
  D_P2,      // <p, p>
  D_PLEN,    // max |p| / (1 + |u|)
  D_JP2,     // <Jp, Jp>
  D_FJP,     // <f, Jp>
  D_U2,      // <u, u>
  D_COUNT,
  D_DQ = 40  // five slots of the difference-quotient product (launch_dq_prepare)
};

constexpr int NK_MAX_KRYLOV = 64;  // largest Krylov dimension (KrylovDimension)
constexpr int NK_MAX_L = NK_MAX_KRYLOV + 2;

// graph bodies whose executions are counted (launches = sum over bodies of
// kernels per body x executions)
enum {
  NKB_TOP = 0,
  NKB_NEWTON,
  NKB_CYCLE,
  NKB_RESTART,
  NKB_POST,
  NKB_OK,
  NKB_SCALE,
  NKB_LS1,
  NKB_LS2,
  NKB_LS3,
  NKB_GM0,  // + l: GMRES iteration l
  NKB_COUNT = NKB_GM0 + NK_MAX_L
};

struct NkConst {
  double fnormtol, scsteptol, epsmin, ealpha, egamma, eta0, bsign;
  int etaflag, mxiter, lmax, max_restarts, use_dq;
  int inexact;  // KINInexactNewton: the first trial step is taken, no backtracking
};

struct NkState {
  NkConst k;
  // Newton
  double fnorm, f1norm, eta, eps, mxnewtstep;
  // line search
  double sJpnorm, sfdotJp, pnorm, ratio, slpi, rlength, rlmin, rl, rlprev, rllo, rldiff, rlincr;
  double alpha_cond, beta_cond, fnormp, f1normp, fmax, lam;
  int ncscmx, ret, globalret, maxStepTaken, nfesav, ls_it, ls_phase, scaled, refined, do_copy,
      cont;
  // GMRES
  double r_norm, beta, delta, rho;
  int krydim, converged, ntries, gm_status, zero_x, accumulate;
  // counters (pfgpu_stats)
  int nonlin_iters, lin_iters, fevals, pc_setups, pc_solves, lin_conv_fails, beta_cond_fails,
      backtracks, kinsol_status;
  int early;  // KINSol returned at its initial stop test
  int err;    // 1: a loop bound was hit (the solve stops; the host reports it)
  unsigned long long execs[NKB_COUNT];
};

struct NkConds {
  cudaGraphConditionalHandle newton, ok, scale, ls1, ls2, ls3, restart, do_restart, post;
  cudaGraphConditionalHandle iter[NK_MAX_L];  // iter[l], l >= 1: GMRES iteration l runs
};

// control points, each one single-thread launch on stream st
void launch_nk_init(NkState *S, const double *dsc, NkConds c, cudaStream_t st);
void launch_nk_iter(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_cycle_begin(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_gm_iter(NkState *S, const double *sc, int l, NkConds c, cudaStream_t st);
void launch_nk_cycle_end(NkState *S, const double *sc, NkConds c, cudaStream_t st);
void launch_nk_count(NkState *S, int body, int pc_solves, cudaStream_t st);
void launch_nk_after_gmres(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_ls_init(NkState *S, const double *dsc, NkConds c, cudaStream_t st);
void launch_nk_ls_setup(NkState *S, const double *dsc, NkConds c, cudaStream_t st);
void launch_nk_ls1(NkState *S, const double *dsc, NkConds c, cudaStream_t st);
void launch_nk_ls2_init(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_ls2(NkState *S, const double *dsc, NkConds c, cudaStream_t st);
void launch_nk_ls3_decide(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_ls3(NkState *S, const double *dsc, cudaStream_t st);
void launch_nk_newton_end(NkState *S, cudaStream_t st);
void launch_nk_tail(NkState *S, NkConds c, cudaStream_t st);
void launch_nk_final(NkState *S, cudaStream_t st);

// vector steps of the graph solve whose scalars live on the device
// (krylov_kernels.cu)
void launch_v0_init(double *v0, const double *src, const NkState *S, const double *sc,
                    long long n, cudaStream_t st);
void launch_gmres_scalar_dev(int op, double *S, const int *l, int lmax, cudaStream_t st);
void launch_combine_dev(double *xcor, double *const *V, int nv, const double *yg, const int *kdim,
                        const int *accumulate, long long n, cudaStream_t st);
void launch_restart_v0_dev(double *const *V, int nv, const double *yg, const int *kdim,
                           long long n, cudaStream_t st);
void launch_scale_inv_dev_unless(double *x, const double *s, const int *skip, long long n,
                                 cudaStream_t st);
void launch_fill_if(double *x, double v, const int *flag, long long n, cudaStream_t st);
void launch_xpay_lam(double *z, const double *x, const double *lam, const double *y, long long n,
                     cudaStream_t st);
void launch_scale_by(double *x, const double *a, long long n, cudaStream_t st);
void launch_copy_if(double *dst, const double *src, const int *flag, long long n, cudaStream_t st);

}  // namespace pfgpu
