// Control kernels of the graph-captured Newton-Krylov solve (nk_control.h).
//
// Each kernel is one thread on device-resident scalars.  They restate the
// host-driven solver's decisions in the same order and with the same
// arithmetic: KINSol's loop and stop test (pfsimulator/kinsol/kinsol.c:690-910,
// 1507-1589), the line search (kinsol.c:1228-1420), the forcing term
// (kinsol.c:1054-1090) and SPGMR's stop test, restarts and exits
// (pfsimulator/kinsol/spgmr.c:168-450).  This file is compiled with
// -fmad=false: no multiply-add is contracted, so every value equals the
// host's IEEE double result.
//
// Every loop of the graph ends: the Newton loop at the iteration limit (and a
// hard guard), the restart loop at Solver.Linear.MaxRestarts, the two
// line-search loops after at most 1000 trials each (error word set).
#include <cfloat>

#include "nk_control.h"
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

namespace {
constexpr double LS_ALPHA = 0.0001, LS_BETA = 0.9;  // KINLineSearch's alpha and beta
constexpr int LS_MAX_ITERS = 1000;
constexpr int NEWTON_GUARD = 100000;

__device__ __forceinline__ void setc(cudaGraphConditionalHandle h, bool v) {
  cudaGraphSetConditional(h, v ? 1u : 0u);
}
// KINStop's scaled step length (kinsol.c:1540-1541): the step is formed in
// vtemp1, which KINScSteplength (kinsol.c:1490-1498) then overwrites with
// 1/uscale + |unew| before dividing the step by it, so every component is
// (1 + |unew|) / (1 + |unew|) and the length is 1
__device__ __forceinline__ double kinstop_steplength() { return 1.0; }
// the trial step's norms (launch_step_norms)
__device__ __forceinline__ void take_trial(NkState *S, const double *dsc) {
  S->fevals++;
  S->fnormp = sqrt(dsc[D_F2]);
  S->f1normp = 0.5 * S->fnormp * S->fnormp;
  S->fmax = dsc[D_FMAX];
}
}  // namespace

// KINSolInit's maximum Newton step and KINInitialStop (kinsol.c:540-545, 726-731)
__global__ void k_nk_init(NkState *S, const double *dsc, NkConds c) {
  pdl_enter();
  S->nonlin_iters = S->lin_iters = S->pc_setups = S->pc_solves = 0;
  S->lin_conv_fails = S->beta_cond_fails = S->backtracks = S->kinsol_status = 0;
  S->err = 0;
  S->early = 0;
  for (int b = 0; b < NKB_COUNT; b++) S->execs[b] = 0;
  S->execs[NKB_TOP] = 1;
  S->fevals = 1;
  double mx = 1000.0 * sqrt(dsc[D_U2]);
  if (mx < 1.0) mx = 1.0;
  S->mxnewtstep = mx;
  if (dsc[D_FMAX] <= 0.01 * S->k.fnormtol) {
    // KINSol returns before loading its optional outputs: counters stay zero
    S->fevals = 0;
    S->kinsol_status = 2;
    S->fnorm = sqrt(dsc[D_F2]);
    S->early = 1;
    S->ret = 2;
    setc(c.newton, false);
    return;
  }
  S->fnorm = sqrt(dsc[D_F2]);
  S->f1norm = 0.5 * S->fnorm * S->fnorm;
  S->ret = 0;
  S->ncscmx = 0;
  S->eta = S->k.eta0;
  S->cont = 1;
  setc(c.newton, true);
}

// top of a Newton iteration: the linear tolerance and SPGMR's start
// (right-hand side -f with the norm of the last residual, x0 = 0)
__global__ void k_nk_iter(NkState *S, NkConds c) {
  pdl_enter();
  S->execs[NKB_NEWTON]++;
  S->nonlin_iters++;
  S->pc_setups++;
  if (S->nonlin_iters > NEWTON_GUARD) S->err = 1;
  double eps = (S->eta + DBL_EPSILON) * S->fnorm;
  if (eps < S->k.epsmin) eps = S->k.epsmin;
  S->eps = eps;
  S->r_norm = S->fnorm;
  S->beta = S->r_norm;
  S->delta = eps;
  S->ntries = 0;
  S->converged = 0;
  S->krydim = 0;
  S->rho = 0.0;
  S->zero_x = 0;
  S->cont = 0;
  S->do_copy = 0;
  if (S->r_norm <= S->delta || S->err) {
    S->gm_status = 0;  // x = 0
    S->zero_x = 1;
    setc(c.restart, false);
  } else {
    S->gm_status = 2;
    setc(c.restart, true);
  }
  setc(c.post, false);
}

// start of a GMRES cycle: only iteration 0 is armed
__global__ void k_nk_cycle_begin(NkState *S, NkConds c) {
  pdl_enter();
  S->execs[NKB_CYCLE]++;
  S->accumulate = S->ntries > 0 ? 1 : 0;
  for (int l = 1; l < S->k.lmax; l++) setc(c.iter[l], false);
}

// end of GMRES iteration l: the residual estimate against delta
__global__ void k_nk_gm_iter(NkState *S, const double *sc, int l, NkConds c) {
  pdl_enter();
  S->execs[NKB_GM0 + l]++;
  S->lin_iters++;
  S->pc_solves++;
  if (S->k.use_dq) S->fevals++;
  S->krydim = l + 1;
  const double rho = sc[SCI_RHO];
  S->rho = rho;
  if (rho <= S->delta)
    S->converged = 1;
  else if (l + 1 < S->k.lmax)
    setc(c.iter[l + 1], true);
}

// end of a GMRES cycle: QR failure, convergence, the restart limit, or a restart
__global__ void k_nk_cycle_end(NkState *S, const double *sc, NkConds c) {
  pdl_enter();
  bool restart = false;
  if (sc[SCI_QRFAIL] != 0.0) {
    S->gm_status = 6;
    S->zero_x = 1;
  } else if (S->converged) {
    S->gm_status = 0;  // x = M^{-1} V y
  } else if (S->ntries == S->k.max_restarts) {
    if (S->rho < S->beta) {
      S->gm_status = 1;
    } else {
      S->gm_status = 2;
      S->zero_x = 1;
    }
  } else {
    S->ntries++;
    restart = true;
  }
  setc(c.do_restart, restart);
  setc(c.restart, restart);
}

// executions of a body without a control kernel of its own (and the
// preconditioner solves it made)
__global__ void k_nk_count(NkState *S, int body, int pc_solves) {
  pdl_enter();
  S->execs[body]++;
  S->pc_solves += pc_solves;
}

// after SPGMR: its solution is M^{-1} V y unless x = 0; a failed linear
// solve ends KINSol with 8
__global__ void k_nk_after_gmres(NkState *S, NkConds c) {
  pdl_enter();
  const int st = S->gm_status;
  setc(c.post, !S->zero_x && (st == 0 || st == 1));
  if (st != 0 && st != 1) {
    S->lin_conv_fails++;
    S->ret = 8;
    S->cont = 0;
    setc(c.ok, false);
  } else if (S->err) {
    S->cont = 0;
    setc(c.ok, false);
  } else {
    setc(c.ok, true);
  }
}

// sJpnorm, sfdotJp (kinspgmr.c:384-398) and the line search's first steps
__global__ void k_nk_ls_init(NkState *S, const double *dsc, NkConds c) {
  pdl_enter();
  S->execs[NKB_OK]++;
  if (S->k.use_dq) S->fevals++;
  S->sJpnorm = sqrt(dsc[D_JP2]);
  S->sfdotJp = dsc[D_FJP];
  S->globalret = 0;
  S->maxStepTaken = 0;
  S->refined = 0;
  S->pnorm = sqrt(dsc[D_P2]);
  S->ratio = 1.0;
  if (S->pnorm > S->mxnewtstep) {
    S->ratio = S->mxnewtstep / S->pnorm;
    S->scaled = 1;
  } else {
    S->scaled = 0;
  }
  setc(c.scale, S->scaled != 0);
}

__global__ void k_nk_ls_setup(NkState *S, const double *dsc, NkConds c) {
  pdl_enter();
  if (S->scaled) S->pnorm = S->mxnewtstep;
  S->slpi = S->sfdotJp * S->ratio;
  S->rlength = dsc[D_PLEN];
  S->rlmin = S->k.scsteptol / S->rlength;
  S->rl = 1.0;
  S->rlprev = 0.0;
  S->nfesav = S->fevals;
  S->lam = S->rl;
  S->ls_it = 0;
  S->ls_phase = 0;
  setc(c.ls1, true);
}

// after each trial of the backtracking loop
__global__ void k_nk_ls1(NkState *S, const double *dsc, NkConds c) {
  pdl_enter();
  S->execs[NKB_LS1]++;
  take_trial(S, dsc);
  if (S->k.inexact) {  // KINInexactNewton takes the full step (kinsol.c:1152-1208)
    setc(c.ls1, false);
    return;
  }
  if (S->ls_phase == 1) {  // the step was too small: u itself was re-evaluated
    S->backtracks = S->fevals - S->nfesav - 1;
    S->globalret = 1;
    setc(c.ls1, false);
    return;
  }
  S->alpha_cond = S->f1norm + LS_ALPHA * S->slpi * S->rl;
  if (S->f1normp <= S->alpha_cond) {
    setc(c.ls1, false);
    return;
  }
  if (S->rl < S->rlmin) {
    S->ls_phase = 1;
    S->lam = 0.0;
    setc(c.ls1, true);
    return;
  }
  double rltmp = -S->slpi / (2.0 * (S->f1normp - S->f1norm - S->slpi));
  if (rltmp > 0.5 * S->rl) rltmp = 0.5 * S->rl;
  S->rlprev = S->rl;
  const double pt1trl = 0.1 * S->rl;
  S->rl = (pt1trl > rltmp) ? pt1trl : rltmp;
  S->lam = S->rl;
  if (++S->ls_it > LS_MAX_ITERS) {
    S->err = 1;
    setc(c.ls1, false);
    return;
  }
  setc(c.ls1, true);
}

// the beta condition and the start of the refinement loop
__global__ void k_nk_ls2_init(NkState *S, NkConds c) {
  pdl_enter();
  bool run = false;
  if (S->globalret != 1 && !S->err && !S->k.inexact) {
    S->beta_cond = S->f1norm + LS_BETA * S->slpi * S->rl;
    if (S->f1normp < S->beta_cond) {
      // (rl == 1 && pnorm < stepl) never holds without constraints
      if (S->rl < 1.0 || ((S->rl > 1.0) && (S->f1normp > S->alpha_cond))) {
        S->rllo = (S->rl < S->rlprev) ? S->rl : S->rlprev;
        S->rldiff = fabs(S->rlprev - S->rl);
        S->refined = 1;
        S->ls_it = 1;
        S->rlincr = 0.5 * S->rldiff;
        S->rl = S->rllo + S->rlincr;
        S->lam = S->rl;
        run = true;
      }
    }
  }
  setc(c.ls2, run);
}

// after each trial of the refinement loop
__global__ void k_nk_ls2(NkState *S, const double *dsc, NkConds c) {
  pdl_enter();
  S->execs[NKB_LS2]++;
  take_trial(S, dsc);
  S->alpha_cond = S->f1norm + LS_ALPHA * S->slpi * S->rl;
  S->beta_cond = S->f1norm + LS_BETA * S->slpi * S->rl;
  if (S->f1normp > S->alpha_cond) {
    S->rldiff = S->rlincr;
  } else if (S->f1normp < S->beta_cond) {
    S->rllo = S->rl;
    S->rldiff = S->rldiff - S->rlincr;
  }
  if (S->f1normp > S->alpha_cond || ((S->f1normp < S->beta_cond) && (S->rldiff > S->rlmin))) {
    if (++S->ls_it > LS_MAX_ITERS) {
      S->err = 1;
      setc(c.ls2, false);
      return;
    }
    S->rlincr = 0.5 * S->rldiff;
    S->rl = S->rllo + S->rlincr;
    S->lam = S->rl;
    setc(c.ls2, true);
    return;
  }
  setc(c.ls2, false);
}

// the refinement ended below the beta condition: step rllo instead
__global__ void k_nk_ls3_decide(NkState *S, NkConds c) {
  pdl_enter();
  const bool run = S->refined && !S->err && S->f1normp < S->beta_cond;
  if (run) S->lam = S->rllo;
  setc(c.ls3, run);
}
__global__ void k_nk_ls3(NkState *S, const double *dsc) {
  pdl_enter();
  S->execs[NKB_LS3]++;
  take_trial(S, dsc);
  S->beta_cond_fails++;
}

// end of the line search, the forcing term and KINStop
__global__ void k_nk_newton_end(NkState *S) {
  pdl_enter();
  S->do_copy = 0;
  S->cont = 0;
  if (S->err) return;
  if (S->globalret != 1) {
    S->backtracks = S->fevals - S->nfesav - 1;
    S->sfdotJp = S->sfdotJp * S->rl * S->ratio;
    S->sJpnorm = S->sJpnorm * S->rl * S->ratio;
    if (S->rl * S->pnorm > 0.99 * S->mxnewtstep) S->maxStepTaken = 1;
  }
  if (S->beta_cond_fails > 10) {
    S->ret = 7;
    return;
  }
  const int etaflag = S->k.etaflag;
  if (etaflag != 0) {
    const double eta_max = 0.9, eta_min = 0.0001;
    double eta_safe = 0.5, eta = S->eta;
    const double fnorm = S->fnorm, fnormp = S->fnormp;
    if (etaflag == 1) {
      const double linmodel_norm =
          sqrt(fnorm * fnorm + 2.0 * S->sfdotJp + S->sJpnorm * S->sJpnorm);
      eta_safe = pow(eta, S->k.ealpha);
      eta = fabs(fnormp - linmodel_norm) / fnorm;
    }
    if (etaflag == 2) {
      eta_safe = S->k.egamma * pow(eta, S->k.ealpha);
      eta = S->k.egamma * pow(fnormp / fnorm, S->k.ealpha);
    }
    if (eta_safe < 0.1) eta_safe = 0.0;
    if (eta < eta_safe) eta = eta_safe;
    if (eta < eta_min) eta = eta_min;
    if (eta > eta_max) eta = eta_max;
    S->eta = eta;
  }
  S->fnorm = S->fnormp;
  int sret = 0;
  if (S->globalret == 1)
    sret = 3;
  else if (S->fmax <= S->k.fnormtol)
    sret = 1;
  else if (kinstop_steplength() <= S->k.scsteptol)
    sret = 2;
  else if (S->nonlin_iters >= S->k.mxiter)
    sret = 4;
  else {
    S->ncscmx = S->maxStepTaken ? S->ncscmx + 1 : 0;
    if (S->ncscmx == 5) sret = 5;
  }
  S->do_copy = 1;  // u <- unew
  S->f1norm = S->f1normp;
  if (sret != 0)
    S->ret = sret;
  else
    S->cont = 1;
}

__global__ void k_nk_tail(NkState *S, NkConds c) {
  pdl_enter();
  setc(c.newton, S->cont && !S->err);
}

__global__ void k_nk_final(NkState *S) {
  pdl_enter();
  if (!S->early) S->kinsol_status = S->ret;
}

void launch_nk_init(NkState *S, const double *dsc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_init, dim3(1), dim3(1), st, S, dsc, c);
}
void launch_nk_iter(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_iter, dim3(1), dim3(1), st, S, c);
}
void launch_nk_cycle_begin(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_cycle_begin, dim3(1), dim3(1), st, S, c);
}
void launch_nk_gm_iter(NkState *S, const double *sc, int l, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_gm_iter, dim3(1), dim3(1), st, S, sc, l, c);
}
void launch_nk_cycle_end(NkState *S, const double *sc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_cycle_end, dim3(1), dim3(1), st, S, sc, c);
}
void launch_nk_count(NkState *S, int body, int pc_solves, cudaStream_t st) {
  launch_pdl(k_nk_count, dim3(1), dim3(1), st, S, body, pc_solves);
}
void launch_nk_after_gmres(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_after_gmres, dim3(1), dim3(1), st, S, c);
}
void launch_nk_ls_init(NkState *S, const double *dsc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls_init, dim3(1), dim3(1), st, S, dsc, c);
}
void launch_nk_ls_setup(NkState *S, const double *dsc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls_setup, dim3(1), dim3(1), st, S, dsc, c);
}
void launch_nk_ls1(NkState *S, const double *dsc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls1, dim3(1), dim3(1), st, S, dsc, c);
}
void launch_nk_ls2_init(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls2_init, dim3(1), dim3(1), st, S, c);
}
void launch_nk_ls2(NkState *S, const double *dsc, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls2, dim3(1), dim3(1), st, S, dsc, c);
}
void launch_nk_ls3_decide(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_ls3_decide, dim3(1), dim3(1), st, S, c);
}
void launch_nk_ls3(NkState *S, const double *dsc, cudaStream_t st) {
  launch_pdl(k_nk_ls3, dim3(1), dim3(1), st, S, dsc);
}
void launch_nk_newton_end(NkState *S, cudaStream_t st) {
  launch_pdl(k_nk_newton_end, dim3(1), dim3(1), st, S);
}
void launch_nk_tail(NkState *S, NkConds c, cudaStream_t st) {
  launch_pdl(k_nk_tail, dim3(1), dim3(1), st, S, c);
}
void launch_nk_final(NkState *S, cudaStream_t st) {
  launch_pdl(k_nk_final, dim3(1), dim3(1), st, S);
}

}  // namespace pfgpu
