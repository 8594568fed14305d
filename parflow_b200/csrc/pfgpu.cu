// libpfgpu: handle, C ABI entry points and the device-resident KINSOL /
// SPGMR / MGSemi driver.
//
// Control flow mirrors the embedded KINSOL of ParFlow (pfsimulator/kinsol/
// kinsol.c:690-910, kinspgmr.c:344-440, spgmr.c:168-450, iterativ.c:30-286)
// with every vector and every GMRES scalar in device memory.  By default a
// whole Newton solve is one CUDA graph launch: control kernels on the device
// take the decisions and steer the graph's conditional nodes, and the host
// reads the solve's counters once at its end.  The host-driven form (one
// small read per GMRES iteration and per line-search evaluation) remains for
// phase timing and as the reference the graph solve is tested against.  The
// multigrid V-cycle is a fixed kernel sequence and is replayed from a CUDA
// graph.
#include <cuda_runtime.h>

#include <cfloat>
#include <chrono>
#include <cmath>
#include <algorithm>
#include <array>
#include <atomic>
#include <climits>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/pfgpu.h"
#include "nk_control.h"
#include "pdl.cuh"
#include "pfgpu_kernels.h"

using namespace pfgpu;

static thread_local char g_err[512] = "";

static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// lets other translation units of the library report through pfgpu_last_error
void pfgpu::record_error(const char *msg) { set_err("%s", msg); }

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return PFGPU_ERR_CUDA;                                                            \
    }                                                                                   \
  } while (0)

namespace {

struct Handle;

template <typename T>
struct MG {
  std::vector<MGLevel<T>> L;
  MGLevel<T> *Ldev = nullptr;  // device copy of the level table (tail kernels)
  int tail = 0;                // first level run by the single-block tail kernels
  int mid = 0;                 // first level run by the cluster kernel (== tail: none)
  int mid_cs = 0;              // blocks in that kernel's cluster
  int grid_blocks = 0;         // levels mid .. tail-1 on cooperative grid kernels instead
  unsigned *gbar = nullptr;    // their barrier: counter, generation
  size_t tail_smem = 0;        // shared-memory bytes of the V-cycle tail (0: global)
  std::vector<char> waved;     // level smoothed by the wavefront kernel
  std::vector<WaveLevel> wave; // its control words
  bool h16 = false;            // scaled FP16 operator storage (float levels only)
  int *hflag = nullptr;        // some scaled diagonal is not +1 (set by the setup)
  int flip = 1;                // alternate the block order of consecutive launches
  int flip_out = 0;            // block order for the launch after a V-cycle
  T *wtmp = nullptr;           // Jacobi temp (finest size)
  std::vector<char> fused;     // level smoothed by the fused red/black/red kernel
  std::vector<RbrMaps> maps;   // its tensor maps (input iterate = x)
  int *kerr = nullptr;         // pipeline-wait error word of the fused kernel
  // buffer holding the smoothed result of level l (post-smoother output)
  T *res(int l) const { return (l < (int)fused.size() && fused[l]) ? L[l].x2 : L[l].x; }
};

// Tuning (read once per handle from the environment; all variants compute
// the same V-cycle):
//   PFGPU_TAIL_CELLS  levels at or below this many cells may run inside the
//                     single-block tail kernels, as far as the tail fits in
//                     shared memory (default 1024)
//   PFGPU_TAIL_SMEM   0 runs the V-cycle tail from global memory
//   PFGPU_MID_CELLS   grid levels at or below this many cells run, with the
//                     tail, inside one thread-block-cluster kernel (default 0:
//                     none; on B200 each of its phases waits about as long on
//                     L2 as a grid launch does, so it is slower overall)
//   PFGPU_MID_CLUSTER most blocks in that cluster (default 16, as many as the
//                     device can co-schedule)
//   PFGPU_GRID_CELLS  grid levels at or below this many cells run, per V-cycle
//                     leg, inside one cooperative kernel over the whole GPU
//                     (grid barriers between phases instead of one launch
//                     per phase; default 0: off, slower on B200)
//   PFGPU_GRID_PER_SM resident blocks per SM of those kernels (default 1)
//   PFGPU_FLIP        0 runs every V-cycle launch in forward block order
//   PFGPU_SPLIT       0 keeps x and b of the grid levels in the natural
//                     (interleaved-colour) layout; the TMA-fused and wavefront
//                     smoothers need it
//   PFGPU_PHASE_TIMES 1 times the solver phases with CUDA events and prints
//                     the sums to stderr when the handle is destroyed
//   PFGPU_WAVE_CELLS  grid levels with at least this many cells use the
//                     wavefront red/black/red kernel (red/black Gauss-Seidel
//                     smoother only; default: no level, the per-colour sweeps
//                     are faster on B200)
//   PFGPU_WAVE_CTAS   resident blocks per SM of the wavefront kernel (default:
//                     as many as fit)
//   PFGPU_WAVE_LAG    planes by which each wavefront sweep trails the previous
//   PFGPU_WAVE_CHUNK  cells of one colour per wavefront work item
//   PFGPU_RBR_FUSED_CELLS  grid levels with at least this many cells (and a
//                     row pitch TMA can address) use the TMA-pipelined fused
//                     red/black/red smoother; the rest one kernel per colour
//                     sweep (default: no level; the fused kernel is slower)
static long long env_ll(const char *name, long long dflt) {
  const char *v = getenv(name);
  return v && *v ? atoll(v) : dflt;
}

}  // namespace

struct pfgpu_handle {
  int device = 0;
  cudaStream_t st = nullptr;
  pfgpu_desc d;
  DevProblem P;
  int nx, ny, nz;
  long long N, NP;  // interior cells, ParFlow-layout cells
  bool mixed = false;  // FP32 multigrid and Jacobian storage
  bool h16 = false;    // ... with the scaled FP16 multigrid operator
  // fields
  double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  double *alpha = nullptr, *vgn = nullptr, *sres = nullptr, *ssat = nullptr, *zmult = nullptr;
  // surface: 7 column arrays of ny*nx (TFG g sin / g cos of x and y slopes,
  // overland slopes x / y, Manning's n) in one allocation
  double *surf = nullptr;
  double *fb[3] = {nullptr, nullptr, nullptr};  // flow barriers x, y, z (or none)
  double *bcv[6] = {nullptr};
  // state and work vectors (dense interior layout)
  double *u = nullptr;      // current iterate / handle pressure state
  double *unew = nullptr, *fval = nullptr, *pp = nullptr, *bb = nullptr;
  double *p_old = nullptr, *s_old = nullptr;
  double *kr = nullptr, *dkr = nullptr, *sat = nullptr, *dsat = nullptr;
  const double *vg_for = nullptr;  // iterate the cached kr/dkr/S/dS belong to
  double *zface = nullptr;
  double *xcor = nullptr, *vtemp = nullptr;
  std::vector<double *> V;
  // Mixed forms keep the preconditioned basis Z[l] = M^{-1} V[l] and form the
  // correction as Z y: one V-cycle less per linear solve than M^{-1} (V y).
  // Equal in exact arithmetic; the reduced-precision V-cycle is not exactly
  // linear, so the two differ by its rounding.  The FP64 form follows SPGMR
  // (M^{-1} (V y), spgmr.c:364-388) as the reference does.
  bool zbasis = false;
  std::vector<double *> Z;
  double *gs = nullptr;   // GMRES scalars
  double *dsc = nullptr;  // named device scalars
  double *hsc = nullptr;  // pinned host mirror of dsc / rho
  ReduceBuf rb{};
  double *stage = nullptr;  // ParFlow-layout staging (device)
  double *stage2 = nullptr;
  // Jacobian
  JacOut<double> Jd{};
  JacOut<float> Jf{};
  // multigrid
  MG<double> mgd;
  MG<float> mgf;
  int nlev = 0;
  double *pc_in = nullptr, *pc_out = nullptr;  // FP64 level-0 staging when mixed
  cudaGraphExec_t vgraph = nullptr;
  long long graph_nodes = 0;
  bool pc_ready = false;
  long long launches = 0;
  int jac_valid = 0;
  // Solver.Nonlinear.UseJacobian (1: analytic J v; 0: KINSOL's difference
  // quotient with sqrt(DerivativeEpsilon)) and its two work vectors
  int use_jacobian = 1;
  int globalization = PFGPU_GLOBAL_LINE_SEARCH;  // Solver.Nonlinear.Globalization
  int pc_matrix = PFGPU_PCM_SYMMETRIC;  // Solver.Linear.Preconditioner.PCMatrixType
  int mg_max_iter = 1;                  // Solver.Linear.Preconditioner.MGSemi.MaxIter
  double sqrt_relfunc = 0.0;
  double *dq_w = nullptr, *dq_f = nullptr;
  double *krt = nullptr;  // relative-permeability lookup table (device)
  double *et = nullptr;   // evap_trans sink/source per cell (dense, device)
  // face velocities and overland fluxes (pfgpu_face_velocities): dense
  // vx, vy, vz, qx, qy in one allocation, and a staging buffer of the
  // largest ParFlow-layout face grid for host outputs
  double *vel = nullptr, *vstage = nullptr;
  int *kerr = nullptr;   // device error word of the pipelined kernels
  int *hkerr = nullptr;  // pinned host mirror
  // discrete adjoint: recorded trajectory p_0 .. p_len (dense, device) and
  // the dt of each recorded step; work vectors of the backward sweep
  double *hist = nullptr;
  int hist_cap = 0, hist_len = 0;
  bool recording = false, hist_overflow = false;
  std::vector<double> hist_dt;
  double *adj = nullptr;  // 8 vectors: lam, lam_next, rhs, r, dx, g_lnk, g_a, g_n
  bool adj_transpose = false;  // matvec applies J^T (adjoint solves)
  // optional per-phase device timing (PFGPU_PHASE_TIMES=1): events recorded
  // around each phase on the solver stream, summed after every Newton solve
  // and printed to stderr when the handle is destroyed
  // time-cycled boundary tables (pfgpu_set_bc_cycle) and the time step
  // selection of the native time loop (pfgpu_set_time_step, pfgpu_run)
  struct BcCycle {
    int nint = 0, repeat = -1, cycle_len = 0;
    std::vector<int> lengths, types;
    double *table = nullptr;  // device: nint face tables
    long long face_cells = 0;
    double base_unit = 1.0, start_time = 0.0;
  } cyc[6];
  int ts_type = 0;  // 0 constant, 1 growth (select_time_step.c:42-51)
  double ts_step = 0.0, ts_factor = 1.0, ts_min = 0.0, ts_max = 0.0;
  int max_failures = 3;
  bool ptime = false;
  std::vector<cudaEvent_t> pev;                  // event pool
  std::vector<std::array<int, 3>> pmark;        // (phase, start event, end event)
  double pacc[8] = {};
  long long pcnt[8] = {};
  // the Newton solve captured as one CUDA graph (device-side control)
  struct NkGraph {
    bool enabled = true;   // pfgpu_solve_graph / PFGPU_SOLVE_GRAPH
    bool failed = false;   // capture or instantiation failed: host-driven solves
    bool used_last = false;
    bool capturing = false;
    cudaGraphExec_t exec = nullptr;
    NkState *S = nullptr;   // device control state
    NkState *hS = nullptr;  // pinned host copy
    double *dt = nullptr, *hdt = nullptr;
    std::vector<cudaStream_t> cs;  // capture streams, one per nesting depth
    long long kernels[NKB_COUNT] = {};
    std::vector<std::array<long long, 3>> stack;  // (body, launches at entry, nested)
    std::vector<unsigned char> key;  // what the graph was captured for (nk_key)
    bool valid = false;
    // earlier graphs of the handle (a time cycle switches between a few
    // boundary tables): most recent last
    struct Kept {
      std::vector<unsigned char> key;
      cudaGraphExec_t exec;
      std::array<long long, NKB_COUNT> kernels;
    };
    std::vector<Kept> kept;
  } nk;
  unsigned long long uid = 0;  // never reused: names the handle in ensemble graphs
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
// Error word of the pipelined kernels: nonzero once a bounded pipeline wait
// expired (the results of that launch are then invalid).  Cleared when read.
static int check_kernel_error(pfgpu_handle *h) {
  CK(cudaMemcpyAsync(h->hkerr, h->kerr, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (*h->hkerr) {
    const int code = *h->hkerr;
    *h->hkerr = 0;
    CK(cudaMemsetAsync(h->kerr, 0, sizeof(int), h->st));
    set_err(code == 3 ? "a cooperative multigrid kernel gave up waiting at a grid barrier"
            : code == 2 ? "the wavefront smoother gave up waiting for a neighbouring plane"
                        : "a pipelined smoother kernel gave up waiting for its TMA copies");
    return PFGPU_ERR_CUDA;
  }
  return 0;
}

static bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
static int dalloc(T **p, long long n) {
  if (cudaMalloc((void **)p, (size_t)(n > 0 ? n : 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    set_err("cudaMalloc of %lld bytes failed", (long long)(n * sizeof(T)));
    return PFGPU_ERR_NOMEM;
  }
  return 0;
}

// ParFlow-layout input (host or device) -> dense device array
static int in_vec(pfgpu_handle *h, const double *src, double *dense) {
  if (h->vg_for == dense) h->vg_for = nullptr;
  if (is_device_ptr(src)) {
    launch_unpad(src, dense, h->nx, h->ny, h->nz, h->st);
  } else {
    CK(cudaMemcpyAsync(h->stage, src, h->NP * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_unpad(h->stage, dense, h->nx, h->ny, h->nz, h->st);
  }
  h->launches++;
  return 0;
}

static int out_vec(pfgpu_handle *h, const double *dense, double *dst) {
  if (is_device_ptr(dst)) {
    launch_pad(dense, dst, h->nx, h->ny, h->nz, h->st);
    h->launches++;
  } else {
    launch_pad(dense, h->stage, h->nx, h->ny, h->nz, h->st);
    h->launches++;
    CK(cudaMemcpyAsync(dst, h->stage, h->NP * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  return 0;
}

static int read_scalars(pfgpu_handle *h, int first, int count) {
  CK(cudaMemcpyAsync(h->hsc + first, h->dsc + first, count * sizeof(double),
                     cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// ---------------------------------------------------------------------------
// physics building blocks
// ---------------------------------------------------------------------------
// van Genuchten state at u (kr, dkr, S, dS), unless already cached for u
static void vg_state(pfgpu_handle *h, const double *u, bool reuse) {
  if (reuse && h->vg_for == u) return;
  launch_vg_all(h->P, u, h->kr, h->dkr, h->sat, h->dsat, h->st);
  h->launches++;
  h->vg_for = u;
}

// ---- phase timing (diagnostics) -------------------------------------------
enum { PH_FEVAL = 0, PH_PCSETUP, PH_PCAPPLY, PH_MATVEC, PH_NEWTON, PH_COUNT };
static const char *const kPhaseName[PH_COUNT] = {"residual (with VG state)",
                                                 "preconditioner setup (J + MG setup)",
                                                 "preconditioner apply (V-cycle)",
                                                 "Jacobian matvec", "Newton solve total"};
static int ph_event(pfgpu_handle *h) {
  const int i = (int)h->pmark.size() * 2 + 1;  // a fresh slot per mark
  while ((int)h->pev.size() <= i) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    h->pev.push_back(e);
  }
  return i;
}
static int ph_begin(pfgpu_handle *h) {
  if (!h->ptime) return -1;
  const int i = ph_event(h);
  if (i < 0) return -1;
  h->pmark.push_back({-1, i - 1, i});
  cudaEventRecord(h->pev[i - 1], h->st);
  return (int)h->pmark.size() - 1;
}
static void ph_end(pfgpu_handle *h, int mark, int phase) {
  if (!h->ptime || mark < 0) return;
  h->pmark[mark][0] = phase;
  cudaEventRecord(h->pev[h->pmark[mark][2]], h->st);
}
static void ph_collect(pfgpu_handle *h) {
  if (!h->ptime || h->pmark.empty()) return;
  cudaStreamSynchronize(h->st);
  for (auto &m : h->pmark) {
    float ms = 0.0f;
    if (m[0] >= 0 && cudaEventElapsedTime(&ms, h->pev[m[1]], h->pev[m[2]]) == cudaSuccess) {
      h->pacc[m[0]] += ms;
      h->pcnt[m[0]]++;
    }
  }
  h->pmark.clear();
}

static void feval(pfgpu_handle *h, const double *u, double dt, double *f) {
  const int m = ph_begin(h);
  vg_state(h, u, false);
  launch_residual(h->P, u, h->p_old, h->s_old, h->kr, h->sat, dt, f, h->st);
  h->launches++;
  ph_end(h, m, PH_FEVAL);
}

// the multigrid's finest operator as a full 7-array matrix (FullJacobian)
template <typename T>
static JacOut<T> level0_full(MG<T> &mg) {
  MGLevel<T> &L = mg.L[0];
  return JacOut<T>{L.a[0], L.lo[0], L.a[1], L.lo[1], L.a[2], L.lo[2], L.a[3]};
}

template <typename T>
static void assemble_T(pfgpu_handle *h, MG<T> &mg, JacOut<T> &Jh, const double *u, double dt,
                       bool want_J, bool want_M) {
  // Solver.Nonlinear.UseJacobian False: the preconditioner matrix without
  // the overland surface terms (PCOut::fd); J for a matvec keeps them
  const int fd = want_M && !h->use_jacobian;
  if (want_M && h->pc_matrix == PFGPU_PCM_FULL) {
    // FullJacobian: the Jacobian itself is the finest multigrid operator
    PCOut<T> M{};
    M.fd = fd;
    JacOut<T> L0 = level0_full(mg);
    launch_jacobian<T, T>(h->P, u, h->kr, h->dkr, h->sat, h->dsat, dt, L0, M, h->st);
    h->launches++;
    if (want_J && !fd) {
      T *const src[7] = {L0.c, L0.w, L0.e, L0.s, L0.n, L0.l, L0.u};
      T *const dst[7] = {Jh.c, Jh.w, Jh.e, Jh.s, Jh.n, Jh.l, Jh.u};
      for (int q = 0; q < 7; q++)
        cudaMemcpyAsync(dst[q], src[q], h->N * sizeof(T), cudaMemcpyDeviceToDevice, h->st);
      return;
    }
    if (!want_J) return;
    want_M = false;
  }
  PCOut<T> M{};
  if (want_M) M = {mg.L[0].a[0], mg.L[0].a[1], mg.L[0].a[2], mg.L[0].a[3], mg.L[0].wg, 0};
  JacOut<T> J{};
  if (want_J) J = Jh;
  if (fd && want_M && want_J) {
    // J with the surface terms, then the preconditioner without them
    PCOut<T> none{};
    launch_jacobian<T, T>(h->P, u, h->kr, h->dkr, h->sat, h->dsat, dt, J, none, h->st);
    h->launches++;
    J = JacOut<T>{};
  }
  M.fd = want_M ? fd : 0;
  launch_jacobian<T, T>(h->P, u, h->kr, h->dkr, h->sat, h->dsat, dt, J, M, h->st);
  h->launches++;
}

// assemble J (full) and the preconditioner matrix at u (one pass); the VG
// state of the last residual evaluation is reused when it was taken at u
static void assemble(pfgpu_handle *h, const double *u, double dt, bool want_J, bool want_M,
                     bool reuse_vg = false) {
  vg_state(h, u, reuse_vg);
  if (h->mixed)
    assemble_T<float>(h, h->mgf, h->Jf, u, dt, want_J, want_M);
  else
    assemble_T<double>(h, h->mgd, h->Jd, u, dt, want_J, want_M);
}

static void matvec_impl(pfgpu_handle *h, const double *x, double *y) {
  if (h->adj_transpose) {
    if (h->mixed) {
      JacIn<float> J{h->Jf.c, h->Jf.w, h->Jf.e, h->Jf.s, h->Jf.n, h->Jf.l, h->Jf.u};
      launch_matvec7_t<float>(h->nx, h->ny, h->nz, J, x, y, h->st);
    } else {
      JacIn<double> J{h->Jd.c, h->Jd.w, h->Jd.e, h->Jd.s, h->Jd.n, h->Jd.l, h->Jd.u};
      launch_matvec7_t<double>(h->nx, h->ny, h->nz, J, x, y, h->st);
    }
    h->launches++;
    return;
  }
  if (h->mixed) {
    JacIn<float> J{h->Jf.c, h->Jf.w, h->Jf.e, h->Jf.s, h->Jf.n, h->Jf.l, h->Jf.u};
    launch_matvec7<float>(h->nx, h->ny, h->nz, J, x, y, h->st, h->P.tile[2]);
  } else {
    JacIn<double> J{h->Jd.c, h->Jd.w, h->Jd.e, h->Jd.s, h->Jd.n, h->Jd.l, h->Jd.u};
    launch_matvec7<double>(h->nx, h->ny, h->nz, J, x, y, h->st, h->P.tile[2]);
  }
  h->launches++;
}
static void matvec(pfgpu_handle *h, const double *x, double *y) {
  const int m = ph_begin(h);
  matvec_impl(h, x, y);
  ph_end(h, m, PH_MATVEC);
}

template <typename T>
static long long mg_setup_T(MG<T> &mg, cudaStream_t st) {
  long long k = 0;
  const int nl = (int)mg.L.size();
  // FullJacobian: every level from the generic setup (mg_full.cu)
  if (mg.L[0].lo[0]) return launch_mg_full_setup<T>(mg.L.data(), nl, st);
  if (mg.h16) cudaMemsetAsync(mg.hflag, 0, sizeof(int), st);
  for (int l = 0; l < mg.tail && l + 1 < nl; l++) {
    launch_mg_setup_level<T>(mg.L[l], mg.L[l + 1], st, mg.h16);
    k++;
  }
  if (mg.tail < nl - 1) {
    launch_setup_tail<T>(mg.Ldev, mg.tail, nl, st);
    k++;
  }
  if constexpr (std::is_same<T, float>::value) {
    if (mg.h16) {
      // the grid levels were scaled by their setup kernels; the tail levels
      // once their operators are final
      launch_h16_scale_tail(mg.Ldev, mg.tail, nl, st);
      k++;
    }
  }
  return k;
}

// One V-cycle with zero initial guess on level-0 (b -> x)
// (pfsimulator/parflow_lib/mg_semi.c:93-432 with MaxIter 1)
// Levels below mg.mid use one grid-wide kernel per phase; levels mg.mid ..
// mg.tail-1 (when there are any) run in one cluster kernel, which also runs
// levels mg.tail .. nl-1 (a few thousand cells each) in one of its blocks;
// otherwise those run inside one single-block kernel.
template <typename T>
static long long vcycle_T(MG<T> &mg, int smoother, double w, cudaStream_t st,
                          int max_iter = 1) {
  long long k = 0;
  const int nl = (int)mg.L.size();
  const int first = mg.mid;
  // block order of the next grid launch: with mg.flip every launch runs in
  // the opposite order of the one before it (the input conversion runs
  // forward), so it starts on the data still in L2
  int f = mg.flip ? 1 : 0;
  int *fp = mg.flip ? &f : nullptr;
  auto next = [&]() {
    const int r = f;
    if (mg.flip) f ^= 1;
    return r;
  };
  // MGSemi.MaxIter cycles (mg_semi.c:198-365 with KinsolPC's tolerance 0):
  // a cycle after the first begins with a smoothing of the finest level's
  // current iterate (the level runs on the grid kernels then, on the plain
  // colour sweeps); the coarse levels start from zero in every cycle
  for (int cyc = 0; cyc < max_iter; cyc++) {
  const int zero0 = cyc == 0 ? 1 : 0;
  for (int l = 0; l < first; l++) {
    MGLevel<T> &Ll = mg.L[l];
    const int zero = l == 0 ? zero0 : 1;
    if (Ll.lo[0]) {
      // the non-symmetric finest operator of FullJacobian (mg_full.cu)
      k += launch_mg_full_smooth<T>(Ll, Ll.x, Ll.b, zero, smoother != PFGPU_SMOOTH_RBGS_NONSYM,
                                    st);
      launch_mg_full_residual<T>(Ll, Ll.x, Ll.b, Ll.t, st);
      launch_mg_restrict<T>(Ll, mg.L[l + 1], Ll.t, mg.L[l + 1].b, st, next(), mg.h16);
      k += 2;
      continue;
    }
    if (mg.fused[l]) {
      launch_rbr_fused<T>(Ll, mg.maps[l], Ll.x, 1, mg.kerr, st);  // zero guess: x not read
      k++;
    } else if (mg.waved[l]) {
      launch_rbr_wave<T>(Ll, mg.wave[l], Ll.x, Ll.b, 1, mg.kerr, st);
      f = mg.flip ? 1 : 0;  // the wave ends on the top planes
      k++;
    } else {
      k += launch_mg_smooth<T>(Ll, Ll.x, Ll.b, zero, smoother, w, mg.wtmp, st, fp, mg.h16);
    }
    // after the plain red/black pre-smoother the colour swept last (red, or
    // black for the non-symmetric order) has a zero residual up to rounding
    launch_mg_residual<T>(Ll, Ll.x, Ll.b, Ll.t, st, next(), mg.h16, Ll.zc);
    launch_mg_restrict<T>(Ll, mg.L[l + 1], Ll.t, mg.L[l + 1].b, st, next(), mg.h16);
    k += 2;
  }
  // levels first .. nl-1, coarse solve (RedBlackGSPoint, mg_semi.c:1276) included
  if (mg.mid < mg.tail && mg.grid_blocks > 0) {
    const GridCtl ctl{mg.gbar, mg.gbar + 1, mg.kerr};
    launch_vcycle_grid<T>(mg.Ldev, mg.mid, mg.tail, 0, smoother, w, mg.wtmp, mg.grid_blocks, ctl,
                          st, mg.h16);
    launch_vcycle_tail<T>(mg.Ldev, mg.tail, nl, smoother, w, mg.wtmp, mg.tail_smem, st, mg.h16);
    launch_vcycle_grid<T>(mg.Ldev, mg.mid, mg.tail, 1, smoother, w, mg.wtmp, mg.grid_blocks, ctl,
                          st, mg.h16);
    k += 3;
  } else if (mg.mid < mg.tail) {
    launch_vcycle_mid<T>(mg.Ldev, mg.mid, mg.tail, nl, smoother, w, mg.wtmp, mg.tail_smem,
                         mg.mid_cs, st, mg.h16);
    k++;
  } else {
    launch_vcycle_tail<T>(mg.Ldev, first, nl, smoother, w, mg.wtmp, mg.tail_smem, st, mg.h16);
    k++;
  }
  for (int l = first - 1; l >= 0; l--) {
    MGLevel<T> &Ll = mg.L[l];
    const MGLevel<T> &C = mg.L[l + 1];
    // the plain red/black post-smoothers begin with a red sweep
    const int skip_red = (smoother == PFGPU_SMOOTH_RBGS || smoother == PFGPU_SMOOTH_RBGS_NONSYM) &&
                         !mg.fused[l] && !mg.waved[l];
    launch_mg_prolong_add<T>(Ll, C, mg.res(l + 1), Ll.x, st, next(), mg.h16, skip_red);
    if (Ll.lo[0]) {
      k += 1 + launch_mg_full_smooth<T>(Ll, Ll.x, Ll.b, 0,
                                        smoother != PFGPU_SMOOTH_RBGS_NONSYM, st);
    } else if (mg.fused[l]) {
      launch_rbr_fused<T>(Ll, mg.maps[l], Ll.x2, 0, mg.kerr, st);
      k += 2;
    } else if (mg.waved[l]) {
      launch_rbr_wave<T>(Ll, mg.wave[l], Ll.x, Ll.b, 0, mg.kerr, st);
      f = mg.flip ? 1 : 0;
      k += 2;
    } else {
      k += 1 + launch_mg_smooth<T>(Ll, Ll.x, Ll.b, 0, smoother, w, mg.wtmp, st, fp, mg.h16);
    }
  }
  }
  mg.flip_out = f;
  return k;
}

// buffer holding the level-0 result of a V-cycle
template <typename T>
static T *vcycle_out(MG<T> &mg, int) {
  return mg.res(0);
}

static long long vcycle_launch(pfgpu_handle *h) {
  if (h->mixed)
    return vcycle_T<float>(h->mgf, h->d.mg_smoother, h->d.wjacobi_weight, h->st, h->mg_max_iter);
  return vcycle_T<double>(h->mgd, h->d.mg_smoother, h->d.wjacobi_weight, h->st, h->mg_max_iter);
}

static int build_vgraph(pfgpu_handle *h) {
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  long long k = vcycle_launch(h);
  CK(cudaStreamEndCapture(h->st, &g));
  CK(cudaGraphInstantiate(&h->vgraph, g, 0));
  CK(cudaGraphDestroy(g));
  h->graph_nodes = k;
  return 0;
}

// z = M^{-1} r (dense FP64 device vectors; r and z may alias)
static int pc_apply_dense_impl(pfgpu_handle *h, const double *r, double *z) {
  int k = 0;
  if (h->mg_max_iter == 0) {
    // MGSemi.MaxIter 0: x = b (mg_semi.c:198-203)
    if (z != r)
      CK(cudaMemcpyAsync(z, r, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    return 0;
  }
  if (h->mixed)
    k += launch_level_in<float>(h->mgf.L[0], r, h->h16 ? h->mgf.L[0].sinv : nullptr, h->st);
  else
    k += launch_level_in<double>(h->mgd.L[0], r, nullptr, h->st);
  CK(cudaGetLastError());
  if (h->nk.capturing) {
    k += (int)vcycle_launch(h);  // inline in the solve's graph
  } else {
    CK(cudaGraphLaunch(h->vgraph, h->st));
    h->launches += h->graph_nodes;
  }
  if (h->mixed)
    k += launch_level_out<float>(h->mgf.L[0], vcycle_out(h->mgf, h->d.mg_smoother), z,
                                 h->h16 ? h->mgf.L[0].sinv : nullptr, h->mgf.flip_out, h->st);
  else
    k += launch_level_out<double>(h->mgd.L[0], vcycle_out(h->mgd, h->d.mg_smoother), z, nullptr,
                                  h->mgd.flip_out, h->st);
  CK(cudaGetLastError());
  h->launches += k;
  return 0;
}
static int pc_apply_dense(pfgpu_handle *h, const double *r, double *z) {
  const int m = ph_begin(h);
  const int rc = pc_apply_dense_impl(h, r, z);
  ph_end(h, m, PH_PCAPPLY);
  return rc;
}

static void pc_setup_dense_impl(pfgpu_handle *h, const double *u, double dt, bool also_J,
                                bool reuse_vg) {
  assemble(h, u, dt, also_J, true, reuse_vg);
  if (h->mixed)
    h->launches += mg_setup_T<float>(h->mgf, h->st);
  else
    h->launches += mg_setup_T<double>(h->mgd, h->st);
  if (also_J) h->jac_valid = 1;
  h->pc_ready = true;
}
static void pc_setup_dense(pfgpu_handle *h, const double *u, double dt, bool also_J,
                           bool reuse_vg = false) {
  const int m = ph_begin(h);
  pc_setup_dense_impl(h, u, dt, also_J, reuse_vg);
  ph_end(h, m, PH_PCSETUP);
}

// ---------------------------------------------------------------------------
// SPGMR (pfsimulator/kinsol/spgmr.c:168-450), x0 = 0, right preconditioning,
// modified Gram-Schmidt.  Returns 0 success, 1 residual reduced, 2 failure,
// 6 QR failure; J is assembled at the first matvec if not current.
// ---------------------------------------------------------------------------
// The right-hand side is b = bsign * src.  When its norm is already known
// (bnorm >= 0, with bnorm^2 in device memory at *bn2_dev: the Newton step
// reuses the norm of f from the line search) the start needs no reduction and
// no host synchronisation; V0 = b / ||b|| is then formed in one pass.  The
// solution x is written only on return, as M^{-1} (V y) (x0 = 0).
// z = J(u) v: the analytic matvec (J assembled at u on first use), or the
// difference quotient (F(u + sigma v) - F(u)) / sigma of KINSpgmrAtimesDQ
// (kinsol/kinspgmr.c:481-518, uscale = 1) with F(u) in h->fval
static void atimes(pfgpu_handle *h, const double *u, double dt, const double *v, double *z,
                   pfgpu_stats *stats) {
  if (h->use_jacobian) {
    if (!h->jac_valid) {
      assemble(h, u, dt, true, false, true);
      h->jac_valid = 1;
    }
    matvec(h, v, z);
    return;
  }
  launch_dq_prepare(u, v, h->N, h->dsc + D_DQ, h->sqrt_relfunc, h->rb, h->st);
  launch_dq_point(h->dq_w, u, v, h->dsc + D_DQ, h->N, h->st);
  h->launches += 3;
  feval(h, h->dq_w, dt, h->dq_f);
  stats->fevals++;
  launch_dq_finish(z, h->dq_f, h->fval, h->dsc + D_DQ, h->N, h->st);
  h->launches++;
}

static int spgmr(pfgpu_handle *h, double *x, const double *src, double bsign,
                 const double *bn2_dev, double bnorm, double delta, const double *u, double dt,
                 pfgpu_stats *stats, int *status) {
  const long long N = h->N;
  const int lmax = h->d.krylov_dim;
  double *S = h->gs;
  double *sc = S + gs_sc_offset(lmax);
  double *H = S;
  auto Hp = [&](int i, int j) { return H + (long long)i * lmax + j; };
  int krydim = 0, converged = 0;
  double rho = 0.0, r_norm;

  *status = 0;
  if (bnorm >= 0.0) {
    CK(cudaMemcpyAsync(sc + SCI_RNORM, bn2_dev, sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    launch_gmres_scalar(GM_START, S, 0, lmax, h->st);
    h->launches++;
    r_norm = bnorm;
  } else {
    launch_dot(src, src, N, sc + SCI_RNORM, h->rb, h->st);
    launch_gmres_scalar(GM_START, S, 0, lmax, h->st);
    h->launches += 2;
    CK(cudaMemcpyAsync(h->hsc + D_COUNT, sc + SCI_RNORM, sizeof(double), cudaMemcpyDeviceToHost,
                       h->st));
    CK(cudaStreamSynchronize(h->st));
    r_norm = h->hsc[D_COUNT];
  }
  const double beta = r_norm;
  if (r_norm <= delta) {
    launch_fill(x, 0.0, N, h->st);
    h->launches++;
    return 0;
  }

  for (int ntries = 0; ntries <= h->d.max_restarts; ntries++) {
    if (ntries == 0) {
      // V0 = b / r_norm = src * (bsign / r_norm)
      launch_axpby(h->V[0], src, bsign * (1.0 / r_norm), 0.0, N, h->st);
    } else {
      // the restart direction (built below) scaled by 1 / r_norm
      launch_scale_inv_dev(h->V[0], sc + SCI_RNORM, N, h->st);
    }
    h->launches++;
    int l;
    for (l = 0; l < lmax; l++) {
      stats->lin_iters++;
      krydim = l + 1;
      // z = M^{-1} V[l] (the preconditioner reads V[l], writes z: vtemp, or
      // the kept preconditioned basis vector Z[l])
      double *z = h->zbasis ? h->Z[l] : h->vtemp;
      if (pc_apply_dense(h, h->V[l], z)) return PFGPU_ERR_CUDA;
      stats->pc_solves++;
      atimes(h, u, dt, z, h->V[l + 1], stats);
      // ModifiedGS (iterativ.c:30-86): <vk,vk> and h(0) in one pass, then each
      // projection vk -= h(i) v_i fused with the next dot (h(i+1), or the
      // new <vk,vk> after the last); same per-element arithmetic
      const int k = l + 1;
      launch_mgs_first(h->V[k], h->V[0], N, sc + SCI_VKNORM2, Hp(0, k - 1), h->rb, h->st);
      h->launches++;
      for (int i = 0; i < k; i++) {
        const bool more = i + 1 < k;
        launch_axpy_dot(h->V[k], h->V[i], Hp(i, k - 1), -1.0, more ? h->V[i + 1] : nullptr, N,
                        more ? Hp(i + 1, k - 1) : sc + SCI_NEWNORM2, h->rb, h->st);
        h->launches++;
      }
      launch_gmres_scalar(GM_AFTER_GS, S, l, lmax, h->st);
      h->launches++;
      for (int i = 0; i < k; i++) {
        launch_dot_gated(h->V[i], h->V[k], N, sc + SCI_NP, sc + SCI_FLAG, h->rb, h->st);
        launch_reorth_decide(S, i, l, lmax, h->st);
        launch_axpy_gated(h->V[k], h->V[i], sc + SCI_COEF, sc + SCI_GATE, N, h->st);
        h->launches += 3;
      }
      launch_gmres_scalar(GM_REORTH_DONE, S, l, lmax, h->st);
      launch_gmres_scalar(GM_QR, S, l, lmax, h->st);
      h->launches += 2;
      CK(cudaMemcpyAsync(h->hsc + D_COUNT, sc + SCI_RHO, sizeof(double), cudaMemcpyDeviceToHost,
                         h->st));
      CK(cudaStreamSynchronize(h->st));
      rho = h->hsc[D_COUNT];
      if (rho <= delta) {
        converged = 1;
        break;
      }
      launch_scale_inv_dev(h->V[l + 1], Hp(l + 1, l), N, h->st);
      h->launches++;
    }
    // QRsol and xcor (+)= V y; with the kept basis x (+)= Z y directly
    launch_gmres_scalar(GM_QRSOL, S, krydim, lmax, h->st);
    if (h->zbasis)
      launch_combine(x, h->Z.data(), S + gs_yg_offset(lmax), krydim, N, h->st,
                     ntries > 0 ? 1 : 0);
    else
      launch_combine(h->xcor, h->V.data(), S + gs_yg_offset(lmax), krydim, N, h->st,
                     ntries > 0 ? 1 : 0);
    h->launches += 2;
    CK(cudaMemcpyAsync(h->hsc + D_COUNT, sc + SCI_QRFAIL, sizeof(double),
                       cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (h->hsc[D_COUNT] != 0.0) {
      *status = 6;
      launch_fill(x, 0.0, N, h->st);  // no solution: x stays x0 = 0
      h->launches++;
      return 0;
    }
    if (converged) {
      if (!h->zbasis) {
        if (pc_apply_dense(h, h->xcor, x)) return PFGPU_ERR_CUDA;  // x = 0 + M^{-1} V y
        stats->pc_solves++;
      }
      *status = 0;
      return 0;
    }
    if (ntries == h->d.max_restarts) break;
    // restart (spgmr.c:390-409): the new residual direction from the
    // Givens rotations and the current basis, then a fresh cycle
    launch_gmres_scalar(GM_RESTART, S, krydim, lmax, h->st);
    launch_restart_v0(h->V.data(), S + gs_yg_offset(lmax), krydim, N, h->st);
    launch_gmres_scalar(GM_RESTART_INIT, S, 0, lmax, h->st);
    h->launches += 3;
  }
  if (rho < beta) {
    if (!h->zbasis) {
      if (pc_apply_dense(h, h->xcor, x)) return PFGPU_ERR_CUDA;
      stats->pc_solves++;
    }
    *status = 1;
  } else {
    *status = 2;
    launch_fill(x, 0.0, N, h->st);
    h->launches++;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// KINSol with LineSearch (pfsimulator/kinsol/kinsol.c:363-910, 1054-1589).
// u (dense, device) holds the initial guess on entry and the result on exit.
// ---------------------------------------------------------------------------
static int newton_impl(pfgpu_handle *h, double dt, pfgpu_stats *stats) {
  const long long N = h->N;
  const pfgpu_desc &d = h->d;
  const double uround = DBL_EPSILON;
  double fnormtol = d.residual_tol, scsteptol = d.step_tol;
  if (scsteptol <= 0.0) scsteptol = pow(uround, 2.0 / 3.0);
  if (fnormtol <= 0.0) fnormtol = pow(uround, 1.0 / 3.0);
  const int mxiter = d.max_iter > 0 ? d.max_iter : 200;
  int etaflag = d.eta_choice;
  double ealpha = 0.0, egamma = 0.0;
  if (etaflag == 1) ealpha = (1.0 + sqrt(5.0)) / 2.0;
  if (etaflag == 2) {
    ealpha = d.eta_alpha;
    egamma = d.eta_gamma;
    if (ealpha <= 1.0 || ealpha > 2.0) ealpha = 2.0;
    if (egamma <= 0.0 || egamma > 1.0) egamma = 0.9;
  }
  double eta = (etaflag == 0) ? d.eta_value : 0.5;
  if (eta <= 0.0 || eta > 1.0) eta = 0.1;
  const bool callForcingTerm = (etaflag != 0);
  const double epsmin = 0.01 * fnormtol;
  memset(stats, 0, sizeof(*stats));
  double *u = h->u;
  double *unew = h->unew;
  double *dsc = h->dsc, *hsc = h->hsc;
  h->vg_for = nullptr;

  // mxnewtstep = 1000 ||u|| (KINSolInit, kinsol.c:540-545)
  // KINInitialStop; <u,u>, max|f| and <f,f> in one pass
  feval(h, u, dt, h->fval);
  stats->fevals++;
  launch_init_norms(u, h->fval, N, dsc + D_U2, dsc + D_FMAX, dsc + D_F2, h->rb, h->st);
  h->launches++;
  if (read_scalars(h, 0, D_COUNT)) return PFGPU_ERR_CUDA;
  double mxnewtstep = 1000.0 * sqrt(hsc[D_U2]);
  if (mxnewtstep < 1.0) mxnewtstep = 1.0;
  if (hsc[D_FMAX] <= 0.01 * fnormtol) {
    // KINSol returns before loading its optional outputs: counters stay zero
    // (pfsimulator/kinsol/kinsol.c:726-731, 851-862)
    stats->fevals = 0;
    stats->kinsol_status = 2;
    stats->fnorm = sqrt(hsc[D_F2]);
    return PFGPU_OK;
  }
  double fnorm = sqrt(hsc[D_F2]);
  double f1norm = 0.5 * fnorm * fnorm;
  int ret = 0, ncscmx = 0;

  for (int guard = 0; guard < 100000; guard++) {
    stats->nonlin_iters++;
    double eps = (eta + uround) * fnorm;
    if (eps < epsmin) eps = epsmin;
    // preconditioner setup every iteration (msbpre = 1); J at the same u
    h->jac_valid = 0;
    pc_setup_dense(h, u, dt, h->use_jacobian != 0, true);
    stats->pc_setups++;
    // b = -f; its norm is the fnorm of the last residual evaluation
    int sstat = 0;
    int rc = spgmr(h, h->pp, h->fval, -1.0, dsc + D_F2, fnorm, eps, u, dt, stats, &sstat);
    if (rc) return rc;
    if (sstat != 0 && sstat != 1) {
      stats->lin_conv_fails++;
      ret = 8;
      break;
    }
    // sJpnorm, sfdotJp (kinspgmr.c:384-398) and line-search inputs; J p by
    // KINSpgmrAtimes, analytic or by difference quotient
    atimes(h, u, dt, h->pp, h->bb, stats);
    launch_linesearch_inputs(h->bb, h->fval, h->pp, u, N, dsc + D_JP2, dsc + D_FJP, dsc + D_P2,
                             dsc + D_PLEN, h->rb, h->st);
    h->launches++;
    if (read_scalars(h, 0, D_COUNT)) return PFGPU_ERR_CUDA;
    double sJpnorm = sqrt(hsc[D_JP2]);
    double sfdotJp = hsc[D_FJP];

    // KINLineSearch (kinsol.c:1228-1420)
    int globalret = 0, maxStepTaken = 0;
    double fnormp = 0.0, f1normp = 0.0, fmax = 0.0;
    // KINStop's scaled step length is 1 whatever the step (kinsol.c:1540-1541
    // pass the step in the work vector that KINScSteplength, :1490-1498,
    // overwrites with 1/uscale + |unew| before dividing by it)
    const double steplen_new = 1.0;
    double pnorm = sqrt(hsc[D_P2]);
    double ratio = 1.0;
    const double alpha = 0.0001, beta = 0.9;
    if (pnorm > mxnewtstep) {
      ratio = mxnewtstep / pnorm;
      launch_scale(h->pp, ratio, N, h->st);
      launch_steplen(h->pp, u, N, dsc + D_PLEN, h->rb, h->st);
      h->launches += 2;
      if (read_scalars(h, D_PLEN, 1)) return PFGPU_ERR_CUDA;
      pnorm = mxnewtstep;
    }
    const double stepl = pnorm;
    const double slpi = sfdotJp * ratio;
    const double rlength = hsc[D_PLEN];
    const double rlmin = scsteptol / rlength;
    double rl = 1.0, rlprev = 0.0, alpha_cond, beta_cond;
    const int nfesav = stats->fevals;
    auto try_step = [&](double lam) -> int {
      if (lam == 0.0) {  // N_VScale(ONE, uu, unew)
        if (cudaMemcpyAsync(unew, u, N * sizeof(double), cudaMemcpyDeviceToDevice, h->st) !=
            cudaSuccess)
          return PFGPU_ERR_CUDA;
      } else {
        launch_xpay(unew, u, lam, h->pp, N, h->st);
      }
      feval(h, unew, dt, h->fval);
      stats->fevals++;
      launch_step_norms(h->fval, N, dsc + D_F2, dsc + D_FMAX, h->rb, h->st);
      h->launches += 2;
      if (read_scalars(h, 0, 2)) return PFGPU_ERR_CUDA;
      fnormp = sqrt(hsc[D_F2]);
      f1normp = 0.5 * fnormp * fnormp;
      fmax = hsc[D_FMAX];
      return 0;
    };
    if (h->globalization == PFGPU_GLOBAL_INEXACT_NEWTON) {
      // KINInexactNewton (kinsol.c:1152-1208): the full (possibly shortened)
      // step; the common tail below scales sfdotJp and sJpnorm by ratio
      // (rl = 1) and takes maxStepTaken from pnorm
      if (try_step(rl)) return PFGPU_ERR_CUDA;
    } else {
      for (int it = 0;; it++) {
        if (it > 1000) {
          set_err("line search exceeded its iteration bound");
          return PFGPU_ERR_STATE;
        }
        if (try_step(rl)) return PFGPU_ERR_CUDA;
        alpha_cond = f1norm + alpha * slpi * rl;
        if (f1normp <= alpha_cond) break;
        if (rl < rlmin) {
          // unew = u, re-evaluate and return 1
          if (try_step(0.0)) return PFGPU_ERR_CUDA;
          stats->backtracks = stats->fevals - nfesav - 1;
          globalret = 1;
          goto ls_done;
        }
        {
          double rltmp = -slpi / (2.0 * (f1normp - f1norm - slpi));
          if (rltmp > 0.5 * rl) rltmp = 0.5 * rl;
          rlprev = rl;
          double pt1trl = 0.1 * rl;
          rl = (pt1trl > rltmp) ? pt1trl : rltmp;
        }
      }
      beta_cond = f1norm + beta * slpi * rl;
      if (f1normp < beta_cond) {
        // (rl == 1 && pnorm < stepl) never holds without constraints
        if (rl < 1.0 || ((rl > 1.0) && (f1normp > alpha_cond))) {
          double rllo = (rl < rlprev) ? rl : rlprev;
          double rldiff = fabs(rlprev - rl);
          int it = 0;
          do {
            if (++it > 1000) {
              set_err("line search refinement exceeded its iteration bound");
              return PFGPU_ERR_STATE;
            }
            double rlincr = 0.5 * rldiff;
            rl = rllo + rlincr;
            if (try_step(rl)) return PFGPU_ERR_CUDA;
            alpha_cond = f1norm + alpha * slpi * rl;
            beta_cond = f1norm + beta * slpi * rl;
            if (f1normp > alpha_cond)
              rldiff = rlincr;
            else if (f1normp < beta_cond) {
              rllo = rl;
              rldiff = rldiff - rlincr;
            }
          } while (f1normp > alpha_cond || ((f1normp < beta_cond) && (rldiff > rlmin)));
          if (f1normp < beta_cond) {
            if (try_step(rllo)) return PFGPU_ERR_CUDA;
            stats->beta_cond_fails++;
          }
        }
      }
    }
    stats->backtracks = stats->fevals - nfesav - 1;
    sfdotJp = sfdotJp * rl * ratio;
    sJpnorm = sJpnorm * rl * ratio;
    if (rl * pnorm > 0.99 * mxnewtstep) maxStepTaken = 1;
    (void)stepl;
  ls_done:
    if (stats->beta_cond_fails > 10) {
      ret = 7;
      break;
    }
    // KINForcingTerm (kinsol.c:1054-1090)
    if (callForcingTerm) {
      double eta_max = 0.9, eta_min = 0.0001, eta_safe = 0.5;
      if (etaflag == 1) {
        double linmodel_norm = sqrt(fnorm * fnorm + 2.0 * sfdotJp + sJpnorm * sJpnorm);
        eta_safe = pow(eta, ealpha);
        eta = fabs(fnormp - linmodel_norm) / fnorm;
      }
      if (etaflag == 2) {
        eta_safe = egamma * pow(eta, ealpha);
        eta = egamma * pow(fnormp / fnorm, ealpha);
      }
      if (eta_safe < 0.1) eta_safe = 0.0;
      if (eta < eta_safe) eta = eta_safe;
      if (eta < eta_min) eta = eta_min;
      if (eta > eta_max) eta = eta_max;
    }
    fnorm = fnormp;
    // KINStop (kinsol.c:1507-1589); the preconditioner is always current
    int sret = 0;
    if (globalret == 1)
      sret = 3;
    else if (fmax <= fnormtol)
      sret = 1;
    else if (steplen_new <= scsteptol)
      sret = 2;
    else if (stats->nonlin_iters >= mxiter)
      sret = 4;
    else {
      ncscmx = maxStepTaken ? ncscmx + 1 : 0;
      if (ncscmx == 5) sret = 5;
    }
    // u <- unew (swap)
    double *t = h->u;
    h->u = h->unew;
    h->unew = t;
    u = h->u;
    unew = h->unew;
    f1norm = f1normp;
    if (sret != 0) {
      ret = sret;
      break;
    }
  }
  stats->kinsol_status = ret;
  stats->fnorm = fnorm;
  return (ret == 1 || ret == 2) ? PFGPU_OK : PFGPU_NOT_CONVERGED;
}
// ---------------------------------------------------------------------------
// The Newton solve as one CUDA graph.  The same launches as newton_impl and
// spgmr, captured once per handle; the decisions the host makes there between
// launches are made on the device by the control kernels of nk_control.cu,
// which steer conditional nodes:
//
//   F(u), norms, init
//   WHILE newton:
//     iter; J and preconditioner setup; SPGMR start
//     WHILE restart:                        (one GMRES cycle)
//       cycle_begin; V0
//       iteration 0, IF iteration 1, ..., IF iteration lmax-1
//       QR solve; x (+)= V y; cycle_end
//       IF restart: restart direction
//     after_gmres; IF post: x = M^{-1} V y; x = 0 when SPGMR gave none
//     IF ok:
//       J p, line-search inputs; ls_init; IF scale: scale p
//       WHILE backtrack: trial; ls1
//       WHILE refine: trial; ls2
//       IF rllo: trial; ls3
//       newton_end; u <- unew
//     tail
//   final
//
// The vectors and the iterate keep their buffers (u <- unew is a copy where
// the host-driven loop swaps pointers); dt is read from device memory, so one
// graph serves every timestep until the problem's device description, the
// iterate buffers or the Jacobian mode change.
// ---------------------------------------------------------------------------
static void nk_begin(pfgpu_handle *h, int body) {
  h->nk.stack.push_back({(long long)body, h->launches, 0});
}
static void nk_end(pfgpu_handle *h) {
  const std::array<long long, 3> t = h->nk.stack.back();
  h->nk.stack.pop_back();
  const long long total = h->launches - t[1];
  h->nk.kernels[t[0]] += total - t[2];
  if (!h->nk.stack.empty()) h->nk.stack.back()[2] += total;
}

// a conditional handle of the graph being captured on stream s
static int nk_handle(cudaStream_t s, cudaGraphConditionalHandle *hd) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
  CK(cudaGraphConditionalHandleCreate(hd, g, 0, 0));
  return 0;
}

// appends a conditional node at the capture point of stream s; returns its body
static int nk_cond(cudaStream_t s, cudaGraphConditionalHandle hd,
                   cudaGraphConditionalNodeType type, cudaGraph_t *body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = hd;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, deps, nd, &p));
  CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  *body = p.conditional.phGraph_out[0];
  return 0;
}

// captures fn's launches into a conditional node's body on the capture
// stream of nesting depth `depth`, attributing them to body `count`
template <typename F>
static int nk_body(pfgpu_handle *h, cudaGraphConditionalHandle hd,
                   cudaGraphConditionalNodeType type, int depth, int count, F fn) {
  cudaGraph_t body = nullptr;
  if (nk_cond(h->st, hd, type, &body)) return PFGPU_ERR_CUDA;
  cudaStream_t s = h->nk.cs[depth];
  CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  cudaStream_t saved = h->st;
  h->st = s;
  nk_begin(h, count);
  int rc = fn();
  if (!rc && cudaPeekAtLastError() != cudaSuccess) {
    set_err("launch failed while capturing the solve graph: %s",
            cudaGetErrorString(cudaGetLastError()));
    rc = PFGPU_ERR_CUDA;
  }
  nk_end(h);
  h->st = saved;
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &out);
  if (rc) return rc;
  CK(e);
  return 0;
}

static void nk_try_step(pfgpu_handle *h, double dt) {
  const long long N = h->N;
  double *dsc = h->dsc;
  launch_xpay_lam(h->unew, h->u, &h->nk.S->lam, h->pp, N, h->st);
  feval(h, h->unew, dt, h->fval);
  launch_step_norms(h->fval, N, dsc + D_F2, dsc + D_FMAX, h->rb, h->st);
  h->launches += 2;
}

// one GMRES iteration l of a cycle (as the body of spgmr's inner loop)
static int nk_gmres_iter(pfgpu_handle *h, int l, double dt, NkConds &C) {
  const long long N = h->N;
  const int lmax = h->d.krylov_dim;
  double *S = h->gs;
  double *sc = S + gs_sc_offset(lmax);
  auto Hp = [&](int i, int j) { return S + (long long)i * lmax + j; };
  pfgpu_stats dummy{};
  double *z = h->zbasis ? h->Z[l] : h->vtemp;
  if (pc_apply_dense_impl(h, h->V[l], z)) return PFGPU_ERR_CUDA;
  atimes(h, h->u, dt, z, h->V[l + 1], &dummy);
  const int k = l + 1;
  launch_mgs_first(h->V[k], h->V[0], N, sc + SCI_VKNORM2, Hp(0, k - 1), h->rb, h->st);
  h->launches++;
  for (int i = 0; i < k; i++) {
    const bool more = i + 1 < k;
    launch_axpy_dot(h->V[k], h->V[i], Hp(i, k - 1), -1.0, more ? h->V[i + 1] : nullptr, N,
                    more ? Hp(i + 1, k - 1) : sc + SCI_NEWNORM2, h->rb, h->st);
    h->launches++;
  }
  launch_gmres_scalar(GM_AFTER_GS, S, l, lmax, h->st);
  h->launches++;
  for (int i = 0; i < k; i++) {
    launch_dot_gated(h->V[i], h->V[k], N, sc + SCI_NP, sc + SCI_FLAG, h->rb, h->st);
    launch_reorth_decide(S, i, l, lmax, h->st);
    launch_axpy_gated(h->V[k], h->V[i], sc + SCI_COEF, sc + SCI_GATE, N, h->st);
    h->launches += 3;
  }
  launch_gmres_scalar(GM_REORTH_DONE, S, l, lmax, h->st);
  launch_gmres_scalar(GM_QR, S, l, lmax, h->st);
  launch_nk_gm_iter(h->nk.S, sc, l, C, h->st);
  launch_scale_inv_dev_unless(h->V[l + 1], Hp(l + 1, l), &h->nk.S->converged, N, h->st);
  h->launches += 4;
  return 0;
}

// one GMRES cycle (the body of spgmr's restart loop)
static int nk_gmres_cycle(pfgpu_handle *h, double dt, NkConds &C) {
  const long long N = h->N;
  const int lmax = h->d.krylov_dim;
  double *S = h->gs;
  double *sc = S + gs_sc_offset(lmax);
  NkState *St = h->nk.S;
  for (int l = 1; l < lmax; l++)
    if (nk_handle(h->st, &C.iter[l])) return PFGPU_ERR_CUDA;
  if (nk_handle(h->st, &C.do_restart)) return PFGPU_ERR_CUDA;
  launch_nk_cycle_begin(St, C, h->st);
  launch_v0_init(h->V[0], h->fval, St, sc, N, h->st);
  h->launches += 2;
  // iteration l + 1 nests inside iteration l's body: once GMRES stops, no
  // further conditional node is evaluated
  std::function<int(int)> iteration = [&](int l) -> int {
    const int rc = nk_gmres_iter(h, l, dt, C);
    if (rc || l + 1 >= lmax) return rc;
    return nk_body(h, C.iter[l + 1], cudaGraphCondTypeIf, 4 + l, NKB_GM0 + l + 1,
                   [&]() { return iteration(l + 1); });
  };
  nk_begin(h, NKB_GM0);
  int rc = iteration(0);
  nk_end(h);
  if (rc) return rc;
  launch_gmres_scalar_dev(GM_QRSOL, S, &St->krydim, lmax, h->st);
  if (h->zbasis)
    launch_combine_dev(h->pp, h->Z.data(), lmax, S + gs_yg_offset(lmax), &St->krydim,
                       &St->accumulate, N, h->st);
  else
    launch_combine_dev(h->xcor, h->V.data(), lmax + 1, S + gs_yg_offset(lmax), &St->krydim,
                       &St->accumulate, N, h->st);
  launch_nk_cycle_end(St, sc, C, h->st);
  h->launches += 3;
  return nk_body(h, C.do_restart, cudaGraphCondTypeIf, 3, NKB_RESTART, [&]() {
    launch_gmres_scalar_dev(GM_RESTART, S, &St->krydim, lmax, h->st);
    launch_restart_v0_dev(h->V.data(), lmax + 1, S + gs_yg_offset(lmax), &St->krydim, N, h->st);
    launch_gmres_scalar(GM_RESTART_INIT, S, 0, lmax, h->st);
    launch_nk_count(St, NKB_RESTART, 0, h->st);
    h->launches += 4;
    return 0;
  });
}

// the line search after a successful linear solve (kinsol.c:1228-1420)
static int nk_line_search(pfgpu_handle *h, double dt, NkConds &C) {
  const long long N = h->N;
  double *dsc = h->dsc;
  NkState *St = h->nk.S;
  pfgpu_stats dummy{};
  if (nk_handle(h->st, &C.scale) || nk_handle(h->st, &C.ls1) || nk_handle(h->st, &C.ls2) ||
      nk_handle(h->st, &C.ls3))
    return PFGPU_ERR_CUDA;
  atimes(h, h->u, dt, h->pp, h->bb, &dummy);
  launch_linesearch_inputs(h->bb, h->fval, h->pp, h->u, N, dsc + D_JP2, dsc + D_FJP, dsc + D_P2,
                           dsc + D_PLEN, h->rb, h->st);
  launch_nk_ls_init(St, dsc, C, h->st);
  h->launches += 2;
  int rc = nk_body(h, C.scale, cudaGraphCondTypeIf, 3, NKB_SCALE, [&]() {
    launch_scale_by(h->pp, &St->ratio, N, h->st);
    launch_steplen(h->pp, h->u, N, dsc + D_PLEN, h->rb, h->st);
    launch_nk_count(St, NKB_SCALE, 0, h->st);
    h->launches += 3;
    return 0;
  });
  if (rc) return rc;
  launch_nk_ls_setup(St, dsc, C, h->st);
  h->launches++;
  rc = nk_body(h, C.ls1, cudaGraphCondTypeWhile, 3, NKB_LS1, [&]() {
    nk_try_step(h, dt);
    launch_nk_ls1(St, dsc, C, h->st);
    h->launches++;
    return 0;
  });
  if (rc) return rc;
  launch_nk_ls2_init(St, C, h->st);
  h->launches++;
  rc = nk_body(h, C.ls2, cudaGraphCondTypeWhile, 3, NKB_LS2, [&]() {
    nk_try_step(h, dt);
    launch_nk_ls2(St, dsc, C, h->st);
    h->launches++;
    return 0;
  });
  if (rc) return rc;
  launch_nk_ls3_decide(St, C, h->st);
  h->launches++;
  rc = nk_body(h, C.ls3, cudaGraphCondTypeIf, 3, NKB_LS3, [&]() {
    nk_try_step(h, dt);
    launch_nk_ls3(St, dsc, h->st);
    h->launches++;
    return 0;
  });
  if (rc) return rc;
  launch_nk_newton_end(St, h->st);
  launch_copy_if(h->u, h->unew, &St->do_copy, N, h->st);
  h->launches += 2;
  return 0;
}

// one Newton iteration (the body of newton_impl's loop)
static int nk_newton_iter(pfgpu_handle *h, double dt, NkConds &C) {
  const long long N = h->N;
  const int lmax = h->d.krylov_dim;
  double *S = h->gs;
  double *sc = S + gs_sc_offset(lmax);
  NkState *St = h->nk.S;
  if (nk_handle(h->st, &C.ok) || nk_handle(h->st, &C.restart) || nk_handle(h->st, &C.post))
    return PFGPU_ERR_CUDA;
  launch_nk_iter(St, C, h->st);
  h->launches++;
  h->jac_valid = 0;
  pc_setup_dense_impl(h, h->u, dt, h->use_jacobian != 0, true);
  CK(cudaMemcpyAsync(sc + SCI_RNORM, h->dsc + D_F2, sizeof(double), cudaMemcpyDeviceToDevice,
                     h->st));
  launch_gmres_scalar(GM_START, S, 0, lmax, h->st);
  h->launches++;
  int rc = nk_body(h, C.restart, cudaGraphCondTypeWhile, 2, NKB_CYCLE,
                   [&]() { return nk_gmres_cycle(h, dt, C); });
  if (rc) return rc;
  launch_nk_after_gmres(St, C, h->st);
  h->launches++;
  rc = nk_body(h, C.post, cudaGraphCondTypeIf, 2, NKB_POST, [&]() {
    if (h->zbasis) {  // x = Z y is already formed
      launch_nk_count(St, NKB_POST, 0, h->st);
    } else {
      if (pc_apply_dense_impl(h, h->xcor, h->pp)) return (int)PFGPU_ERR_CUDA;
      launch_nk_count(St, NKB_POST, 1, h->st);
    }
    h->launches++;
    return 0;
  });
  if (rc) return rc;
  launch_fill_if(h->pp, 0.0, &St->zero_x, N, h->st);
  h->launches++;
  rc = nk_body(h, C.ok, cudaGraphCondTypeIf, 2, NKB_OK,
               [&]() { return nk_line_search(h, dt, C); });
  if (rc) return rc;
  launch_nk_tail(St, C, h->st);
  h->launches++;
  return 0;
}

// everything a captured solve bakes in: the problem's device description
// (its dt pointer aside), the solver settings, the iterate buffers and the
// Jacobian mode.  Copied bytewise: a spurious difference only costs a capture.
static std::vector<unsigned char> nk_key(pfgpu_handle *h) {
  DevProblem P;
  memcpy(&P, &h->P, sizeof(P));
  P.dtp = nullptr;
  const double *ptrs[2] = {h->u, h->unew};
  std::vector<unsigned char> k(sizeof(P) + sizeof(h->d) + sizeof(ptrs) + 4 * sizeof(int) +
                               sizeof(double));
  unsigned char *q = k.data();
  memcpy(q, &P, sizeof(P));
  q += sizeof(P);
  memcpy(q, &h->d, sizeof(h->d));
  q += sizeof(h->d);
  memcpy(q, ptrs, sizeof(ptrs));
  q += sizeof(ptrs);
  memcpy(q, &h->use_jacobian, sizeof(int));
  q += sizeof(int);
  memcpy(q, &h->sqrt_relfunc, sizeof(double));
  q += sizeof(double);
  memcpy(q, &h->globalization, sizeof(int));
  q += sizeof(int);
  memcpy(q, &h->pc_matrix, sizeof(int));
  q += sizeof(int);
  memcpy(q, &h->mg_max_iter, sizeof(int));
  return k;
}

// Captures the solve into a new graph, or (target given) as one more root
// branch of the ensemble graph `target`: there the branch also takes the
// step's start (dt in, p_old = u, s_old = S(u)) and ends with the control
// state and the error word copied to pinned host memory.
static int nk_capture(pfgpu_handle *h, cudaGraph_t *graph, cudaGraph_t target) {
  pfgpu_handle::NkGraph &G = h->nk;
  const long long N = h->N;
  double *dsc = h->dsc;
  NkConds C{};
  for (auto &k : G.kernels) k = 0;
  G.stack.clear();
  cudaStream_t s0 = G.cs[0];
  if (target)
    CK(cudaStreamBeginCaptureToGraph(s0, target, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
  else
    CK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  cudaStream_t saved = h->st;
  h->st = s0;
  int rc = nk_handle(s0, &C.newton);
  if (!rc && target) {
    if (cudaMemcpyAsync(G.dt, G.hdt, sizeof(double), cudaMemcpyHostToDevice, s0) !=
            cudaSuccess ||
        cudaMemcpyAsync(h->p_old, h->u, N * sizeof(double), cudaMemcpyDeviceToDevice, s0) !=
            cudaSuccess) {
      set_err("solve graph: copy capture failed: %s", cudaGetErrorString(cudaGetLastError()));
      rc = PFGPU_ERR_CUDA;
    }
    launch_saturation(h->P, h->u, h->s_old, s0);
  }
  if (!rc) {
    nk_begin(h, NKB_TOP);
    h->vg_for = nullptr;
    const double dt = 0.0;  // the kernels read dt from G.dt (P.dtp)
    feval(h, h->u, dt, h->fval);
    launch_init_norms(h->u, h->fval, N, dsc + D_U2, dsc + D_FMAX, dsc + D_F2, h->rb, h->st);
    launch_nk_init(G.S, dsc, C, h->st);
    h->launches += 2;
    rc = nk_body(h, C.newton, cudaGraphCondTypeWhile, 1, NKB_NEWTON,
                 [&]() { return nk_newton_iter(h, dt, C); });
    launch_nk_final(G.S, h->st);
    h->launches++;
    nk_end(h);
  }
  if (!rc && target &&
      (cudaMemcpyAsync(G.hS, G.S, sizeof(NkState), cudaMemcpyDeviceToHost, s0) != cudaSuccess ||
       cudaMemcpyAsync(h->hkerr, h->kerr, sizeof(int), cudaMemcpyDeviceToHost, s0) !=
           cudaSuccess)) {
    set_err("solve graph: copy capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    rc = PFGPU_ERR_CUDA;
  }
  h->st = saved;
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s0, &out);
  if (graph) *graph = target ? nullptr : out;
  if (rc) {
    if (out && !target) cudaGraphDestroy(out);
    if (graph) *graph = nullptr;
    return rc;
  }
  CK(e);
  return 0;
}

// the solver constants on the device and the capture streams (once per handle)
static int nk_setup(pfgpu_handle *h) {
  pfgpu_handle::NkGraph &G = h->nk;
  if (!G.S) {
    if (dalloc(&G.S, 1) || dalloc(&G.dt, 1)) return PFGPU_ERR_CUDA;
    CK(cudaMallocHost(&G.hS, sizeof(NkState)));
    CK(cudaMallocHost(&G.hdt, sizeof(double)));
    // depths: top, Newton body, GMRES cycle / line search, their bodies, and
    // the nested GMRES iterations
    G.cs.assign(h->d.krylov_dim + 6, nullptr);
    for (auto &s : G.cs) CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  }
  // constants of the solve (newton_impl's set-up)
  const pfgpu_desc &d = h->d;
  const double uround = DBL_EPSILON;
  NkConst k{};
  k.fnormtol = d.residual_tol;
  k.scsteptol = d.step_tol;
  if (k.scsteptol <= 0.0) k.scsteptol = pow(uround, 2.0 / 3.0);
  if (k.fnormtol <= 0.0) k.fnormtol = pow(uround, 1.0 / 3.0);
  k.mxiter = d.max_iter > 0 ? d.max_iter : 200;
  k.etaflag = d.eta_choice;
  if (k.etaflag == 1) k.ealpha = (1.0 + sqrt(5.0)) / 2.0;
  if (k.etaflag == 2) {
    k.ealpha = d.eta_alpha;
    k.egamma = d.eta_gamma;
    if (k.ealpha <= 1.0 || k.ealpha > 2.0) k.ealpha = 2.0;
    if (k.egamma <= 0.0 || k.egamma > 1.0) k.egamma = 0.9;
  }
  k.eta0 = (k.etaflag == 0) ? d.eta_value : 0.5;
  if (k.eta0 <= 0.0 || k.eta0 > 1.0) k.eta0 = 0.1;
  k.epsmin = 0.01 * k.fnormtol;
  k.bsign = -1.0;
  k.lmax = d.krylov_dim;
  k.max_restarts = d.max_restarts;
  k.use_dq = h->use_jacobian ? 0 : 1;
  k.inexact = h->globalization == PFGPU_GLOBAL_INEXACT_NEWTON ? 1 : 0;
  CK(cudaMemcpy(&G.S->k, &k, sizeof(k), cudaMemcpyHostToDevice));
  return 0;
}

// nk_capture with the handle switched to capture mode (device dt, inline
// V-cycles) and its host-side state restored afterwards
static int nk_capture_guarded(pfgpu_handle *h, cudaGraph_t *graph, cudaGraph_t target) {
  pfgpu_handle::NkGraph &G = h->nk;
  const DevProblem P0 = h->P;
  const long long launches0 = h->launches;
  const int jac0 = h->jac_valid;
  h->P.dtp = G.dt;
  G.capturing = true;
  const int rc = nk_capture(h, graph, target);
  G.capturing = false;
  h->P = P0;
  h->launches = launches0;
  h->jac_valid = jac0;
  h->vg_for = nullptr;
  return rc;
}

// (re)builds the solve graph when what it was captured for has changed
static int nk_prepare(pfgpu_handle *h) {
  pfgpu_handle::NkGraph &G = h->nk;
  std::vector<unsigned char> key = nk_key(h);
  if (G.valid) {
    if (key == G.key) return 0;
    pfgpu_handle::NkGraph::Kept old{std::move(G.key), G.exec, {}};
    std::copy(std::begin(G.kernels), std::end(G.kernels), old.kernels.begin());
    G.kept.push_back(std::move(old));
    G.exec = nullptr;
    G.valid = false;
    for (size_t i = 0; i < G.kept.size(); i++)
      if (G.kept[i].key == key) {
        G.exec = G.kept[i].exec;
        G.key = std::move(G.kept[i].key);
        std::copy(G.kept[i].kernels.begin(), G.kept[i].kernels.end(), std::begin(G.kernels));
        G.kept.erase(G.kept.begin() + (long)i);
        G.valid = true;
        return 0;
      }
    constexpr size_t KEEP = 4;
    while (G.kept.size() > KEEP) {
      cudaGraphExecDestroy(G.kept.front().exec);
      G.kept.erase(G.kept.begin());
    }
  }
  if (nk_setup(h)) return PFGPU_ERR_CUDA;
  cudaGraph_t graph = nullptr;
  bool pdl_used = pdl_on();
  int rc = nk_capture_guarded(h, &graph, nullptr);
  cudaGraphExec_t exec = nullptr;
  if (!rc && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    // programmatic launches inside conditional bodies are what a driver may
    // refuse: capture again without them
    cudaGetLastError();
    cudaGraphDestroy(graph);
    graph = nullptr;
    exec = nullptr;
    pdl_capture_off() = true;
    pdl_used = false;
    rc = nk_capture_guarded(h, &graph, nullptr);
    pdl_capture_off() = false;
    if (!rc && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
      set_err("solve graph: instantiation failed: %s", cudaGetErrorString(cudaGetLastError()));
      exec = nullptr;
      rc = PFGPU_ERR_CUDA;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  if (rc) return rc;
  CK(cudaGraphUpload(exec, h->st));
  G.exec = exec;
  G.valid = true;
  G.key = nk_key(h);
  if (env_ll("PFGPU_GRAPH_INFO", 0)) {
    long long nk = 0;
    for (long long c : G.kernels) nk += c;
    fprintf(stderr, "pfgpu solve graph (%dx%dx%d): %lld kernel nodes, programmatic launches %s\n",
            h->nx, h->ny, h->nz, nk, pdl_used ? "on" : "off");
  }
  return 0;
}

static bool nk_usable(pfgpu_handle *h) {
  const pfgpu_handle::NkGraph &G = h->nk;
  if (!G.enabled || G.failed || h->ptime) return false;
  // cooperative launches stay out of captured graphs
  return (h->mixed ? h->mgf.grid_blocks : h->mgd.grid_blocks) == 0;
}

static int newton_graph(pfgpu_handle *h, double dt, pfgpu_stats *stats) {
  pfgpu_handle::NkGraph &G = h->nk;
  *G.hdt = dt;
  CK(cudaMemcpyAsync(G.dt, G.hdt, sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaGraphLaunch(G.exec, h->st));
  CK(cudaMemcpyAsync(G.hS, G.S, sizeof(NkState), cudaMemcpyDeviceToHost, h->st));
  // every loop of the graph is bounded by its control kernels; the host
  // still waits at most PFGPU_SOLVE_TIMEOUT_S seconds (default 600)
  {
    static const double limit = (double)env_ll("PFGPU_SOLVE_TIMEOUT_S", 600);
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t q = cudaStreamQuery(h->st);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) CK(q);
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit) {
        set_err("solve graph did not finish within %.0f s", limit);
        return PFGPU_ERR_STATE;
      }
      std::this_thread::yield();
    }
  }
  const NkState &S = *G.hS;
  long long k = 0;
  for (int b = 0; b < NKB_COUNT; b++) k += G.kernels[b] * (long long)S.execs[b];
  h->launches += k;
  h->vg_for = nullptr;
  h->jac_valid = 0;
  memset(stats, 0, sizeof(*stats));
  stats->nonlin_iters = S.nonlin_iters;
  stats->lin_iters = S.lin_iters;
  stats->fevals = S.fevals;
  stats->pc_setups = S.pc_setups;
  stats->pc_solves = S.pc_solves;
  stats->lin_conv_fails = S.lin_conv_fails;
  stats->beta_cond_fails = S.beta_cond_fails;
  stats->backtracks = S.backtracks;
  stats->kinsol_status = S.kinsol_status;
  stats->fnorm = S.fnorm;
  if (S.err) {
    set_err("line search exceeded its iteration bound");
    return PFGPU_ERR_STATE;
  }
  const int ret = S.kinsol_status;
  return (ret == 1 || ret == 2) ? PFGPU_OK : PFGPU_NOT_CONVERGED;
}

static int newton(pfgpu_handle *h, double dt, pfgpu_stats *stats) {
  h->nk.used_last = false;
  if (nk_usable(h)) {
    const int rc = nk_prepare(h);
    if (rc == PFGPU_OK) {
      h->nk.used_last = true;
      return newton_graph(h, dt, stats);
    }
    // the solve runs host-driven from now on; the reason stays readable
    // through pfgpu_last_error until the next failing call
    h->nk.failed = true;
  }
  const int m = ph_begin(h);
  const int rc = newton_impl(h, dt, stats);
  ph_end(h, m, PH_NEWTON);
  ph_collect(h);
  return rc;
}

// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------
template <typename T>
static int alloc_mg(pfgpu_handle *h, MG<T> &mg) {
  double DX = h->d.dx, DY = h->d.dy, DZ = h->d.dz;
  int NX = h->nx, NY = h->ny, NZ = h->nz;
  // smallest size that is coarsened per direction (mg_semi.c:869-872)
  int minN[3];
  for (int q = 0; q < 3; q++)
    minN[q] = std::max(2 * std::max(h->d.mg_max_min_n[q], 1) - 1, 2);
  int max_levels = h->d.mg_max_levels > 0 ? h->d.mg_max_levels : 100;
  std::vector<int> dirs;
  // coarsening directions (mg_semi.c:858-923)
  for (int l = 0; l < max_levels - 1; l++) {
    double ms = DX + DY + DZ;
    int dd = -1;
    if ((NX >= minN[0]) && (DX < ms)) { ms = DX; dd = 0; }
    if ((NY >= minN[1]) && (DY < ms)) { ms = DY; dd = 1; }
    if ((NZ >= minN[2]) && (DZ < ms)) { ms = DZ; dd = 2; }
    if (dd == -1) break;
    if (dd == 0) { DX *= 2; NX = (NX + 1) / 2; }
    if (dd == 1) { DY *= 2; NY = (NY + 1) / 2; }
    if (dd == 2) { DZ *= 2; NZ = (NZ + 1) / 2; }
    dirs.push_back(dd);
  }
  int nl = (int)dirs.size() + 1;
  mg.L.resize(nl);
  int nx = h->nx, ny = h->ny, nz = h->nz;
  for (int l = 0; l < nl; l++) {
    MGLevel<T> &L = mg.L[l];
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.n = (long long)nx * ny * nz;
    L.dir = l < nl - 1 ? dirs[l] : -1;
    L.hx = (nx + 1) / 2;
    for (int s = 0; s < 4; s++)
      if (dalloc(&L.a[s], L.n)) return PFGPU_ERR_NOMEM;
    // x and b sized for the colour-split layout too (one slot more per row of
    // the shorter colour when nx is odd)
    const long long nxb = std::max(L.n, 2LL * L.hx * ny * nz);
    if (dalloc(&L.x, nxb) || dalloc(&L.b, nxb) || dalloc(&L.t, L.n)) return PFGPU_ERR_NOMEM;
    if (dalloc(&L.wg, (long long)ny * nz)) return PFGPU_ERR_NOMEM;
    CK(cudaMemset(L.wg, 0, (long long)ny * nz * sizeof(T)));
    if (l < nl - 1) {
      if (dalloc(&L.p1, L.n) || dalloc(&L.p2, L.n)) return PFGPU_ERR_NOMEM;
      CK(cudaMemset(L.p1, 0, L.n * sizeof(T)));
      CK(cudaMemset(L.p2, 0, L.n * sizeof(T)));
    }
    CK(cudaMemset(L.x, 0, L.n * sizeof(T)));
    if (mg.h16) {
      // FP16 arrays padded so that whole 32-bit words can be copied
      if (!mg.hflag) {
        CK(cudaMalloc((void **)&mg.hflag, sizeof(int)));
        CK(cudaMemset(mg.hflag, 0, sizeof(int)));
      }
      L.hflag = mg.hflag;
      for (int s = 0; s < 4; s++) {
        if (dalloc(&L.h[s], L.n + 8)) return PFGPU_ERR_NOMEM;
        CK(cudaMemset(L.h[s], 0, (L.n + 8) * sizeof(__half)));
      }
      if (l < nl - 1 && (dalloc(&L.q1, L.n) || dalloc(&L.q2, L.n))) return PFGPU_ERR_NOMEM;
      if (l == 0 && dalloc(&L.sinv, L.n)) return PFGPU_ERR_NOMEM;
    }
    if (L.dir == 0) nx = (nx + 1) / 2;
    if (L.dir == 1) ny = (ny + 1) / 2;
    if (L.dir == 2) nz = (nz + 1) / 2;
  }
  if (dalloc(&mg.wtmp, mg.L[0].n)) return PFGPU_ERR_NOMEM;
  // first level of the single-block tail: the largest whose tail fits in
  // shared memory (else the coarsest level alone, run from global memory)
  mg.tail = nl - 1;
  const long long tail_cells = env_ll("PFGPU_TAIL_CELLS", 1024);
  for (int l = 0; l < nl; l++)
    if (mg.L[l].n <= tail_cells && tail_smem_bytes<T>(mg.L.data(), l, nl, mg.h16) <= TAIL_SMEM_MAX) {
      mg.tail = l;
      break;
    }
  {
    const size_t b = tail_smem_bytes<T>(mg.L.data(), mg.tail, nl, mg.h16);
    mg.tail_smem = b <= TAIL_SMEM_MAX && env_ll("PFGPU_TAIL_SMEM", 1) ? b : 0;
  }
  mg.flip = env_ll("PFGPU_FLIP", 1) != 0;
  // middle levels: the grid levels at or below PFGPU_MID_CELLS cells just
  // above the tail, when the device can co-schedule a cluster for them
  mg.mid = mg.tail;
  {
    const long long mid_cells = env_ll("PFGPU_MID_CELLS", 0);
    int l = mg.tail;
    while (mid_cells > 0 && l > 1 && mg.L[l - 1].n <= mid_cells) l--;
    if (l < mg.tail) {
      int cs = vcycle_mid_cluster_size<T>(mg.h16, mg.tail_smem);
      const int cap = (int)env_ll("PFGPU_MID_CLUSTER", 16);
      if (cs > cap) cs = cap;
      if (cs >= 2) {
        mg.mid = l;
        mg.mid_cs = cs;
      }
    }
  }
  // else the grid levels at or below PFGPU_GRID_CELLS cells just above the
  // tail, on cooperative kernels over the whole GPU (one launch per V-cycle
  // leg instead of one per phase: these levels are bound by launch latency)
  if (mg.mid == mg.tail) {
    const long long grid_cells = env_ll("PFGPU_GRID_CELLS", 0);
    int l = mg.tail;
    while (grid_cells > 0 && l > 1 && mg.L[l - 1].n <= grid_cells) l--;
    if (l < mg.tail) {
      const int blocks = vcycle_grid_blocks<T>(mg.h16, (int)env_ll("PFGPU_GRID_PER_SM", 1));
      if (blocks > 0) {
        CK(cudaMalloc((void **)&mg.gbar, 2 * sizeof(unsigned)));
        CK(cudaMemset(mg.gbar, 0, 2 * sizeof(unsigned)));
        mg.mid = l;
        mg.grid_blocks = blocks;
      }
    }
  }
  // colour-split x / b on the grid levels (red/black smoother); the tail
  // levels keep the natural layout
  const bool split = (h->d.mg_smoother == PFGPU_SMOOTH_RBGS ||
                      h->d.mg_smoother == PFGPU_SMOOTH_RBGS_NONSYM) &&
                     env_ll("PFGPU_SPLIT", 1) != 0;
  for (int l = 0; l < nl; l++) mg.L[l].split = split && l < mg.mid ? 1 : 0;
  // grid levels large enough for the fused smoother get an output buffer
  // distinct from the input iterate
  const long long fused_cells = env_ll("PFGPU_RBR_FUSED_CELLS", LLONG_MAX);
  mg.fused.assign(nl, 0);
  mg.maps.resize(nl);
  for (int l = 0; l < mg.mid; l++) {
    MGLevel<T> &L = mg.L[l];
    if (mg.h16 || L.split || h->d.mg_smoother != PFGPU_SMOOTH_RBGS || L.n < fused_cells ||
        !rbr_fused_eligible(L))
      continue;
    if (dalloc(&L.x2, L.n)) return PFGPU_ERR_NOMEM;
    CK(cudaMemset(L.x2, 0, L.n * sizeof(T)));
    if (make_rbr_maps<T>(L, L.x, &mg.maps[l]) != 0) {
      set_err("tensor map creation failed for multigrid level %d", l);
      return PFGPU_ERR_CUDA;
    }
    mg.fused[l] = 1;
  }
  // grid levels large enough for the wavefront smoother (not the fused one)
  const long long wave_cells = env_ll("PFGPU_WAVE_CELLS", LLONG_MAX);
  const int wave_ctas = (int)env_ll("PFGPU_WAVE_CTAS", 0);
  const int wave_lag = (int)env_ll("PFGPU_WAVE_LAG", 8);
  const int wave_chunk = (int)env_ll("PFGPU_WAVE_CHUNK", 2048);
  mg.waved.assign(nl, 0);
  mg.wave.resize(nl);
  for (int l = 0; l < mg.mid; l++) {
    if (mg.h16 || mg.L[l].split || h->d.mg_smoother != PFGPU_SMOOTH_RBGS || mg.fused[l] ||
        mg.L[l].n < wave_cells)
      continue;
    if (wave_setup<T>(mg.L[l], wave_ctas, wave_lag, wave_chunk, &mg.wave[l]) != 0) {
      set_err("wavefront smoother setup failed for multigrid level %d", l);
      return PFGPU_ERR_CUDA;
    }
    mg.waved[l] = 1;
  }
  // the residual after the pre-smoother: the colour swept last is solved
  // against its current neighbours, its residual zero up to rounding
  // (PFGPU_PAIR_RESIDUAL=0 computes it anyway)
  const bool pair = env_ll("PFGPU_PAIR_RESIDUAL", 1) != 0;
  for (int l = 0; l < nl; l++) {
    const int sm = h->d.mg_smoother;
    // (the fused and wavefront smoothers run the same red/black/red sweeps)
    mg.L[l].zc = !pair                           ? -1
                 : sm == PFGPU_SMOOTH_RBGS        ? 0
                 : sm == PFGPU_SMOOTH_RBGS_NONSYM ? 1
                                                  : -1;
  }
  mg.kerr = h->kerr;
  CK(cudaMalloc((void **)&mg.Ldev, nl * sizeof(MGLevel<T>)));
  CK(cudaMemcpy(mg.Ldev, mg.L.data(), nl * sizeof(MGLevel<T>), cudaMemcpyHostToDevice));
  h->nlev = nl;
  return 0;
}

// The finest level on the per-phase grid kernels with the plain colour
// sweeps: out of the single-block tail and cluster kernels and of the fused /
// wavefront smoothers (FullJacobian's non-symmetric operator; MGSemi.MaxIter
// cycles after the first, whose pre-smoothing reads the current iterate)
template <typename T>
static int mg_level0_on_grid(pfgpu_handle *h, MG<T> &mg) {
  const int nl = (int)mg.L.size();
  MGLevel<T> &L0 = mg.L[0];
  if (nl > 1) {
    if (mg.tail < 1) {
      mg.tail = 1;
      const size_t b = tail_smem_bytes<T>(mg.L.data(), 1, nl, mg.h16);
      mg.tail_smem = b <= TAIL_SMEM_MAX && env_ll("PFGPU_TAIL_SMEM", 1) ? b : 0;
    }
    if (mg.mid < 1) mg.mid = 1;
  }
  mg.fused[0] = 0;
  mg.waved[0] = 0;
  L0.split = (h->d.mg_smoother == PFGPU_SMOOTH_RBGS ||
              h->d.mg_smoother == PFGPU_SMOOTH_RBGS_NONSYM) &&
             env_ll("PFGPU_SPLIT", 1) != 0 && nl > 1;
  CK(cudaMemcpy(mg.Ldev, mg.L.data(), nl * sizeof(MGLevel<T>), cudaMemcpyHostToDevice));
  return PFGPU_OK;
}

// FullJacobian storage for a hierarchy: W S L on level 0, the S / L ghost
// planes on every level, level 0 taken out of the fused / wavefront smoothers
// and the single-block kernels (their kernels assume a symmetric operator)
template <typename T>
static int mg_enable_full(pfgpu_handle *h, MG<T> &mg) {
  const int nl = (int)mg.L.size();
  MGLevel<T> &L0 = mg.L[0];
  if (!L0.lo[0])
    for (int s = 0; s < 3; s++)
      if (dalloc(&L0.lo[s], L0.n)) return PFGPU_ERR_NOMEM;
  for (int l = 0; l < nl; l++) {
    MGLevel<T> &L = mg.L[l];
    if (!L.sg && (dalloc(&L.sg, (long long)L.nx * L.nz) || dalloc(&L.lg, (long long)L.nx * L.ny)))
      return PFGPU_ERR_NOMEM;
    CK(cudaMemset(L.sg, 0, (long long)L.nx * L.nz * sizeof(T)));
    CK(cudaMemset(L.lg, 0, (long long)L.nx * L.ny * sizeof(T)));
  }
  L0.zc = -1;
  return mg_level0_on_grid(h, mg);
}
template <typename T>
static int mg_disable_full(MG<T> &mg) {
  MGLevel<T> &L0 = mg.L[0];
  for (int s = 0; s < 3; s++) {
    cudaFree(L0.lo[s]);
    L0.lo[s] = nullptr;
  }
  CK(cudaMemcpy(mg.Ldev, mg.L.data(), mg.L.size() * sizeof(MGLevel<T>),
                cudaMemcpyHostToDevice));
  return PFGPU_OK;
}

template <typename T>
static void free_mg(MG<T> &mg) {
  for (auto &L : mg.L) {
    for (int s = 0; s < 4; s++) cudaFree(L.a[s]);
    cudaFree(L.x); cudaFree(L.b); cudaFree(L.t); cudaFree(L.p1); cudaFree(L.p2);
    cudaFree(L.x2); cudaFree(L.wg);
    for (int s = 0; s < 3; s++) cudaFree(L.lo[s]);
    cudaFree(L.sg); cudaFree(L.lg);
    for (int s = 0; s < 4; s++) cudaFree(L.h[s]);
    cudaFree(L.q1); cudaFree(L.q2); cudaFree(L.sinv);
  }
  cudaFree(mg.wtmp);
  cudaFree(mg.Ldev);
  for (auto &w : mg.wave) wave_free(&w);
  cudaFree(mg.hflag);
  mg.hflag = nullptr;
  cudaFree(mg.gbar);
  mg.gbar = nullptr;
  mg.wave.clear();
  mg.L.clear();
}

static int create_impl(pfgpu_handle *h) {
  const pfgpu_desc &d = h->d;
  const long long N = h->N;
  CK(cudaSetDevice(h->device));
  CK(mg_prepare_kernels());
  CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  double **vecs[] = {&h->kx, &h->u, &h->unew, &h->fval, &h->pp, &h->bb, &h->p_old,
                     &h->s_old, &h->kr, &h->dkr, &h->sat, &h->dsat, &h->xcor, &h->vtemp};
  for (double **v : vecs)
    if (dalloc(v, N)) return PFGPU_ERR_NOMEM;
  h->ky = h->kx;
  h->kz = h->kx;
  if (dalloc(&h->zmult, h->nz)) return PFGPU_ERR_NOMEM;
  std::vector<double> zm(h->nz, 1.0);
  if (d.z_mult)
    for (int k = 0; k < h->nz; k++) zm[k] = d.z_mult[k];
  CK(cudaMemcpy(h->zmult, zm.data(), h->nz * sizeof(double), cudaMemcpyHostToDevice));
  // per z face constants: 1/(dz mean(z_k, z_k+1)), z_k/(z_k+z_k+1), z_k+1/(z_k+z_k+1)
  std::vector<double> zf(3 * (size_t)h->nz, 0.0);
  for (int k = 0; k + 1 < h->nz; k++) {
    double za = zm[k], zb = zm[k + 1];
    zf[3 * k] = 1.0 / (d.dz * (0.5 * (za + zb)));
    zf[3 * k + 1] = za / (za + zb);
    zf[3 * k + 2] = zb / (za + zb);
  }
  if (dalloc(&h->zface, 3 * h->nz)) return PFGPU_ERR_NOMEM;
  CK(cudaMemcpy(h->zface, zf.data(), zf.size() * sizeof(double), cudaMemcpyHostToDevice));
  for (int f = 0; f < 6; f++) {
    long long fs = f < 2 ? (long long)h->nz * h->ny : f < 4 ? (long long)h->nz * h->nx
                                                           : (long long)h->ny * h->nx;
    if (dalloc(&h->bcv[f], fs)) return PFGPU_ERR_NOMEM;
    CK(cudaMemset(h->bcv[f], 0, fs * sizeof(double)));
  }
  h->V.resize(d.krylov_dim + 1);
  for (auto &v : h->V)
    if (dalloc(&v, N)) return PFGPU_ERR_NOMEM;
  if (h->zbasis) {
    h->Z.resize(d.krylov_dim);
    for (auto &v : h->Z)
      if (dalloc(&v, N)) return PFGPU_ERR_NOMEM;
  }
  if (dalloc(&h->gs, gs_size(d.krylov_dim)) || dalloc(&h->dsc, 64) ||
      dalloc(&h->stage, h->NP) || dalloc(&h->rb.partial, reduce_partials()))
    return PFGPU_ERR_NOMEM;
  CK(cudaMemset(h->gs, 0, gs_size(d.krylov_dim) * sizeof(double)));
  CK(cudaMalloc((void **)&h->rb.ticket, sizeof(unsigned int)));
  CK(cudaMemset(h->rb.ticket, 0, sizeof(unsigned int)));
  h->rb.blocks = reduce_blocks();
  CK(cudaMallocHost((void **)&h->hsc, 64 * sizeof(double)));
  CK(cudaMalloc((void **)&h->kerr, sizeof(int)));
  CK(cudaMemset(h->kerr, 0, sizeof(int)));
  CK(cudaMallocHost((void **)&h->hkerr, sizeof(int)));
  *h->hkerr = 0;

  // Jacobian storage
  if (h->mixed) {
    float **J[] = {&h->Jf.c, &h->Jf.w, &h->Jf.e, &h->Jf.s, &h->Jf.n, &h->Jf.l, &h->Jf.u};
    for (float **a : J)
      if (dalloc(a, N)) return PFGPU_ERR_NOMEM;
    h->mgf.h16 = h->h16;
    if (int rc = alloc_mg<float>(h, h->mgf)) return rc;
  } else {
    double **J[] = {&h->Jd.c, &h->Jd.w, &h->Jd.e, &h->Jd.s, &h->Jd.n, &h->Jd.l, &h->Jd.u};
    for (double **a : J)
      if (dalloc(a, N)) return PFGPU_ERR_NOMEM;
    if (int rc = alloc_mg<double>(h, h->mgd)) return rc;
  }
  CK(cudaMemsetAsync(h->u, 0, N * sizeof(double), h->st));
  // device problem
  DevProblem &P = h->P;
  memset(&P, 0, sizeof(P));
  P.nx = h->nx; P.ny = h->ny; P.nz = h->nz; P.n = N;
  P.dx = d.dx; P.dy = d.dy; P.dz = d.dz;
  P.gravity = d.gravity; P.viscosity = d.viscosity; P.density = d.density;
  P.porosity = d.porosity; P.sstorage = d.specific_storage;
  P.alpha0 = d.vg_alpha; P.vgn0 = d.vg_n; P.sres0 = d.s_res; P.ssat0 = d.s_sat;
  P.vg_from_file = d.vg_from_file;
  P.kx = h->kx; P.ky = h->ky; P.kz = h->kz;
  P.zmult = h->zmult;
  P.zface = h->zface;
  P.ov_pold = h->p_old;
  P.inv_dx = 1.0 / d.dx;
  P.inv_dy = 1.0 / d.dy;
  P.inv_visc = 1.0 / d.viscosity;
  for (int f = 0; f < 6; f++) {
    P.bc_type[f] = PFGPU_BC_FLUX;
    P.bc_val[f] = h->bcv[f];
  }
  if (build_vgraph(h)) return PFGPU_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// ---------------------------------------------------------------------------
// Ensemble timesteps as one graph launch.  Every member's step (dt in, old
// state, the whole Newton solve with its own device-side control, the control
// state back to pinned memory) is a root branch of one graph, so one launch
// advances all members and each converges on its own.  A member whose solve
// fails is retried host-side with the halved dt, as pfgpu_advance does.
// Graphs are kept per member set (named by the handles' uids) and rebuilt
// when a member's captured solve no longer matches it.
// ---------------------------------------------------------------------------
namespace {
struct EnsembleGraph {
  std::vector<unsigned long long> uids;
  std::vector<std::vector<unsigned char>> keys;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t st = nullptr;
  int device = 0;
};
std::mutex g_ens_mu;
std::vector<EnsembleGraph *> g_ens;
std::atomic<unsigned long long> g_uid{1};

void ens_free(EnsembleGraph *E) {
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(E->device);
  if (E->exec) cudaGraphExecDestroy(E->exec);
  if (E->st) cudaStreamDestroy(E->st);
  cudaSetDevice(cur);
  delete E;
}
}  // namespace

// drops every ensemble graph that holds the handle
static void ens_forget(unsigned long long uid) {
  std::lock_guard<std::mutex> lk(g_ens_mu);
  for (size_t i = 0; i < g_ens.size();) {
    const auto &u = g_ens[i]->uids;
    if (std::find(u.begin(), u.end(), uid) != u.end()) {
      ens_free(g_ens[i]);
      g_ens.erase(g_ens.begin() + (long)i);
    } else {
      i++;
    }
  }
}

static int ens_build(pfgpu_handle *const *members, int n, EnsembleGraph *E) {
  // the members' own graphs keep their launch counts whatever happens here
  std::vector<std::array<long long, NKB_COUNT>> counts(n);
  for (int m = 0; m < n; m++)
    std::copy(std::begin(members[m]->nk.kernels), std::end(members[m]->nk.kernels),
              counts[m].begin());
  auto restore = [&]() {
    for (int m = 0; m < n; m++)
      std::copy(counts[m].begin(), counts[m].end(), std::begin(members[m]->nk.kernels));
  };
  for (int attempt = 0; attempt < 2; attempt++) {
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    pdl_capture_off() = attempt == 1;
    int rc = 0;
    for (int m = 0; m < n && !rc; m++) rc = nk_capture_guarded(members[m], nullptr, g);
    pdl_capture_off() = false;
    if (!rc && cudaGraphInstantiate(&E->exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      E->exec = nullptr;
      rc = PFGPU_ERR_CUDA;
      set_err("ensemble graph: instantiation failed");
    }
    cudaGraphDestroy(g);
    if (!rc) {
      restore();
      CK(cudaGraphUpload(E->exec, E->st));
      return 0;
    }
    if (attempt == 1) {
      restore();
      return rc;
    }
  }
  restore();
  return PFGPU_ERR_CUDA;
}

namespace pfgpu {
int ensemble_graph_advance(pfgpu_handle *const *members, int n, const double *dt, int nsteps,
                           pfgpu_stats *stats, int *status, bool *handled);
}
int pfgpu::ensemble_graph_advance(pfgpu_handle *const *members, int n, const double *dt,
                                  int nsteps, pfgpu_stats *stats, int *status, bool *handled) {
  *handled = false;
  static const bool on = env_ll("PFGPU_ENSEMBLE_GRAPH", 1) != 0;
  if (!on || n < 1) return PFGPU_OK;
  const int dev = members[0]->device;
  for (int m = 0; m < n; m++) {
    pfgpu_handle *h = members[m];
    if (!nk_usable(h) || h->recording || h->device != dev) return PFGPU_OK;
    for (int q = 0; q < m; q++)
      if (members[q] == h) return PFGPU_OK;
  }
  CK(cudaSetDevice(dev));
  for (int m = 0; m < n; m++)
    if (nk_prepare(members[m]) != PFGPU_OK) return PFGPU_OK;  // the per-member path decides
  std::vector<unsigned long long> uids(n);
  std::vector<std::vector<unsigned char>> keys(n);
  for (int m = 0; m < n; m++) {
    uids[m] = members[m]->uid;
    keys[m] = nk_key(members[m]);
  }
  EnsembleGraph *E = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ens_mu);
    for (size_t i = 0; i < g_ens.size(); i++)
      if (g_ens[i]->uids == uids) {
        E = g_ens[i];
        g_ens.erase(g_ens.begin() + (long)i);
        break;
      }
  }
  if (E && E->keys != keys) {
    ens_free(E);
    E = nullptr;
  }
  if (!E) {
    E = new EnsembleGraph();
    E->uids = uids;
    E->keys = keys;
    E->device = dev;
    if (cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking) != cudaSuccess ||
        ens_build(members, n, E) != 0) {
      cudaGetLastError();
      ens_free(E);
      return PFGPU_OK;  // not handled: the per-member path runs
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_ens_mu);
    g_ens.push_back(E);
  }
  *handled = true;
  for (int m = 0; m < n; m++) status[m] = PFGPU_OK;
  static const double limit = (double)env_ll("PFGPU_SOLVE_TIMEOUT_S", 600);
  std::vector<char> done(n, 0);  // member stopped (failed step or error)
  bool all = true;               // every member still in the graph
  for (int s = 0; s < nsteps; s++) {
    if (!all) {
      // a member stopped: the rest finish on the per-member path
      for (int m = 0; m < n; m++) {
        if (done[m]) continue;
        pfgpu_stats st{};
        const int rc = pfgpu_advance(members[m], dt[m], 1, &st);
        if (stats) stats[(size_t)m * nsteps + s] = st;
        if (rc != PFGPU_OK) {
          status[m] = rc;
          done[m] = 1;
        }
      }
      continue;
    }
    for (int m = 0; m < n; m++) {
      *members[m]->nk.hdt = dt[m];
      CK(cudaStreamSynchronize(members[m]->st));  // the member's earlier work
    }
    CK(cudaGraphLaunch(E->exec, E->st));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t q = cudaStreamQuery(E->st);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) CK(q);
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit) {
        set_err("ensemble graph did not finish within %.0f s", limit);
        return PFGPU_ERR_STATE;
      }
      std::this_thread::yield();
    }
    for (int m = 0; m < n; m++) {
      pfgpu_handle *h = members[m];
      const NkState &S = *h->nk.hS;
      long long k = 1;  // the saturation of the step's start
      for (int b = 0; b < NKB_COUNT; b++) k += h->nk.kernels[b] * (long long)S.execs[b];
      h->launches += k;
      h->vg_for = nullptr;
      h->jac_valid = 0;
      h->nk.used_last = true;
      pfgpu_stats st{};
      st.nonlin_iters = S.nonlin_iters;
      st.lin_iters = S.lin_iters;
      st.fevals = S.fevals;
      st.pc_setups = S.pc_setups;
      st.pc_solves = S.pc_solves;
      st.lin_conv_fails = S.lin_conv_fails;
      st.beta_cond_fails = S.beta_cond_fails;
      st.backtracks = S.backtracks;
      st.kinsol_status = S.kinsol_status;
      st.fnorm = S.fnorm;
      int rc = S.err ? PFGPU_ERR_STATE
                     : (S.kinsol_status == 1 || S.kinsol_status == 2) ? PFGPU_OK
                                                                      : PFGPU_NOT_CONVERGED;
      if (S.err) set_err("line search exceeded its iteration bound");
      if (rc >= 0 && *h->hkerr) rc = check_kernel_error(h) ? PFGPU_ERR_CUDA : rc;
      // failed solves: the retries of pfgpu_advance (u back to p_old, dt halved)
      // as pfgpu_advance: after every failed attempt u goes back to p_old
      // and dt is halved; at most three attempts
      double dts = dt[m];
      for (int fail = 1; rc == PFGPU_NOT_CONVERGED; fail++) {
        CK(cudaMemcpyAsync(h->u, h->p_old, h->N * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->st));
        h->vg_for = nullptr;
        dts *= 0.5;
        if (fail == 3) break;
        rc = newton(h, dts, &st);
        if (rc >= 0 && check_kernel_error(h)) rc = PFGPU_ERR_CUDA;
      }
      if (stats) stats[(size_t)m * nsteps + s] = st;
      if (rc == PFGPU_NOT_CONVERGED)
        set_err("pfgpu_advance: time step %d failed after 3 convergence failures", s);
      if (rc != PFGPU_OK) {
        status[m] = rc;
        done[m] = 1;
        all = false;
      }
    }
  }
  for (int m = 0; m < n; m++) CK(cudaStreamSynchronize(members[m]->st));
  int rc = PFGPU_OK;
  for (int m = 0; m < n; m++) {
    if (status[m] == PFGPU_OK) continue;
    if (status[m] < 0 && rc >= 0) rc = status[m];
    else if (rc == PFGPU_OK) rc = PFGPU_NOT_CONVERGED;
  }
  return rc;
}

static void destroy_impl(pfgpu_handle *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  ens_forget(h->uid);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->ptime && h->pcnt[PH_NEWTON] > 0) {
    fprintf(stderr, "pfgpu phase times (%lldx%lldx%lld, %s): device ms summed over %lld solves\n",
            (long long)h->nx, (long long)h->ny, (long long)h->nz, h->mixed ? "mixed" : "fp64",
            h->pcnt[PH_NEWTON]);
    for (int q = 0; q < PH_COUNT; q++)
      fprintf(stderr, "  %-40s %10.3f ms  %6lld calls  %8.4f ms/call\n", kPhaseName[q],
              h->pacc[q], h->pcnt[q], h->pcnt[q] ? h->pacc[q] / h->pcnt[q] : 0.0);
  }
  for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
  cudaFree(h->dq_w);
  cudaFree(h->dq_f);
  cudaFree(h->krt);
  cudaFree(h->et);
  cudaFree(h->vel);
  cudaFree(h->vstage);
  if (h->vgraph) cudaGraphExecDestroy(h->vgraph);
  if (h->nk.exec) cudaGraphExecDestroy(h->nk.exec);
  for (auto &kv : h->nk.kept) cudaGraphExecDestroy(kv.exec);
  cudaFree(h->nk.S);
  cudaFree(h->nk.dt);
  if (h->nk.hS) cudaFreeHost(h->nk.hS);
  if (h->nk.hdt) cudaFreeHost(h->nk.hdt);
  for (cudaStream_t s : h->nk.cs)
    if (s) cudaStreamDestroy(s);
  cudaFree(h->hist);
  cudaFree(h->adj);
  double *vecs[] = {h->u, h->unew, h->fval, h->pp, h->bb, h->p_old, h->s_old, h->kr,
                    h->dkr, h->sat, h->dsat, h->xcor, h->vtemp, h->gs, h->dsc, h->stage,
                    h->rb.partial, h->zmult, h->zface, h->alpha, h->vgn, h->sres, h->ssat,
                    h->surf};
  for (double *v : vecs) cudaFree(v);
  if (h->kx) cudaFree(h->kx);
  if (h->ky && h->ky != h->kx) cudaFree(h->ky);
  if (h->kz && h->kz != h->kx && h->kz != h->ky) cudaFree(h->kz);
  for (int f = 0; f < 6; f++) cudaFree(h->bcv[f]);
  for (double *f : h->fb) cudaFree(f);
  for (int f = 0; f < 6; f++) cudaFree(h->cyc[f].table);
  for (auto v : h->V) cudaFree(v);
  for (auto v : h->Z) cudaFree(v);
  cudaFree(h->rb.ticket);
  cudaFree(h->kerr);
  if (h->hkerr) cudaFreeHost(h->hkerr);

  double *jd[] = {h->Jd.c, h->Jd.w, h->Jd.e, h->Jd.s, h->Jd.n, h->Jd.l, h->Jd.u};
  for (double *a : jd) cudaFree(a);
  float *jf[] = {h->Jf.c, h->Jf.w, h->Jf.e, h->Jf.s, h->Jf.n, h->Jf.l, h->Jf.u};
  for (float *a : jf) cudaFree(a);
  free_mg(h->mgd);
  free_mg(h->mgf);
  if (h->hsc) cudaFreeHost(h->hsc);
  if (h->st) cudaStreamDestroy(h->st);
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *pfgpu_last_error(void) { return g_err; }

pfgpu_handle *pfgpu_create(const pfgpu_desc *desc, int device) {
  if (!desc || desc->abi_version != PFGPU_ABI_VERSION) {
    set_err("pfgpu_create: null descriptor or ABI version mismatch");
    return nullptr;
  }
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1 ||
      (long long)desc->nx * desc->ny * desc->nz < 2) {
    set_err("pfgpu_create: grid must hold at least two cells");
    return nullptr;
  }
  // the multigrid kernels index cells in 32 bits (a grid this large would
  // need far more than one device's memory anyway)
  if ((long long)desc->nx * desc->ny * desc->nz >= (1LL << 31)) {
    set_err("pfgpu_create: grid must hold fewer than 2^31 cells");
    return nullptr;
  }
  if (desc->krylov_dim < 1 || desc->krylov_dim > NK_MAX_KRYLOV) {
    set_err("pfgpu_create: krylov_dim must be in [1, %d]", NK_MAX_KRYLOV);
    return nullptr;
  }
  if (desc->max_restarts < 0) {
    set_err("pfgpu_create: max_restarts must not be negative");
    return nullptr;
  }
  if (desc->mg_smoother != PFGPU_SMOOTH_RBGS && desc->mg_smoother != PFGPU_SMOOTH_WJACOBI &&
      desc->mg_smoother != PFGPU_SMOOTH_RBGS_NONSYM) {
    set_err("pfgpu_create: unknown multigrid smoother %d", desc->mg_smoother);
    return nullptr;
  }
  if (desc->precision != PFGPU_PREC_FP64 && desc->precision != PFGPU_PREC_MIXED &&
      desc->precision != PFGPU_PREC_MIXED_H16) {
    set_err("pfgpu_create: unknown precision %d", desc->precision);
    return nullptr;
  }
  if (!(desc->dx > 0 && desc->dy > 0 && desc->dz > 0 && desc->density > 0 &&
        desc->gravity > 0 && desc->viscosity > 0)) {
    set_err("pfgpu_create: spacings, density, gravity and viscosity must be positive");
    return nullptr;
  }
  pfgpu_handle *h = new pfgpu_handle();
  h->uid = g_uid.fetch_add(1);
  h->d = *desc;
  h->d.z_mult = nullptr;
  h->device = device;
  h->nx = desc->nx; h->ny = desc->ny; h->nz = desc->nz;
  h->N = (long long)h->nx * h->ny * h->nz;
  h->NP = (long long)(h->nx + 2) * (h->ny + 2) * (h->nz + 2);
  h->mixed = desc->precision == PFGPU_PREC_MIXED || desc->precision == PFGPU_PREC_MIXED_H16;
  h->h16 = desc->precision == PFGPU_PREC_MIXED_H16;
  h->ptime = env_ll("PFGPU_PHASE_TIMES", 0) != 0;
  h->nk.enabled = env_ll("PFGPU_SOLVE_GRAPH", 1) != 0;
  {
    // PFGPU_PC_BASIS: 0 never keeps the preconditioned basis, 1 (default) in
    // the mixed forms, 2 in every form
    const long long zb = env_ll("PFGPU_PC_BASIS", 1);
    h->zbasis = zb >= 2 || (zb == 1 && h->mixed);
  }
  if (create_impl(h) != 0) {
    destroy_impl(h);
    delete h;
    return nullptr;
  }
  return h;
}

void pfgpu_destroy(pfgpu_handle *h) {
  destroy_impl(h);
  delete h;
}

int pfgpu_set_field(pfgpu_handle *h, int field, const double *values) {
  if (!h) { set_err("pfgpu_set_field: null handle"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (field >= PFGPU_FIELD_FB_X && field <= PFGPU_FIELD_FB_Z) {
    double *&fb = h->fb[field - PFGPU_FIELD_FB_X];
    if (!values) {
      CK(cudaStreamSynchronize(h->st));
      cudaFree(fb);
      fb = nullptr;
    } else {
      if (!fb && dalloc(&fb, h->N)) return PFGPU_ERR_NOMEM;
      if (in_vec(h, values, fb)) return PFGPU_ERR_CUDA;
      CK(cudaStreamSynchronize(h->st));
    }
    h->P.fbx = h->fb[0];
    h->P.fby = h->fb[1];
    h->P.fbz = h->fb[2];
    return PFGPU_OK;
  }
  if (!values) {
    // drop a per-cell van Genuchten array: the descriptor scalar serves again
    double **vg = field == PFGPU_FIELD_VG_ALPHA ? &h->alpha
                  : field == PFGPU_FIELD_VG_N   ? &h->vgn
                  : field == PFGPU_FIELD_S_RES  ? &h->sres
                  : field == PFGPU_FIELD_S_SAT  ? &h->ssat
                                                : nullptr;
    if (!vg) {
      set_err("pfgpu_set_field: values may be null only for van Genuchten fields");
      return PFGPU_ERR_ARG;
    }
    CK(cudaStreamSynchronize(h->st));
    cudaFree(*vg);
    *vg = nullptr;
    DevProblem &P = h->P;
    P.alpha = h->alpha; P.vgn = h->vgn; P.sres = h->sres; P.ssat = h->ssat;
    h->vg_for = nullptr;  // cached van Genuchten state is stale
    return PFGPU_OK;
  }
  double **dst = nullptr;
  switch (field) {
    case PFGPU_FIELD_PERM_X: dst = &h->kx; break;
    case PFGPU_FIELD_PERM_Y:
      if (h->ky == h->kx && dalloc(&h->ky, h->N)) return PFGPU_ERR_NOMEM;
      dst = &h->ky;
      break;
    case PFGPU_FIELD_PERM_Z:
      if ((h->kz == h->kx || h->kz == h->ky) && dalloc(&h->kz, h->N)) return PFGPU_ERR_NOMEM;
      dst = &h->kz;
      break;
    case PFGPU_FIELD_VG_ALPHA: dst = &h->alpha; break;
    case PFGPU_FIELD_VG_N: dst = &h->vgn; break;
    case PFGPU_FIELD_S_RES: dst = &h->sres; break;
    case PFGPU_FIELD_S_SAT: dst = &h->ssat; break;
    default: set_err("pfgpu_set_field: unknown field %d", field); return PFGPU_ERR_ARG;
  }
  if (!*dst && dalloc(dst, h->N)) return PFGPU_ERR_NOMEM;
  if (in_vec(h, values, *dst)) return PFGPU_ERR_CUDA;
  // a permeability set only in x serves all three directions
  if (field == PFGPU_FIELD_PERM_X) {
    if (h->ky == h->kx) h->ky = h->kx;
    if (h->kz == h->kx) h->kz = h->kx;
  }
  DevProblem &P = h->P;
  P.kx = h->kx; P.ky = h->ky; P.kz = h->kz;
  P.alpha = h->alpha; P.vgn = h->vgn; P.sres = h->sres; P.ssat = h->ssat;
  h->vg_for = nullptr;  // cached van Genuchten state is stale
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

// ---------------------------------------------------------------------------
// PFB files (write_parflow_binary.c:74-205, read_parflow_binary.c:38-120)
// ---------------------------------------------------------------------------
namespace {
void put_be64(FILE *f, double v) {
  unsigned long long u;
  memcpy(&u, &v, 8);
  unsigned char b[8];
  for (int q = 0; q < 8; q++) b[q] = (unsigned char)(u >> (56 - 8 * q));
  fwrite(b, 1, 8, f);
}
void put_be32(FILE *f, int v) {
  const unsigned u = (unsigned)v;
  unsigned char b[4] = {(unsigned char)(u >> 24), (unsigned char)(u >> 16),
                        (unsigned char)(u >> 8), (unsigned char)u};
  fwrite(b, 1, 4, f);
}
bool get_be64(FILE *f, double *v) {
  unsigned char b[8];
  if (fread(b, 1, 8, f) != 8) return false;
  unsigned long long u = 0;
  for (int q = 0; q < 8; q++) u = (u << 8) | b[q];
  memcpy(v, &u, 8);
  return true;
}
bool get_be32(FILE *f, int *v) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return false;
  *v = (int)(((unsigned)b[0] << 24) | ((unsigned)b[1] << 16) | ((unsigned)b[2] << 8) | b[3]);
  return true;
}
}  // namespace

int pfgpu_write_pfb(pfgpu_handle *h, int what, const char *path, double x0, double y0,
                    double z0) {
  if (!h || !path) { set_err("pfgpu_write_pfb: null argument"); return PFGPU_ERR_ARG; }
  if (what != PFGPU_PFB_PRESSURE && what != PFGPU_PFB_SATURATION) {
    set_err("pfgpu_write_pfb: unknown field %d", what);
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  const double *src = h->u;
  if (what == PFGPU_PFB_SATURATION) {
    launch_saturation(h->P, h->u, h->vtemp, h->st);
    src = h->vtemp;
    h->launches++;
  }
  // big-endian values in the staging buffer (NP >= N doubles), one copy out
  unsigned long long *raw = reinterpret_cast<unsigned long long *>(h->stage);
  launch_pfb_pack(src, raw, h->N, h->st);
  h->launches++;
  std::vector<unsigned long long> host((size_t)h->N);
  CK(cudaMemcpyAsync(host.data(), raw, h->N * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  FILE *f = fopen(path, "wb");
  if (!f) { set_err("pfgpu_write_pfb: cannot open %s", path); return PFGPU_ERR_ARG; }
  put_be64(f, x0); put_be64(f, y0); put_be64(f, z0);
  put_be32(f, h->nx); put_be32(f, h->ny); put_be32(f, h->nz);
  put_be64(f, h->d.dx); put_be64(f, h->d.dy); put_be64(f, h->d.dz);
  put_be32(f, 1);
  const int box[9] = {0, 0, 0, h->nx, h->ny, h->nz, 0, 0, 0};
  for (int v : box) put_be32(f, v);
  const size_t w = fwrite(host.data(), sizeof(double), host.size(), f);
  const bool ok = fclose(f) == 0 && w == host.size();
  if (!ok) { set_err("pfgpu_write_pfb: short write to %s", path); return PFGPU_ERR_ARG; }
  return PFGPU_OK;
}

int pfgpu_read_pfb(pfgpu_handle *h, int what, const char *path) {
  if (!h || !path) { set_err("pfgpu_read_pfb: null argument"); return PFGPU_ERR_ARG; }
  if (what != PFGPU_PFB_PRESSURE && (what < PFGPU_FIELD_PERM_X || what > PFGPU_FIELD_FB_Z)) {
    set_err("pfgpu_read_pfb: unknown field %d", what);
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  FILE *f = fopen(path, "rb");
  if (!f) { set_err("pfgpu_read_pfb: cannot open %s", path); return PFGPU_ERR_ARG; }
  double hdr_d[6];
  int nx = 0, ny = 0, nz = 0, nsg = 0;
  bool ok = get_be64(f, hdr_d) && get_be64(f, hdr_d + 1) && get_be64(f, hdr_d + 2) &&
            get_be32(f, &nx) && get_be32(f, &ny) && get_be32(f, &nz) &&
            get_be64(f, hdr_d + 3) && get_be64(f, hdr_d + 4) && get_be64(f, hdr_d + 5) &&
            get_be32(f, &nsg);
  if (!ok || nx != h->nx || ny != h->ny || nz != h->nz || nsg < 1) {
    fclose(f);
    set_err("pfgpu_read_pfb: %s is not a PFB file of a %dx%dx%d grid", path, h->nx, h->ny,
            h->nz);
    return PFGPU_ERR_ARG;
  }
  // dense field assembled in vtemp (free outside a solve); raw bytes staged
  // in the staging buffer (NP >= N doubles) one subgrid at a time
  CK(cudaMemsetAsync(h->vtemp, 0, h->N * sizeof(double), h->st));
  unsigned long long *raw = reinterpret_cast<unsigned long long *>(h->stage);
  std::vector<unsigned long long> host;
  for (int g = 0; g < nsg; g++) {
    int box[9];
    for (int q = 0; q < 9 && ok; q++) ok = get_be32(f, box + q);
    const int ix = box[0], iy = box[1], iz = box[2], snx = box[3], sny = box[4], snz = box[5];
    if (!ok || ix < 0 || iy < 0 || iz < 0 || snx < 0 || sny < 0 || snz < 0 ||
        ix + snx > nx || iy + sny > ny || iz + snz > nz) {
      fclose(f);
      set_err("pfgpu_read_pfb: subgrid %d of %s lies outside the grid", g, path);
      return PFGPU_ERR_ARG;
    }
    const size_t cnt = (size_t)snx * sny * snz;
    if (cnt == 0) continue;
    CK(cudaStreamSynchronize(h->st));  // the staging buffer is free again
    host.resize(cnt);
    if (fread(host.data(), sizeof(double), cnt, f) != cnt) {
      fclose(f);
      set_err("pfgpu_read_pfb: %s ends inside subgrid %d", path, g);
      return PFGPU_ERR_ARG;
    }
    CK(cudaMemcpyAsync(raw, host.data(), cnt * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_pfb_scatter(raw, h->vtemp, nx, ny, ix, iy, iz, snx, sny, snz, h->st);
    h->launches++;
  }
  fclose(f);
  if (what == PFGPU_PFB_PRESSURE) {
    CK(cudaMemcpyAsync(h->u, h->vtemp, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    if (h->vg_for == h->u) h->vg_for = nullptr;
    CK(cudaStreamSynchronize(h->st));
    return PFGPU_OK;
  }
  // a cell field: through pfgpu_set_field in ParFlow layout (device pointer)
  launch_pad(h->vtemp, h->stage, h->nx, h->ny, h->nz, h->st);
  h->launches++;
  return pfgpu_set_field(h, what, h->stage);
}

int pfgpu_set_surface(pfgpu_handle *h, const double *slope_x, const double *slope_y,
                      const double *mannings, int terrain_following, double ov_epsilon) {
  if (!h || !slope_x || !slope_y || !mannings || !(ov_epsilon > 0)) {
    set_err("pfgpu_set_surface: bad argument");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  const int nx = h->nx, ny = h->ny;
  const size_t n2 = (size_t)nx * ny;
  // interior of ParFlow's 2-D subvector layout: (i+1) + (j+1)*(nx+2)
  std::vector<double> col(7 * n2);
  const double g = h->d.gravity;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      const size_t a = i + (size_t)nx * j, q = (i + 1) + (size_t)(nx + 2) * (j + 1);
      const double sx = slope_x[q], sy = slope_y[q];
      col[a] = g * sin(atan(sx));
      col[n2 + a] = g * cos(atan(sx));
      col[2 * n2 + a] = g * sin(atan(sy));
      col[3 * n2 + a] = g * cos(atan(sy));
      col[4 * n2 + a] = sx;
      col[5 * n2 + a] = sy;
      col[6 * n2 + a] = mannings[q];
    }
  if (!h->surf && dalloc(&h->surf, 7 * n2)) return PFGPU_ERR_NOMEM;
  CK(cudaMemcpy(h->surf, col.data(), col.size() * sizeof(double), cudaMemcpyHostToDevice));
  DevProblem &P = h->P;
  if (terrain_following) {
    P.tfg_xs = h->surf;
    P.tfg_xc = h->surf + n2;
    P.tfg_ys = h->surf + 2 * n2;
    P.tfg_yc = h->surf + 3 * n2;
  } else {
    P.tfg_xs = P.tfg_xc = P.tfg_ys = P.tfg_yc = nullptr;
  }
  P.ov_sx = h->surf + 4 * n2;
  P.ov_sy = h->surf + 5 * n2;
  P.ov_n = h->surf + 6 * n2;
  P.ov_eps = ov_epsilon;
  h->vg_for = nullptr;
  return PFGPU_OK;
}

int pfgpu_set_bc(pfgpu_handle *h, int face, int type, const double *values) {
  if (!h || !values || face < 0 || face > 5 ||
      (type != PFGPU_BC_FLUX && type != PFGPU_BC_DIRICHLET && type != PFGPU_BC_OVERLAND_KIN &&
       type != PFGPU_BC_OVERLAND_DIFF && type != PFGPU_BC_OVERLAND && type != PFGPU_BC_SEEPAGE)) {
    set_err("pfgpu_set_bc: bad argument");
    return PFGPU_ERR_ARG;
  }
  if ((type == PFGPU_BC_OVERLAND_KIN || type == PFGPU_BC_OVERLAND_DIFF ||
       type == PFGPU_BC_OVERLAND) &&
      (face != PFGPU_Z_UPPER || !h->P.ov_sx)) {
    set_err("pfgpu_set_bc: overland flow needs face z_upper and pfgpu_set_surface first");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  long long fs = face < 2 ? (long long)h->nz * h->ny : face < 4 ? (long long)h->nz * h->nx
                                                               : (long long)h->ny * h->nx;
  CK(cudaMemcpyAsync(h->bcv[face], values, fs * sizeof(double), cudaMemcpyDefault, h->st));
  h->P.bc_type[face] = type;
  h->P.bc_val[face] = h->bcv[face];
  h->cyc[face].nint = 0;  // a fixed table replaces a time cycle
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

// ---------------------------------------------------------------------------
// Time cycles, time step selection and the native time loop
// ---------------------------------------------------------------------------
namespace {
const int kTimeCycleSubdivisions = 1000;   // time_cycle_data.c:190
const double kTimeEpsilon = FLT_EPSILON * 10.0;  // general.h:257
int pf_round(double x) { return x < 0.0 ? (int)(x - 0.5) : (int)(x + 0.5); }  // general.h:176

// interval of the cycle at time t (TimeCycleDataComputeIntervalNumber,
// time_cycle_data.c:160-199)
int cycle_interval(const pfgpu_handle::BcCycle &c, double t) {
  if (c.repeat < 0 || t < (double)(c.repeat * c.cycle_len * c.base_unit)) {
    const int dtime = pf_round(t / (c.base_unit / kTimeCycleSubdivisions)) / kTimeCycleSubdivisions;
    const int dstart =
        pf_round(c.start_time / (c.base_unit / kTimeCycleSubdivisions)) / kTimeCycleSubdivisions;
    const int done = (dtime - dstart - 1) % c.cycle_len;
    int n = 0, total = c.lengths[0];
    while (done >= total && n + 1 < c.nint) total += c.lengths[++n];
    return n;
  }
  return c.nint - 1;
}

// time to the next interval transition of any cycle, or -1
// (TimeCycleDataComputeNextTransition, time_cycle_data.c:206-297)
double next_transition(const pfgpu_handle *h, double t) {
  double dt = -1.0;
  bool assigned = false;
  for (int f = 0; f < 6; f++) {
    const auto &c = h->cyc[f];
    if (c.nint <= 1) continue;
    const double stop_defined =
        c.repeat > 0 ? (double)(c.repeat * c.cycle_len * c.base_unit) : 1e300;
    if (!(t < stop_defined)) continue;
    const int dtime = pf_round(t / (c.base_unit / kTimeCycleSubdivisions)) / kTimeCycleSubdivisions;
    const int dstart =
        pf_round(c.start_time / (c.base_unit / kTimeCycleSubdivisions)) / kTimeCycleSubdivisions;
    int n = (dtime - dstart) / c.cycle_len;
    const int done = (dtime - dstart - 1) % c.cycle_len;
    int q = 0, total = c.lengths[0];
    while (done >= total && q + 1 < c.nint) total += c.lengths[++q];
    double tt;
    if ((q + 1) % c.nint == 0) {
      n++;
      tt = c.start_time + (double)(n * c.cycle_len) * c.base_unit;
    } else {
      tt = c.start_time + (double)(n * c.cycle_len + total) * c.base_unit;
    }
    if (tt < stop_defined) {
      dt = assigned ? std::min(dt, tt - t) : tt - t;
      assigned = true;
    }
  }
  if (assigned && !((t + dt) - t > kTimeEpsilon)) dt = -1.0;
  return dt;
}
}  // namespace

int pfgpu_set_bc_cycle(pfgpu_handle *h, int face, int nint, const int *types,
                       const double *values, const int *lengths, int repeat, double base_unit,
                       double start_time) {
  if (!h || face < 0 || face > 5 || nint < 1 || !types || !values || !lengths ||
      !(base_unit > 0)) {
    set_err("pfgpu_set_bc_cycle: bad argument");
    return PFGPU_ERR_ARG;
  }
  int len = 0;
  for (int q = 0; q < nint; q++) {
    const int t = types[q];
    const bool ovl =
        t == PFGPU_BC_OVERLAND_KIN || t == PFGPU_BC_OVERLAND_DIFF || t == PFGPU_BC_OVERLAND;
    if ((t != PFGPU_BC_FLUX && t != PFGPU_BC_DIRICHLET && t != PFGPU_BC_SEEPAGE && !ovl) ||
        lengths[q] < 1 ||
        (ovl && (face != PFGPU_Z_UPPER || !h->P.ov_sx))) {
      set_err("pfgpu_set_bc_cycle: bad type or length in interval %d", q);
      return PFGPU_ERR_ARG;
    }
    len += lengths[q];
  }
  CK(cudaSetDevice(h->device));
  auto &c = h->cyc[face];
  c.face_cells = face < 2 ? (long long)h->nz * h->ny : face < 4 ? (long long)h->nz * h->nx
                                                                : (long long)h->ny * h->nx;
  cudaFree(c.table);
  c.table = nullptr;
  if (dalloc(&c.table, c.face_cells * nint)) return PFGPU_ERR_NOMEM;
  CK(cudaMemcpyAsync(c.table, values, c.face_cells * nint * sizeof(double), cudaMemcpyDefault,
                     h->st));
  c.nint = nint;
  c.repeat = repeat;
  c.cycle_len = len;
  c.lengths.assign(lengths, lengths + nint);
  c.types.assign(types, types + nint);
  c.base_unit = base_unit;
  c.start_time = start_time;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

int pfgpu_set_time_step(pfgpu_handle *h, int type, double step, double factor,
                        double min_step, double max_step, int max_failures) {
  if (!h || (type != 0 && type != 1) || !(step > 0) || max_failures < 1 ||
      (type == 1 && !(factor > 0 && min_step > 0 && max_step >= min_step))) {
    set_err("pfgpu_set_time_step: bad argument");
    return PFGPU_ERR_ARG;
  }
  h->ts_type = type;
  h->ts_step = step;
  h->ts_factor = factor;
  h->ts_min = min_step;
  h->ts_max = max_step;
  h->max_failures = max_failures;
  return PFGPU_OK;
}

// point every cycled face at its interval's table for time t
static void bc_cycles_at(pfgpu_handle *h, double t) {
  for (int f = 0; f < 6; f++) {
    const auto &c = h->cyc[f];
    if (c.nint < 1) continue;
    const int q = cycle_interval(c, t);
    h->P.bc_type[f] = c.types[q];
    h->P.bc_val[f] = c.table + q * c.face_cells;
  }
}

// SelectTimeStep (select_time_step.c:58-155) on the running dt: constant
// steps, or growth of the previous dt (dt == 0, only before the loop: the
// initial step) clamped to [min, max]; then cut to the next boundary-cycle
// transition
static double select_time_step(pfgpu_handle *h, double t, double dt) {
  if (h->ts_type == 0) {
    dt = h->ts_step;
  } else if (dt == 0.0) {
    dt = h->ts_step;
  } else {
    dt = dt * h->ts_factor;
    if (dt < h->ts_min) dt = h->ts_min;
    if (dt > h->ts_max) dt = h->ts_max;
  }
  const double bc_dt = next_transition(h, t);
  if (bc_dt > 0.0 && dt > bc_dt) dt = bc_dt;
  return dt;
}

// AdvanceRichards's time loop on the device state, with its control flow
// (solver_richards.c:2075-2090 before the loop, 2965-3410 per step, 3700-3720
// after a step): one time-step selection before the loop (the initial step),
// then per step a selection on the running dt (so growth first multiplies
// the initial step, and multiplies the dt that cuts, halvings and dump
// snapping left), the dump-time snap and the stop-time cut on every attempt,
// the solve, and on failure t and the state put back and dt halved; the dump
// index advances once per converged step that dumped.
int pfgpu_run(pfgpu_handle *h, double t, double stop_time, double dump_interval, int max_steps,
              double *times, double *dts, pfgpu_stats *stats, int *nsteps) {
  if (!h || !(stop_time > t) || max_steps < 1 || !nsteps || !(h->ts_step > 0)) {
    set_err("pfgpu_run: bad argument (set the time step first)");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  const double start = t;
  double dump_index = 1.0;
  int n = 0;
  *nsteps = 0;
  double dt = select_time_step(h, t, 0.0);
  while (t < stop_time && n < max_steps) {
    bool converged = true, dump_files = false;
    int failures = 0;
    pfgpu_stats st{};
    int rc = PFGPU_NOT_CONVERGED;
    do {
      if (converged) {
        dt = select_time_step(h, t, dt);
        CK(cudaMemcpyAsync(h->p_old, h->u, h->N * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->st));
        launch_saturation(h->P, h->u, h->s_old, h->st);
        h->launches++;
      } else {
        t -= dt;
        const double half = 0.5 * dt;
        if (!((t + half) - t > kTimeEpsilon)) {
          set_err("pfgpu_run: time increment too small at t = %g; the solver has failed", t);
          *nsteps = n;
          return PFGPU_NOT_CONVERGED;
        }
        dt = half;
        CK(cudaMemcpyAsync(h->u, h->p_old, h->N * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->st));
        h->vg_for = nullptr;
      }
      dump_files = false;
      if (dump_interval > 0) {
        const double print_dt = start + dump_index * dump_interval - t;
        if ((dt + kTimeEpsilon) > print_dt) {
          if (fabs(dt - print_dt) > kTimeEpsilon) dt = print_dt;
          dump_files = true;
        }
      }
      if (t + dt >= stop_time) {
        const double last = stop_time - t;
        if ((t + last) - t > kTimeEpsilon) dt = last;
      }
      t += dt;
      bc_cycles_at(h, t);
      rc = newton(h, dt, &st);
      if (rc < 0) { *nsteps = n; return rc; }
      if (check_kernel_error(h)) { *nsteps = n; return PFGPU_ERR_CUDA; }
      converged = rc == PFGPU_OK;
      if (!converged) failures++;
    } while (!converged && failures < h->max_failures);
    if (!converged) {
      set_err("pfgpu_run: time step at t = %g failed %d times", t, failures);
      *nsteps = n;
      return PFGPU_NOT_CONVERGED;
    }
    if (dump_files) dump_index += 1.0;
    if (times) times[n] = t;
    if (dts) dts[n] = dt;
    if (stats) stats[n] = st;
    n++;
  }
  *nsteps = n;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

int pfgpu_saturation(pfgpu_handle *h, const double *p, double *s) {
  if (!h || !p || !s) { set_err("pfgpu_saturation: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p, h->unew)) return PFGPU_ERR_CUDA;
  launch_saturation(h->P, h->unew, h->fval, h->st);
  h->launches++;
  return out_vec(h, h->fval, s);
}

int pfgpu_nl_function_eval(pfgpu_handle *h, const double *p, const double *p_old,
                           const double *s_old, double dt, double *f) {
  if (!h || !p || !p_old || !s_old || !f) {
    set_err("pfgpu_nl_function_eval: null argument");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p, h->unew) || in_vec(h, p_old, h->p_old) || in_vec(h, s_old, h->s_old))
    return PFGPU_ERR_CUDA;
  feval(h, h->unew, dt, h->fval);
  return out_vec(h, h->fval, f);
}

int pfgpu_set_evap_trans(pfgpu_handle *h, const double *et) {
  if (!h) { set_err("pfgpu_set_evap_trans: null handle"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (!et) {
    h->P.et = nullptr;
    return PFGPU_OK;
  }
  if (!h->et && dalloc(&h->et, h->N)) return PFGPU_ERR_NOMEM;
  if (in_vec(h, et, h->et)) return PFGPU_ERR_CUDA;
  h->P.et = h->et;
  return PFGPU_OK;
}

int pfgpu_face_velocities(pfgpu_handle *h, const double *p, const double *p_old,
                          const double *s_old, double dt, double *vx, double *vy, double *vz,
                          double *qx, double *qy) {
  if (!h) { set_err("pfgpu_face_velocities: null handle"); return PFGPU_ERR_ARG; }
  if (!(dt > 0.0)) { set_err("pfgpu_face_velocities: dt must be positive"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  const long long nx = h->nx, ny = h->ny, nz = h->nz;
  const long long nvx = (nx + 1) * ny * nz, nvy = nx * (ny + 1) * nz, nvz = nx * ny * (nz + 1);
  const long long nq = nx * ny;
  if (!h->vel) {
    const long long pad_max = std::max({(nx + 3) * (ny + 2) * (nz + 2),
                                        (nx + 2) * (ny + 3) * (nz + 2),
                                        (nx + 4) * (ny + 4) * (nz + 5)});
    if (dalloc(&h->vel, nvx + nvy + nvz + 2 * nq) || dalloc(&h->vstage, pad_max))
      return PFGPU_ERR_NOMEM;
  }
  VelOut V{h->vel, h->vel + nvx, h->vel + nvx + nvy, h->vel + nvx + nvy + nvz,
           h->vel + nvx + nvy + nvz + nq};
  // the overland fluxes exist only on an overland z_upper face: zero elsewhere
  CK(cudaMemsetAsync(V.qx, 0, 2 * nq * sizeof(double), h->st));
  const double *u = h->u;
  if (p) {
    if (in_vec(h, p, h->unew)) return PFGPU_ERR_CUDA;
    u = h->unew;
  }
  if ((p_old && in_vec(h, p_old, h->p_old)) || (s_old && in_vec(h, s_old, h->s_old)))
    return PFGPU_ERR_CUDA;
  h->P.ov_pold = h->p_old;
  vg_state(h, u, false);
  launch_residual(h->P, u, h->p_old, h->s_old, h->kr, h->sat, dt, h->bb, h->st, &V);
  h->launches++;
  CK(cudaGetLastError());
  // ParFlow layouts: the face grids grown by one along their axis
  // (x_grid / y_grid / z_grid, solver_richards.c:5110-5160) with the ghost
  // widths of the state vectors (one for x and y, two for z,
  // solver_richards.c:1035-1045); q on the 2-D grid, one plane, one ghost
  struct Out {
    const double *src;
    double *dst;
    int ax, ay, az, g;
  } outs[5] = {{V.vx, vx, (int)nx + 1, (int)ny, (int)nz, 1},
               {V.vy, vy, (int)nx, (int)ny + 1, (int)nz, 1},
               {V.vz, vz, (int)nx, (int)ny, (int)nz + 1, 2},
               {V.qx, qx, (int)nx, (int)ny, 1, 1},
               {V.qy, qy, (int)nx, (int)ny, 1, 1}};
  for (const Out &o : outs) {
    if (!o.dst) continue;
    const long long np =
        (long long)(o.ax + 2 * o.g) * (o.ay + 2 * o.g) * (o.az + 2 * o.g);
    if (is_device_ptr(o.dst)) {
      launch_pad_ghost(o.src, o.dst, o.ax, o.ay, o.az, o.g, h->st);
      h->launches++;
    } else {
      launch_pad_ghost(o.src, h->vstage, o.ax, o.ay, o.az, o.g, h->st);
      h->launches++;
      CK(cudaMemcpyAsync(o.dst, h->vstage, np * sizeof(double), cudaMemcpyDeviceToHost, h->st));
      CK(cudaStreamSynchronize(h->st));
    }
  }
  CK(cudaGetLastError());
  return PFGPU_OK;
}

int pfgpu_jacobian_matvec(pfgpu_handle *h, const double *p, double dt, const double *x,
                          double *y) {
  if (!h || !p || !x || !y) { set_err("pfgpu_jacobian_matvec: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p, h->unew) || in_vec(h, x, h->vtemp)) return PFGPU_ERR_CUDA;
  assemble(h, h->unew, dt, true, false);
  h->jac_valid = 0;
  matvec(h, h->vtemp, h->bb);
  return out_vec(h, h->bb, y);
}

int pfgpu_pc_setup(pfgpu_handle *h, const double *p, double dt) {
  if (!h || !p) { set_err("pfgpu_pc_setup: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p, h->unew)) return PFGPU_ERR_CUDA;
  pc_setup_dense(h, h->unew, dt, false);
  h->jac_valid = 0;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

// VanGComputeTable (problem_phase_rel_perm.c:116-262): kr and dkr/dhead at
// npts + 1 heads 0, |min_head| / (npts - 1), ..., the linear slopes and the
// monotone cubic Hermite slopes (Fritsch and Carlson 1980); t holds x a d
// a_der d_der slope slope_der, npts + 1 values each
static void vg_table(int linear, int npts, double min_head, double alpha, double n,
                     std::vector<double> &t, double *interval_out) {
  const int m1 = npts + 1;
  t.assign(7 * (size_t)m1, 0.0);
  double *x = t.data(), *a = x + m1, *d = x + 2 * m1, *a_der = x + 3 * m1, *d_der = x + 4 * m1,
         *slope = x + 5 * m1, *slope_der = x + 6 * m1;
  const double interval = min_head / (double)(npts - 1);
  const double ival = fabs(interval);
  *interval_out = ival;
  const double m = 1.0e0 - (1.0e0 / n);
  for (int i = 0; i <= npts; i++) {
    x[i] = fabs(i * interval);
    const double opahn = 1.0 + pow(alpha * x[i], n);
    const double ahnm1 = pow(alpha * x[i], n - 1);
    a[i] = pow(1.0 - ahnm1 / (pow(opahn, m)), 2) / pow(opahn, (m / 2));
    const double coeff = 1.0 - ahnm1 * pow(opahn, -m);
    a_der[i] = 2.0 * (coeff / (pow(opahn, (m / 2)))) *
                   ((n - 1) * pow(alpha * x[i], n - 2) * alpha * pow(opahn, -m) -
                    ahnm1 * m * pow(opahn, -(m + 1)) * n * alpha * ahnm1) +
               pow(coeff, 2) * (m / 2) * pow(opahn, (-(m + 2) / 2)) * n * alpha * ahnm1;
    if ((n < 2) && (i == 0)) a_der[i] = 0;
  }
  if (linear)
    for (int i = 0; i < npts; i++) {
      slope[i] = (a[i + 1] - a[i]) / ival;
      slope_der[i] = (a_der[i + 1] - a_der[i]) / ival;
    }
  std::vector<double> del(m1, 0.0), del_der(m1, 0.0);
  for (int i = 0; i < npts; i++) {
    const double hh = x[i + 1] - x[i];
    del[i] = (a[i + 1] - a[i]) / hh;
    del_der[i] = (a_der[i + 1] - a_der[i]) / hh;
  }
  d[0] = del[0];
  d[npts] = del[npts - 1];
  d_der[0] = del_der[0];
  d_der[npts] = del_der[npts - 1];
  for (int i = 1; i < npts; i++) {
    d[i] = (del[i - 1] + del[i]) / 2;
    d_der[i] = (del_der[i - 1] + del_der[i]) / 2;
  }
  auto limit = [&](double *dd, const double *dl, int i) {
    if (dl[i] == 0.0) {
      dd[i] = 0;
      dd[i + 1] = 0;
    } else {
      const double alph = dd[i] / dl[i], beta = dd[i + 1] / dl[i];
      const double magn = pow(alph, 2) + pow(beta, 2);
      if (magn > 9.0) {
        dd[i] = 3 * alph * dl[i] / magn;
        dd[i + 1] = 3 * beta * dl[i] / magn;
      }
    }
  };
  for (int i = 0; i < npts; i++) {
    limit(d, del.data(), i);
    limit(d_der, del_der.data(), i);
  }
}

int pfgpu_set_relperm_table(pfgpu_handle *h, int method, int num_sample_points,
                            double min_pressure_head) {
  if (!h || method < PFGPU_KRT_NONE || method > PFGPU_KRT_LINEAR ||
      (method != PFGPU_KRT_NONE && (num_sample_points < 2 || !(min_pressure_head < 0.0)))) {
    set_err("pfgpu_set_relperm_table: bad argument");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  if (method == PFGPU_KRT_NONE) {
    h->P.krt = nullptr;
    h->vg_for = nullptr;
    return PFGPU_OK;
  }
  if (h->d.vg_from_file || h->P.alpha || h->P.vgn) {
    set_err("pfgpu_set_relperm_table: the table needs uniform van Genuchten alpha and n");
    return PFGPU_ERR_STATE;
  }
  std::vector<double> t;
  double interval = 0.0;
  vg_table(method == PFGPU_KRT_LINEAR, num_sample_points, min_pressure_head, h->d.vg_alpha,
           h->d.vg_n, t, &interval);
  cudaFree(h->krt);
  h->krt = nullptr;
  if (dalloc(&h->krt, (long long)t.size())) return PFGPU_ERR_NOMEM;
  CK(cudaMemcpy(h->krt, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
  h->P.krt = h->krt;
  h->P.krt_method = method == PFGPU_KRT_LINEAR ? 1 : 0;
  h->P.krt_npts = num_sample_points;
  h->P.krt_interval = interval;
  h->P.krt_min = min_pressure_head;
  h->vg_for = nullptr;  // cached van Genuchten state is stale
  return PFGPU_OK;
}

int pfgpu_set_jacobian_mode(pfgpu_handle *h, int use_jacobian, double derivative_epsilon) {
  if (!h || (use_jacobian != 0 && use_jacobian != 1) || derivative_epsilon < 0.0) {
    set_err("pfgpu_set_jacobian_mode: bad argument");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  if (!use_jacobian && (!h->dq_w || !h->dq_f)) {
    if (dalloc(&h->dq_w, h->N) || dalloc(&h->dq_f, h->N)) return PFGPU_ERR_NOMEM;
  }
  h->use_jacobian = use_jacobian;
  // sqrt_relfunc (kinsol.c:516-531): sqrt of DerivativeEpsilon, or of the
  // unit roundoff when it is 0
  h->sqrt_relfunc = sqrt(derivative_epsilon > 0.0 ? derivative_epsilon : DBL_EPSILON);
  h->jac_valid = 0;
  return PFGPU_OK;
}

int pfgpu_set_old_pressure(pfgpu_handle *h, const double *p_old) {
  if (!h || !p_old) { set_err("pfgpu_set_old_pressure: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p_old, h->p_old)) return PFGPU_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

int pfgpu_pc_apply(pfgpu_handle *h, const double *r, double *z) {
  if (!h || !r || !z) { set_err("pfgpu_pc_apply: null argument"); return PFGPU_ERR_ARG; }
  if (!h->pc_ready) { set_err("pfgpu_pc_apply: call pfgpu_pc_setup first"); return PFGPU_ERR_STATE; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, r, h->vtemp)) return PFGPU_ERR_CUDA;
  if (pc_apply_dense(h, h->vtemp, h->vtemp)) return PFGPU_ERR_CUDA;
  if (check_kernel_error(h)) return PFGPU_ERR_CUDA;
  return out_vec(h, h->vtemp, z);
}

// the three inputs of a step; an initial guess passed in the same buffer as
// the old pressure (as at the start of every AdvanceRichards step) is copied
// in once
static int load_step_inputs(pfgpu_handle *h, const double *p_old, const double *s_old,
                            const double *p) {
  if (in_vec(h, p_old, h->p_old) || in_vec(h, s_old, h->s_old)) return PFGPU_ERR_CUDA;
  if (p == p_old) {
    CK(cudaMemcpyAsync(h->u, h->p_old, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    if (h->vg_for == h->u) h->vg_for = nullptr;
    return 0;
  }
  return in_vec(h, p, h->u);
}

int pfgpu_newton_solve(pfgpu_handle *h, const double *p_old, const double *s_old, double dt,
                       double *p, pfgpu_stats *stats) {
  if (!h || !p_old || !s_old || !p) { set_err("pfgpu_newton_solve: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (load_step_inputs(h, p_old, s_old, p)) return PFGPU_ERR_CUDA;
  pfgpu_stats local;
  int rc = newton(h, dt, stats ? stats : &local);
  if (rc < 0) return rc;
  if (check_kernel_error(h)) return PFGPU_ERR_CUDA;
  int rc2 = out_vec(h, h->u, p);
  return rc2 ? rc2 : rc;
}

int pfgpu_newton_solve_sat(pfgpu_handle *h, const double *p_old, const double *s_old,
                           double dt, double *p, double *s, pfgpu_stats *stats) {
  if (!h || !p_old || !s_old || !p || !s) {
    set_err("pfgpu_newton_solve_sat: null argument");
    return PFGPU_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  if (load_step_inputs(h, p_old, s_old, p)) return PFGPU_ERR_CUDA;
  pfgpu_stats local;
  int rc = newton(h, dt, stats ? stats : &local);
  if (rc < 0) return rc;
  if (check_kernel_error(h)) return PFGPU_ERR_CUDA;
  launch_saturation(h->P, h->u, h->fval, h->st);
  h->launches++;
  int rc2 = out_vec(h, h->u, p);
  if (!rc2) rc2 = out_vec(h, h->fval, s);
  return rc2 ? rc2 : rc;
}

int pfgpu_solve_graph(pfgpu_handle *h, int mode) {
  if (!h) {
    set_err("pfgpu_solve_graph: null handle");
    return PFGPU_ERR_ARG;
  }
  if (mode == 0 || mode == 1) {
    h->nk.enabled = mode == 1;
    h->nk.failed = false;
    return PFGPU_OK;
  }
  if (mode == -1) return h->nk.used_last ? 1 : 0;
  set_err("pfgpu_solve_graph: mode must be 0, 1 or -1");
  return PFGPU_ERR_ARG;
}

int pfgpu_set_mg_max_iter(pfgpu_handle *h, int max_iter) {
  if (!h || max_iter < 0 || max_iter > 1000) {
    set_err("pfgpu_set_mg_max_iter: max_iter must be in [0, 1000]");
    return PFGPU_ERR_ARG;
  }
  if (max_iter == h->mg_max_iter) return PFGPU_OK;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->st));
  if (max_iter > 1) {
    const int rc = h->mixed ? mg_level0_on_grid<float>(h, h->mgf) : mg_level0_on_grid<double>(h, h->mgd);
    if (rc != PFGPU_OK) return rc;
  }
  h->mg_max_iter = max_iter;
  if (h->vgraph) {
    CK(cudaGraphExecDestroy(h->vgraph));
    h->vgraph = nullptr;
  }
  if (build_vgraph(h)) return PFGPU_ERR_CUDA;
  return PFGPU_OK;
}

int pfgpu_set_pc_matrix(pfgpu_handle *h, int type) {
  if (!h || (type != PFGPU_PCM_SYMMETRIC && type != PFGPU_PCM_FULL)) {
    set_err("pfgpu_set_pc_matrix: type must be PFGPU_PCM_SYMMETRIC or PFGPU_PCM_FULL");
    return PFGPU_ERR_ARG;
  }
  if (type == h->pc_matrix) return PFGPU_OK;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->st));
  int rc;
  if (type == PFGPU_PCM_FULL) {
    if (h->mixed && h->mgf.h16) {
      set_err("PCMatrixType FullJacobian: not available with the scaled FP16 multigrid "
              "(PFGPU_PREC_MIXED_H16)");
      return PFGPU_ERR_ARG;
    }
    if (h->d.mg_smoother == PFGPU_SMOOTH_WJACOBI) {
      set_err("PCMatrixType FullJacobian: not available with the WJacobi smoother");
      return PFGPU_ERR_ARG;
    }
    if (h->nlev < 2) {
      set_err("PCMatrixType FullJacobian: needs at least two multigrid levels");
      return PFGPU_ERR_ARG;
    }
    rc = h->mixed ? mg_enable_full<float>(h, h->mgf) : mg_enable_full<double>(h, h->mgd);
  } else {
    rc = h->mixed ? mg_disable_full<float>(h->mgf) : mg_disable_full<double>(h->mgd);
  }
  if (rc != PFGPU_OK) return rc;
  // the host-driven V-cycle graph holds the old level-0 path
  if (h->vgraph) {
    CK(cudaGraphExecDestroy(h->vgraph));
    h->vgraph = nullptr;
  }
  if (build_vgraph(h)) return PFGPU_ERR_CUDA;
  h->pc_matrix = type;
  h->pc_ready = false;
  h->jac_valid = 0;
  return PFGPU_OK;
}

int pfgpu_set_overland_spinup(pfgpu_handle *h, int spinup, double damp_p1, double damp_p2) {
  if (!h || (spinup != 0 && spinup != 1) || !std::isfinite(damp_p1) || !std::isfinite(damp_p2)) {
    set_err("pfgpu_set_overland_spinup: spinup must be 0 or 1 and the damping finite");
    return PFGPU_ERR_ARG;
  }
  h->P.ov_spinup = spinup;
  h->P.ov_p1 = damp_p1;
  h->P.ov_p2 = damp_p2;
  return PFGPU_OK;
}

int pfgpu_set_globalization(pfgpu_handle *h, int strategy) {
  if (!h || (strategy != PFGPU_GLOBAL_LINE_SEARCH && strategy != PFGPU_GLOBAL_INEXACT_NEWTON)) {
    set_err("pfgpu_set_globalization: strategy must be PFGPU_GLOBAL_LINE_SEARCH or "
            "PFGPU_GLOBAL_INEXACT_NEWTON");
    return PFGPU_ERR_ARG;
  }
  h->globalization = strategy;
  return PFGPU_OK;
}

int pfgpu_set_pressure(pfgpu_handle *h, const double *p) {
  if (!h || !p) { set_err("pfgpu_set_pressure: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  if (in_vec(h, p, h->u)) return PFGPU_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

int pfgpu_get_pressure(pfgpu_handle *h, double *p) {
  if (!h || !p) { set_err("pfgpu_get_pressure: null argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  return out_vec(h, h->u, p);
}

// AdvanceRichards step body (solver_richards.c:2965-3406): old state copies,
// nonlinear solve, dt halving on failure (Solver.MaxConvergenceFailures 3).
int pfgpu_advance(pfgpu_handle *h, double dt, int nsteps, pfgpu_stats *stats) {
  if (!h || nsteps < 0 || !(dt > 0)) { set_err("pfgpu_advance: bad argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  for (int s = 0; s < nsteps; s++) {
    CK(cudaMemcpyAsync(h->p_old, h->u, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    launch_saturation(h->P, h->u, h->s_old, h->st);
    h->launches++;
    double dts = dt;
    int rc = PFGPU_NOT_CONVERGED;
    pfgpu_stats st{};
    for (int fail = 0; fail < 3; fail++) {
      rc = newton(h, dts, &st);
      if (rc < 0) return rc;
      if (check_kernel_error(h)) return PFGPU_ERR_CUDA;
          if (rc == PFGPU_OK) break;
      CK(cudaMemcpyAsync(h->u, h->p_old, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
      h->vg_for = nullptr;
      dts *= 0.5;
    }
    if (stats) stats[s] = st;
    if (rc == PFGPU_OK && h->recording) {
      if (h->hist_len < h->hist_cap) {
        CK(cudaMemcpyAsync(h->hist + (size_t)(h->hist_len + 1) * h->N, h->u,
                           h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
        h->hist_dt.push_back(dts);
        h->hist_len++;
      } else {
        h->hist_overflow = true;
      }
    }
    if (rc != PFGPU_OK) {
      set_err("pfgpu_advance: time step %d failed after 3 convergence failures", s);
      return PFGPU_NOT_CONVERGED;
    }
  }
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

// ---------------------------------------------------------------------------
// Discrete adjoint (no counterpart in the reference)
// ---------------------------------------------------------------------------
int pfgpu_adjoint_record(pfgpu_handle *h, int max_steps) {
  if (!h || max_steps < 1) { set_err("pfgpu_adjoint_record: bad argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->st));
  cudaFree(h->hist);
  h->hist = nullptr;
  if (dalloc(&h->hist, (long long)(max_steps + 1) * h->N)) return PFGPU_ERR_NOMEM;
  CK(cudaMemcpyAsync(h->hist, h->u, h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  h->hist_cap = max_steps;
  h->hist_len = 0;
  h->hist_dt.clear();
  h->hist_overflow = false;
  h->recording = true;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

// J^T lam = rhs by right-preconditioned GMRES (the forward SPGMR on the
// transposed operator, same multigrid preconditioner), restarted on the true
// residual until ||rhs - J^T lam|| <= tol ||rhs||
static int adjoint_solve(pfgpu_handle *h, double *lam, const double *rhs, double *r, double *dx,
                         double tol, const double *u, double dt, int *iters) {
  const long long N = h->N;
  double *sc = h->dsc;
  launch_dot(rhs, rhs, N, sc + D_COUNT, h->rb, h->st);
  if (read_scalars(h, D_COUNT, 1)) return PFGPU_ERR_CUDA;
  const double bnorm = sqrt(h->hsc[D_COUNT]);
  launch_fill(lam, 0.0, N, h->st);
  if (bnorm == 0.0) return 0;
  CK(cudaMemcpyAsync(r, rhs, N * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  h->adj_transpose = true;
  int rc = 0;
  for (int outer = 0; outer < 100; outer++) {
    pfgpu_stats st{};
    int status = 0;
    rc = spgmr(h, dx, r, 1.0, nullptr, -1.0, 0.5 * tol * bnorm, u, dt, &st, &status);
    *iters += st.lin_iters;
    if (rc) break;
    launch_xpay(lam, lam, 1.0, dx, N, h->st);
    matvec(h, lam, dx);
    launch_axpby(r, rhs, 1.0, 0.0, N, h->st);
    launch_xpay(r, r, -1.0, dx, N, h->st);
    launch_dot(r, r, N, sc + D_COUNT, h->rb, h->st);
    h->launches += 4;
    if (read_scalars(h, D_COUNT, 1)) { rc = PFGPU_ERR_CUDA; break; }
    if (sqrt(h->hsc[D_COUNT]) <= tol * bnorm) break;
    if (status == 2 || status == 6) {
      set_err("adjoint GMRES made no progress (status %d)", status);
      rc = PFGPU_NOT_CONVERGED;
      break;
    }
  }
  h->adj_transpose = false;
  return rc;
}

int pfgpu_adjoint_gradient(pfgpu_handle *h, int nobs_steps, const int *obs_steps, int nobs,
                           const long long *obs_cells, const double *obs_values, double tol,
                           double *misfit, double *grad_lnk, double *grad_alpha,
                           double *grad_n) {
  if (!h || nobs_steps < 0 || nobs < 0 || (nobs > 0 && (!obs_cells || !obs_values)) ||
      (nobs_steps > 0 && !obs_steps) || !(tol > 0)) {
    set_err("pfgpu_adjoint_gradient: bad argument");
    return PFGPU_ERR_ARG;
  }
  if (!h->recording || h->hist_len < 1) {
    set_err("pfgpu_adjoint_gradient: no recorded steps (pfgpu_adjoint_record, then pfgpu_advance)");
    return PFGPU_ERR_STATE;
  }
  if (h->P.krt) {
    set_err("pfgpu_adjoint_gradient: not available with a relative-permeability table");
    return PFGPU_ERR_STATE;
  }
  if (h->P.fbx || h->P.fby || h->P.fbz) {
    set_err("pfgpu_adjoint_gradient: not available with flow barriers");
    return PFGPU_ERR_STATE;
  }
  if (h->P.ov_spinup || h->P.ov_p2 != 0.0) {
    set_err("pfgpu_adjoint_gradient: not available with overland spin-up or its damping");
    return PFGPU_ERR_STATE;
  }
  if (h->P.bc_type[5] == PFGPU_BC_OVERLAND_DIFF) {
    // the diffusive terms depend on the old pressure through the slope
    // magnitude; that coupling between steps has no adjoint here
    set_err("pfgpu_adjoint_gradient: not available with a diffusive overland face");
    return PFGPU_ERR_STATE;
  }
  if (h->hist_overflow) {
    set_err("pfgpu_adjoint_gradient: more steps were advanced than recorded");
    return PFGPU_ERR_STATE;
  }
  for (int k = 0; k < nobs_steps; k++)
    if (obs_steps[k] < 1 || obs_steps[k] > h->hist_len) {
      set_err("pfgpu_adjoint_gradient: observation step %d outside 1..%d", obs_steps[k], h->hist_len);
      return PFGPU_ERR_ARG;
    }
  for (int m = 0; m < nobs; m++)
    if (obs_cells[m] < 0 || obs_cells[m] >= h->N) {
      set_err("pfgpu_adjoint_gradient: observation cell out of range");
      return PFGPU_ERR_ARG;
    }
  CK(cudaSetDevice(h->device));
  const long long N = h->N;
  if (!h->adj && dalloc(&h->adj, 8 * N)) return PFGPU_ERR_NOMEM;
  double *lam = h->adj, *lam_next = h->adj + N, *rhs = h->adj + 2 * N, *r = h->adj + 3 * N,
         *dx = h->adj + 4 * N, *g_lnk = h->adj + 5 * N, *g_a = h->adj + 6 * N,
         *g_n = h->adj + 7 * N;
  // observations on the device
  long long *d_cells = nullptr;
  double *d_obs = nullptr, *d_pick = nullptr;
  const size_t nov = (size_t)nobs_steps * nobs;
  if (nobs > 0) {
    CK(cudaMalloc((void **)&d_cells, nobs * sizeof(long long)));
    CK(cudaMalloc((void **)&d_obs, (nov + nobs) * sizeof(double)));
    d_pick = d_obs + nov;
    CK(cudaMemcpy(d_cells, obs_cells, nobs * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_obs, obs_values, nov * sizeof(double), cudaMemcpyHostToDevice));
  }
  launch_fill(lam_next, 0.0, N, h->st);
  launch_fill(g_lnk, 0.0, N, h->st);
  launch_fill(g_a, 0.0, N, h->st);
  launch_fill(g_n, 0.0, N, h->st);
  double J = 0.0;
  int rc = 0, iters = 0;
  std::vector<double> pick(nobs);
  for (int n = h->hist_len; n >= 1 && rc == 0; n--) {
    const double *pn = h->hist + (size_t)n * N, *pprev = h->hist + (size_t)(n - 1) * N;
    const double dt = h->hist_dt[n - 1];
    h->vg_for = nullptr;
    pc_setup_dense(h, pn, dt, true);  // VG state, J and the multigrid at p_n
    launch_adj_rhs(h->P, pn, h->sat, h->dsat, lam_next, rhs, h->st);
    h->launches++;
    for (int k = 0; k < nobs_steps; k++)
      if (obs_steps[k] == n) {
        launch_adj_obs(nobs, d_cells, d_obs + (size_t)k * nobs, pn, rhs, h->st);
        launch_gather(nobs, d_cells, pn, d_pick, h->st);
        h->launches += 2;
        CK(cudaMemcpyAsync(pick.data(), d_pick, nobs * sizeof(double), cudaMemcpyDeviceToHost,
                           h->st));
        CK(cudaStreamSynchronize(h->st));
        for (int m = 0; m < nobs; m++) {
          const double e = pick[m] - obs_values[(size_t)k * nobs + m];
          J += e * e;
        }
      }
    rc = adjoint_solve(h, lam, rhs, r, dx, tol, pn, dt, &iters);
    if (rc) break;
    launch_adj_grad(h->P, pn, pprev, lam, h->kr, dt, g_lnk, g_a, g_n, h->st);
    h->launches++;
    std::swap(lam, lam_next);
  }
  cudaFree(d_cells);
  cudaFree(d_obs);
  h->vg_for = nullptr;
  h->jac_valid = 0;
  if (rc) return rc < 0 ? rc : PFGPU_NOT_CONVERGED;
  if (misfit) *misfit = J;
  if (grad_lnk && out_vec(h, g_lnk, grad_lnk)) return PFGPU_ERR_CUDA;
  if (grad_alpha && out_vec(h, g_a, grad_alpha)) return PFGPU_ERR_CUDA;
  if (grad_n && out_vec(h, g_n, grad_n)) return PFGPU_ERR_CUDA;
  CK(cudaStreamSynchronize(h->st));
  return PFGPU_OK;
}

int pfgpu_mg_levels(pfgpu_handle *h, int *levels, int *dims, int max_levels) {
  if (!h || !levels) { set_err("pfgpu_mg_levels: null argument"); return PFGPU_ERR_ARG; }
  *levels = h->nlev;
  if (dims) {
    for (int l = 0; l < h->nlev && l < max_levels; l++) {
      if (h->mixed) {
        const MGLevel<float> &L = h->mgf.L[l];
        dims[4 * l] = L.nx; dims[4 * l + 1] = L.ny; dims[4 * l + 2] = L.nz; dims[4 * l + 3] = L.dir;
      } else {
        const MGLevel<double> &L = h->mgd.L[l];
        dims[4 * l] = L.nx; dims[4 * l + 1] = L.ny; dims[4 * l + 2] = L.nz; dims[4 * l + 3] = L.dir;
      }
    }
  }
  return PFGPU_OK;
}

// Algorithmic HBM bytes per launch (every per-cell array the operation needs,
// counted once; uniform fields count zero).
static double kernel_bytes(pfgpu_handle *h, int kernel) {
  const double N = (double)h->N;
  const double wJ = h->mixed ? 4.0 : 8.0;
  // multigrid operator bytes per cell: C E N U, or three FP16 off-diagonals
  const double wA = h->h16 ? 6.0 : 4 * wJ;
  // x / b bytes per cell of one colour sweep: b of the swept colour, x of the
  // other colour read and of the swept colour written; with the natural
  // layout every line of b and x is read and x written back
  const bool split0 = h->mixed ? (h->mgf.L.size() && h->mgf.L[0].split)
                               : (h->mgd.L.size() && h->mgd.L[0].split);
  const double wXB = split0 ? 1.5 * wJ : 3 * wJ;
  const double vg = (h->alpha ? 8.0 : 0.0) + (h->vgn ? 8.0 : 0.0) + (h->sres ? 8.0 : 0.0) +
                    (h->ssat ? 8.0 : 0.0);
  const double kf = 8.0 * (1 + (h->ky != h->kx) + (h->kz != h->kx && h->kz != h->ky));
  switch (kernel) {
    case PFGPU_KERNEL_RESIDUAL: return N * (8.0 * 4 + kf + vg);         // p p_old s_old f
    case PFGPU_KERNEL_JACOBIAN: return N * (8.0 + kf + vg + 7 * wJ + 4 * wJ);
    case PFGPU_KERNEL_MATVEC: return N * (7 * wJ + 8.0 + 8.0);
    case PFGPU_KERNEL_RB_SWEEP:                                          // C E N U, b, x in + out
    case PFGPU_KERNEL_COLOUR_SWEEP: return N * (wA + wXB);
    default: return 0.0;
  }
}

int pfgpu_time_kernel(pfgpu_handle *h, int kernel, int reps, double *ms, double *bytes) {
  if (!h || reps < 1 || !ms) { set_err("pfgpu_time_kernel: bad argument"); return PFGPU_ERR_ARG; }
  if (!h->pc_ready) { set_err("pfgpu_time_kernel: no assembled state yet"); return PFGPU_ERR_STATE; }
  CK(cudaSetDevice(h->device));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const double dt = 0.05;
  auto one = [&]() {
    switch (kernel) {
      case PFGPU_KERNEL_RESIDUAL: feval(h, h->u, dt, h->fval); break;
      case PFGPU_KERNEL_JACOBIAN: assemble(h, h->u, dt, true, true); break;
      case PFGPU_KERNEL_MATVEC: matvec(h, h->pp, h->bb); break;
      case PFGPU_KERNEL_RB_SWEEP:  // the finest level's post-smoother as the V-cycle runs it
        if (h->mixed) {
          MG<float> &mg = h->mgf;
          MGLevel<float> &L = mg.L[0];
          if (!mg.fused.empty() && mg.fused[0]) launch_rbr_fused<float>(L, mg.maps[0], L.x2, 0, mg.kerr, h->st);
          else launch_mg_smooth<float>(L, L.x, L.b, 0, 0, 1.0, mg.wtmp, h->st, nullptr, mg.h16);
        } else {
          MG<double> &mg = h->mgd;
          MGLevel<double> &L = mg.L[0];
          if (!mg.fused.empty() && mg.fused[0]) launch_rbr_fused<double>(L, mg.maps[0], L.x2, 0, mg.kerr, h->st);
          else launch_mg_smooth<double>(L, L.x, L.b, 0, 0, 1.0, mg.wtmp, h->st);
        }
        h->launches++;
        break;
      case PFGPU_KERNEL_VCYCLE:
        cudaGraphLaunch(h->vgraph, h->st);
        h->launches += h->graph_nodes;
        break;
      case PFGPU_KERNEL_COLOUR_SWEEP:  // one red sweep of the finest level
        if (h->mixed) {
          MGLevel<float> &L = h->mgf.L[0];
          launch_mg_smooth<float>(L, L.x, L.b, 0, 9, 1.0, h->mgf.wtmp, h->st, nullptr, h->mgf.h16);
        } else {
          MGLevel<double> &L = h->mgd.L[0];
          launch_mg_smooth<double>(L, L.x, L.b, 0, 9, 1.0, h->mgd.wtmp, h->st);
        }
        h->launches++;
        break;
      case PFGPU_KERNEL_MG_SETUP:
        h->launches += h->mixed ? mg_setup_T<float>(h->mgf, h->st) : mg_setup_T<double>(h->mgd, h->st);
        break;
    }
  };
  one();  // warm
  CK(cudaEventRecord(e0, h->st));
  for (int r = 0; r < reps; r++) one();
  CK(cudaEventRecord(e1, h->st));
  CK(cudaEventSynchronize(e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = (double)t / reps;
  if (bytes) *bytes = kernel_bytes(h, kernel);
  if (check_kernel_error(h)) return PFGPU_ERR_CUDA;
  h->jac_valid = 0;
  return PFGPU_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the stencil launches' thread-block shapes
// ---------------------------------------------------------------------------
// Candidate shapes (bx, by): bx a multiple of the warp width, bx * by within
// the kernel's launch bound (256 threads for the residual and the matvec,
// 128 for the Jacobian).  The choice depends on the grid (a block wider than
// nx idles lanes, a narrow one multiplies the blocks) and is cached per grid
// size, precision and kernel variant for the life of the process.
namespace {
struct TuneKey {
  int nx, ny, nz, mixed, surf;
  bool operator<(const TuneKey &o) const {
    return std::tie(nx, ny, nz, mixed, surf) < std::tie(o.nx, o.ny, o.nz, o.mixed, o.surf);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::array<int, 6>> g_tune_cache;
}  // namespace

int pfgpu_autotune(pfgpu_handle *h, int reps, int *shapes) {
  if (!h || reps < 1) { set_err("pfgpu_autotune: bad argument"); return PFGPU_ERR_ARG; }
  CK(cudaSetDevice(h->device));
  const int surf = (h->P.tfg_xs || h->P.bc_type[5] >= 2) ? 1 : 0;
  const TuneKey key{h->nx, h->ny, h->nz, h->mixed ? 1 : 0, surf};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      for (int q = 0; q < 3; q++) {
        h->P.tile[q][0] = it->second[2 * q];
        h->P.tile[q][1] = it->second[2 * q + 1];
      }
      if (shapes) std::copy(it->second.begin(), it->second.end(), shapes);
      return PFGPU_OK;
    }
  }
  static const int cand256[][2] = {{32, 8}, {64, 4}, {128, 2}, {256, 1}, {32, 4}, {64, 2},
                                   {128, 1}};
  static const int cand128[][2] = {{32, 4}, {64, 2}, {128, 1}, {32, 2}, {64, 1}, {32, 1}};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const double dt = 0.05;
  vg_state(h, h->u, false);
  auto run = [&](int kernel) {
    if (kernel == 0) {
      launch_residual(h->P, h->u, h->p_old, h->s_old, h->kr, h->sat, dt, h->fval, h->st);
    } else if (kernel == 1) {
      if (h->mixed) {
        PCOut<float> M{h->mgf.L[0].a[0], h->mgf.L[0].a[1], h->mgf.L[0].a[2], h->mgf.L[0].a[3],
                       h->mgf.L[0].wg};
        launch_jacobian<float, float>(h->P, h->u, h->kr, h->dkr, h->sat, h->dsat, dt, h->Jf, M,
                                      h->st);
      } else {
        PCOut<double> M{h->mgd.L[0].a[0], h->mgd.L[0].a[1], h->mgd.L[0].a[2], h->mgd.L[0].a[3],
                        h->mgd.L[0].wg};
        launch_jacobian<double, double>(h->P, h->u, h->kr, h->dkr, h->sat, h->dsat, dt, h->Jd,
                                        M, h->st);
      }
    } else {
      matvec_impl(h, h->u, h->bb);
    }
    h->launches++;
  };
  auto time_of = [&](int kernel) -> float {
    run(kernel);  // warm-up
    cudaEventRecord(e0, h->st);
    for (int r = 0; r < reps; r++) run(kernel);
    cudaEventRecord(e1, h->st);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  // the Jacobian first: the matvec then reads the J it assembled
  const int order[3] = {1, 0, 2};
  for (int oi = 0; oi < 3; oi++) {
    const int q = order[oi];
    const int (*cand)[2] = q == 1 ? cand128 : cand256;
    const int nc = q == 1 ? (int)(sizeof(cand128) / sizeof(cand128[0]))
                          : (int)(sizeof(cand256) / sizeof(cand256[0]));
    h->P.tile[q][0] = h->P.tile[q][1] = 0;
    float best = time_of(q);
    int bx = 0, by = 0;
    for (int c = 0; c < nc; c++) {
      if (cand[c][1] > 1 && cand[c][1] > h->ny) continue;  // rows beyond the grid
      h->P.tile[q][0] = cand[c][0];
      h->P.tile[q][1] = cand[c][1];
      const float t = time_of(q);
      // a shape replaces the heuristic only when it is clearly faster
      if (t < (bx ? best : 0.97f * best)) {
        best = t;
        bx = cand[c][0];
        by = cand[c][1];
      }
    }
    h->P.tile[q][0] = bx;
    h->P.tile[q][1] = by;
  }
  CK(cudaGetLastError());
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the timing runs overwrote J and the preconditioner matrix
  h->jac_valid = 0;
  h->pc_ready = false;
  std::array<int, 6> out{h->P.tile[0][0], h->P.tile[0][1], h->P.tile[1][0],
                         h->P.tile[1][1], h->P.tile[2][0], h->P.tile[2][1]};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = out;
  }
  if (shapes) std::copy(out.begin(), out.end(), shapes);
  return PFGPU_OK;
}


void *pfgpu_stream(pfgpu_handle *h) { return h ? (void *)h->st : nullptr; }

long long pfgpu_kernel_launches(pfgpu_handle *h) { return h ? h->launches : 0; }

}  // extern "C"
