// Ensemble stepping: many independent Richards problems advanced at once.
//
// By default every timestep of all members is one CUDA graph launch: each
// member's whole Newton solve, with its own device-side KINSOL/SPGMR control
// (the member's convergence steers its own conditional nodes), is one root
// branch of the graph, so the members' kernels overlap on the GPU and the
// host waits once per timestep (ensemble_graph_advance in pfgpu.cu).  A
// member whose solve fails is retried with the halved dt on its own.
//
// Otherwise (PFGPU_ENSEMBLE_GRAPH=0, host-driven solves, trajectory
// recording, members on several devices) a pool of host threads drives the
// members' steps, each member on its own non-blocking stream; members are
// taken from a shared counter so uneven grids balance.
//
// The workload is an ensemble of independent realisations (48 members of
// uneven size); the reference runs such members as separate processes one
// after another.  No counterpart in the reference API.
#include <atomic>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pfgpu.h"
#include "pfgpu_kernels.h"

namespace pfgpu {
// Advances the ensemble members as pfgpu_ensemble_advance does, every
// timestep of all members as one CUDA graph launch, when every member can
// run its solve as a graph (same device, distinct handles, no trajectory
// recording); *handled is false when it did nothing (the caller's
// per-member path then runs).
int ensemble_graph_advance(pfgpu_handle *const *members, int n, const double *dt, int nsteps,
                           pfgpu_stats *stats, int *status, bool *handled);
}  // namespace pfgpu

extern "C" int pfgpu_ensemble_advance(pfgpu_handle *const *members, int n, const double *dt,
                                      int nsteps, int nthreads, pfgpu_stats *stats,
                                      int *status) {
  if (!members || n < 1 || !dt || nsteps < 0 || !status) {
    pfgpu::record_error("pfgpu_ensemble_advance: bad argument");
    return PFGPU_ERR_ARG;
  }
  for (int m = 0; m < n; m++)
    if (!members[m] || !(dt[m] > 0)) {
      pfgpu::record_error("pfgpu_ensemble_advance: null member or non-positive dt");
      return PFGPU_ERR_ARG;
    }
  bool handled = false;
  const int grc =
      pfgpu::ensemble_graph_advance(members, n, dt, nsteps, stats, status, &handled);
  if (handled) return grc;
  if (nthreads <= 0 || nthreads > n) nthreads = n;
  std::atomic<int> next{0};
  std::vector<std::string> msg(n);  // a failing member's message (thread-local there)
  auto worker = [&]() {
    for (;;) {
      const int m = next.fetch_add(1);
      if (m >= n) return;
      status[m] = pfgpu_advance(members[m], dt[m], nsteps,
                                stats ? stats + (size_t)m * (nsteps > 0 ? nsteps : 1) : nullptr);
      if (status[m] != PFGPU_OK) msg[m] = pfgpu_last_error();
    }
  };
  std::vector<std::thread> pool;
  pool.reserve(nthreads - 1);
  for (int t = 1; t < nthreads; t++) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  int rc = PFGPU_OK, first = -1;
  for (int m = 0; m < n; m++) {
    if (status[m] == PFGPU_OK) continue;
    if (first < 0 || (status[m] < 0 && rc >= 0)) first = m;
    if (status[m] < 0 && rc >= 0) rc = status[m];
    else if (rc == PFGPU_OK) rc = PFGPU_NOT_CONVERGED;
  }
  if (first >= 0)
    pfgpu::record_error(("ensemble member " + std::to_string(first) + ": " + msg[first]).c_str());
  return rc;
}
