// Ensemble stepping: many independent Richards problems advanced at once.
//
// Each member is its own handle with its own non-blocking stream, its own
// CUDA graph and its own device state, so the members' kernels are free to
// overlap on the GPU: while one member's host loop waits on a Krylov scalar
// or runs the launch-bound coarse multigrid levels, the others stream their
// large-level kernels.  A pool of host threads drives the members' Newton
// loops (KINSOL's control flow is host-driven, one thread per member at a
// time); members are taken from a shared counter so uneven grids balance.
//
// This is the ensemble configuration of the survey (48 members of uneven
// size); the reference runs the members as separate processes one after
// another.  No counterpart in the reference API.
#include <atomic>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pfgpu.h"
#include "pfgpu_kernels.h"

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
