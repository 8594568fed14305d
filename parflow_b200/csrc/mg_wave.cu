// Red/black/red smoothing of one multigrid level as a wavefront through L2.
//
// The three colour sweeps of RedBlackGSPoint (pfsimulator/parflow_lib/
// rb_GS_point.c:107-240: red, black, red, one iteration) run in ONE
// persistent kernel.  The level is cut into work items (sweep s, plane k,
// chunk of rows c).  Sweep s of plane k reads only the other colour on planes
// k-1, k, k+1 as left by sweep s-1, so it may start once sweep s-1 is done on
// those three planes; its writes are read by sweep s+1 of the same planes,
// which wait on it in turn.  Items are numbered in wavefront order
// tau = k + 2 s (sweep s trails sweep s-1 by two planes) and claimed from an
// atomic counter in that order (more generally tau = k + lag s, lag >= 2,
// which keeps more items ready at once), so every item depends only on items claimed
// before it by blocks that are already running: the kernel cannot deadlock,
// whatever the number of resident blocks.
//
// Each plane is read from HBM by the first sweep and, a few planes later, by
// the second and third sweeps while it is still in the 126 MB L2, so the level
// streams its operator and right-hand side once per smoothing instead of
// three times.  The per-cell arithmetic is rb_update, as in the per-colour
// kernels, so the result is bitwise identical to three k_rb_sweep launches.
//
// Synchronisation: per (sweep, plane) completion counters.  A producer block
// fences its stores and then increments the counter; a consumer's thread 0
// waits with acquire loads (bounded by kWaveWaitNs; on expiry it raises the
// abort flag, which makes every block stop waiting, and records error 2),
// and the block reads the iterate through L2 (ld.global.cg) so that no stale
// L1 line is used.  The last block to exit resets the counters for the next
// launch.
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

static const int WAVE_THREADS = 256;
static const unsigned long long kWaveWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long wave_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// one red/black point update reading the iterate through L2
template <typename T>
__device__ __forceinline__ void rb_cell_l2(const MGLevel<T> &L, T *x, const T *__restrict__ b,
                                           int colour, int init, int q, int j, int k) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int want = colour == 0 ? 1 : 0;  // parity of (i+j+k); red = odd
  const int i = 2 * q + ((want ^ (j + k)) & 1);
  if (i >= nx) return;
  const long long sy = nx, sz = (long long)nx * ny;
  const long long c = i + sy * j + sz * k;
  const T *__restrict__ a0 = L.a[0];
  const T *__restrict__ ae = L.a[1];
  const T *__restrict__ an = L.a[2];
  const T *__restrict__ au = L.a[3];
  if (init) {
    __stcg(x + c, b[c] / a0[c]);
    return;
  }
  const T v = rb_update<T>(a0[c], b[c], i > 0 ? ae[c - 1] : T(0), i > 0 ? __ldcg(x + c - 1) : T(0),
                           ae[c], i + 1 < nx ? __ldcg(x + c + 1) : T(0),
                           j > 0 ? an[c - sy] : T(0), j > 0 ? __ldcg(x + c - sy) : T(0),
                           an[c], j + 1 < ny ? __ldcg(x + c + sy) : T(0),
                           k > 0 ? au[c - sz] : T(0), k > 0 ? __ldcg(x + c - sz) : T(0),
                           au[c], k + 1 < nz ? __ldcg(x + c + sz) : T(0));
  __stcg(x + c, v);
}

// ctl: [0] item counter, [1] abort flag, [2] exit counter, [3 + s*nz + k]
// chunks of (sweep s, plane k) completed; plan: (sweep, plane) tasks in
// wavefront order as s*nz + k
template <typename T>
__global__ void __launch_bounds__(WAVE_THREADS) k_rbr_wave(MGLevel<T> L, T *x,
                                                           const T *__restrict__ b, int zero,
                                                           int *ctl, const int *__restrict__ plan,
                                                           int rows, int nchunks, int *err) {
  pdl_enter();
  __shared__ int sh_item, sh_skip;
  const int nz = L.nz, ny = L.ny;
  const int hx = (L.nx + 1) / 2;
  const int total = 3 * nz * nchunks;
  int *done = ctl + 3;
  for (;;) {
    if (threadIdx.x == 0) sh_item = atomicAdd(ctl, 1);
    __syncthreads();
    const int g = sh_item;
    if (g >= total) break;
    const int pt = g / nchunks, c = g - pt * nchunks;
    const int sk = plan[pt];
    const int s = sk / nz, k = sk - s * nz;
    if (threadIdx.x == 0) {
      int skip = *(volatile int *)(ctl + 1);
      if (!skip && s > 0) {
        for (int kk = k - 1; kk <= k + 1 && !skip; kk++) {
          if (kk < 0 || kk >= nz) continue;
          const int *cnt = done + (s - 1) * nz + kk;
          if (ld_acquire(cnt) >= nchunks) continue;
          const unsigned long long t0 = wave_clock();
          while (ld_acquire(cnt) < nchunks) {
            if (*(volatile int *)(ctl + 1)) {
              skip = 1;
              break;
            }
            if (wave_clock() - t0 > kWaveWaitNs) {
              atomicExch(ctl + 1, 1);
              if (err) atomicExch(err, 2);
              skip = 1;
              break;
            }
            __nanosleep(100);
          }
        }
      }
      sh_skip = skip;
    }
    __syncthreads();
    if (!sh_skip) {
      const int colour = s == 1 ? 1 : 0;
      const int init = s == 0 ? zero : 0;
      const int j0 = c * rows;
      const int j1 = j0 + rows < ny ? j0 + rows : ny;
      const int cnt = (j1 - j0) * hx;
      for (int t = threadIdx.x; t < cnt; t += WAVE_THREADS) {
        const int jj = t / hx;
        rb_cell_l2(L, x, b, colour, init, t - jj * hx, j0 + jj, k);
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(done + s * nz + k, 1);
  }
  // the last block out resets the control words for the next launch
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(ctl + 2, 1) == (int)gridDim.x - 1) {
      for (int q = 0; q < 3 * nz; q++) done[q] = 0;
      ctl[0] = 0;
      ctl[1] = 0;
      __threadfence();
      ctl[2] = 0;
    }
  }
}

template <typename T>
int wave_setup(const MGLevel<T> &L, int ctas_per_sm, int lag, int chunk_cells, WaveLevel *w) {
  const int hx = (L.nx + 1) / 2;
  if (lag < 2) lag = 2;
  if (chunk_cells < 1) chunk_cells = 4096;
  int rows = chunk_cells / (hx > 0 ? hx : 1);
  if (rows < 1) rows = 1;
  if (rows > L.ny) rows = L.ny;
  w->rows = rows;
  w->nchunks = (L.ny + rows - 1) / rows;
  const int nz = L.nz;
  std::vector<int> plan;
  plan.reserve(3 * nz);
  for (int tau = 0; tau < nz + 2 * lag; tau++)
    for (int s = 2; s >= 0; s--) {
      const int k = tau - lag * s;
      if (k >= 0 && k < nz) plan.push_back(s * nz + k);
    }
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rbr_wave<T>, WAVE_THREADS, 0) !=
          cudaSuccess)
    return -1;
  if (ctas_per_sm > 0 && ctas_per_sm < occ) occ = ctas_per_sm;
  if (occ < 1) occ = 1;
  const long long items = 3LL * nz * w->nchunks;
  const long long g = (long long)sms * occ;
  w->grid = (int)(g < items ? g : items);
  if (cudaMalloc((void **)&w->ctl, (3 + 3 * nz) * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void **)&w->plan, 3 * nz * sizeof(int)) != cudaSuccess ||
      cudaMemset(w->ctl, 0, (3 + 3 * nz) * sizeof(int)) != cudaSuccess ||
      cudaMemcpy(w->plan, plan.data(), 3 * nz * sizeof(int), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return 0;
}

void wave_free(WaveLevel *w) {
  cudaFree(w->ctl);
  cudaFree(w->plan);
  w->ctl = nullptr;
  w->plan = nullptr;
}

template <typename T>
void launch_rbr_wave(const MGLevel<T> &L, const WaveLevel &w, T *x, const T *b, int zero,
                     int *err, cudaStream_t st) {
  launch_pdl(k_rbr_wave<T>, dim3(w.grid), dim3(WAVE_THREADS), st, L, x, b, zero, w.ctl,
             (const int *)w.plan, w.rows, w.nchunks, err);
}

#define INST(T)                                                                           \
  template int wave_setup<T>(const MGLevel<T> &, int, int, int, WaveLevel *);            \
  template void launch_rbr_wave<T>(const MGLevel<T> &, const WaveLevel &, T *, const T *, \
                                   int, int *, cudaStream_t);
INST(float)
INST(double)

}  // namespace pfgpu
