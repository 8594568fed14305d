// Symmetric red/black Gauss-Seidel (red, black, red: RedBlackGSPoint with
// MaxIter 1 and Symmetric True, pfsimulator/parflow_lib/rb_GS_point.c:107-370)
// fused into one pass over HBM with a TMA pipeline.
//
// A CTA owns a TX x TY column of the level and marches its z planes.  Each
// plane's six arrays (C E N U b and the input iterate x) arrive as one TMA
// box per array, (TX + 8) x (TY + 6) cells wide (the halo rounded so that the
// box starts on a 16-byte boundary), into a ring of NS shared-memory slots,
// each slot guarded by one mbarrier.  The three colour sweeps run as a
// software pipeline, each lagging the previous one by two planes: at step s,
// red sweep 1 on plane s over the tile plus 2 halo cells, the black sweep on
// plane s-2 over the tile plus 1, red sweep 2 on plane s-4 over the tile.
// With that lag no sweep of a step writes a plane another sweep of the same
// step reads, so the three run concurrently between one barrier per plane;
// plane s-4 is then final and its tile is stored.  Halo cells are recomputed
// by every CTA that stages them, from the same inputs and with the same
// arithmetic (rb_update), so all CTAs agree bit for bit with each other and
// with the per-colour kernels.  Out-of-range box cells are zero-filled by the
// TMA unit, which is exactly the zero coefficient / zero value the boundary
// needs.
//
// Status: correct and bitwise equal to the per-colour sweeps, but on B200 it
// stages its halo boxes at about 10 bytes per cycle per SM however the copies
// are issued (one thread, six warps, wider boxes, or plain 16-byte cp.async),
// so on a 512 x 512 x 50 float level it takes 0.21 ms against 0.18 ms for the
// three streaming colour sweeps.  It is therefore off by default
// (PFGPU_RBR_FUSED_CELLS) and kept as the base for fusing the smoother with the
// residual and restriction that follow it.
//
// The result goes to `xout`, a buffer other than the input iterate, so no CTA
// ever reads a value that another CTA has already updated.  Every wait on an
// mbarrier is bounded (about a second); on expiry the kernel records an error
// in *err, keeps going without reading further data as valid, and the host
// reports the failure.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "pfgpu_kernels.h"

namespace pfgpu {

namespace {

template <typename T>
struct Geom {
  static constexpr int TX = RbrTile<T>::TX, TY = RbrTile<T>::TY, NS = RbrTile<T>::NS;
  static constexpr int BX = TX + 2 * RBR_HX, BY = TY + 2 * RBR_HY;
  static constexpr int BOX = BX * BY;                                    // cells per box
  static constexpr int BOXE = ((BOX * (int)sizeof(T) + 127) / 128 * 128) / (int)sizeof(T);
  static constexpr int NTH = RbrTile<T>::NTH;
  static constexpr size_t SMEM = 256 + (size_t)NS * 6 * BOXE * sizeof(T);
  static_assert(SMEM <= 227 * 1024, "ring exceeds shared memory");
  // plane s+2 is waited for at step s and issued at step s+7-NS: earlier only if NS >= 8
  static_assert(NS >= 8, "ring too short for the pipeline");
  static_assert(NTH >= 6 * 32, "one issuing warp per box");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// tiled 3-D TMA load of one box into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

constexpr uint64_t kWaitNs = 1000000000ull;  // one second per wait

}  // namespace

template <typename T>
__global__ void __launch_bounds__(Geom<T>::NTH, 1)
    k_rbr_tma(const __grid_constant__ RbrMaps maps, int nx, int ny, int nz,
              T *__restrict__ xout, int zero, int *__restrict__ err) {
  using G = Geom<T>;
  constexpr int TX = G::TX, TY = G::TY, NS = G::NS, BX = G::BX, BOXE = G::BOXE;
  constexpr int NTH = G::NTH;
  // work items of one step: red-1 cells of the tile + 2, black cells of the
  // tile + 1, red-2 cells of the tile (half of each region, rows alternate)
  constexpr int NA = (TX + 4) / 2 * (TY + 4), NB = (TX + 2) / 2 * (TY + 2), NC = TX / 2 * TY;
  constexpr int NITEM = NA + NB + NC;
  constexpr int IPT = (NITEM + NTH - 1) / NTH;    // items per thread
  constexpr int SPT = (TX * TY + NTH - 1) / NTH;  // stored cells per thread
  constexpr int SLOTE = 6 * BOXE;                 // elements per ring slot
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t pad = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + pad);
  T *sm = reinterpret_cast<T *>(smem_raw + pad + 128);
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int nbox = zero ? 5 : 6;  // zero initial guess: the iterate is not read
  const uint32_t tx_bytes = (uint32_t)(nbox * G::BOX * sizeof(T));

  // per-item constants: box index of the cell for colour offset 0, the stage
  // (0 red-1, 1 black, 2 red-2), whether the cell at offset 0 / 1 lies in the
  // domain, and the parity bit that picks the offset on a given plane
  int iq[IPT], iflag[IPT];
#pragma unroll
  for (int u = 0; u < IPT; u++) {
    const int t = tid + u * NTH;
    iq[u] = 0;
    iflag[u] = 0;
    if (t >= NITEM) continue;
    int stg, tt, h;
    if (t < NA) {
      stg = 0; tt = t; h = 2;
    } else if (t < NA + NB) {
      stg = 1; tt = t - NA; h = 1;
    } else {
      stg = 2; tt = t - NA - NB; h = 0;
    }
    const int hw = (TX + 2 * h) / 2;
    const int r = tt / hw, qq = tt - r * hw;
    const int j = y0 - h + r;
    const int i0 = x0 - h + 2 * qq;  // cell at colour offset 0; offset 1 is i0 + 1
    const int want = stg == 1 ? 0 : 1;
    const bool jin = j >= 0 && j < ny;
    const int v0 = jin && i0 >= 0 && i0 < nx, v1 = jin && i0 + 1 >= 0 && i0 + 1 < nx;
    // offset on plane k: (want ^ (i0 + j + k)) & 1; the lag 2*stg keeps parity
    const int pbit = (want ^ (i0 + j)) & 1;
    iq[u] = (i0 - x0 + RBR_HX) + BX * (j - y0 + RBR_HY);
    iflag[u] = 1 | (stg << 1) | (v0 << 3) | (v1 << 4) | (pbit << 5);
  }
  int sq[SPT];
  long long sg[SPT];
#pragma unroll
  for (int u = 0; u < SPT; u++) {
    const int t = tid + u * NTH;
    const int lx = t % TX, ly = t / TX;
    const int i = x0 + lx, j = y0 + ly;
    const bool ok = t < TX * TY && i < nx && j < ny;
    sq[u] = ok ? (lx + RBR_HX) + BX * (ly + RBR_HY) : -1;
    sg[u] = ok ? i + (long long)nx * j : 0;
  }

  // Loading plane p: one thread arms the slot's mbarrier with the bytes to
  // come (arm), then lane 0 of each of the last nbox warps issues one box
  // (issue_box), so the boxes' issue latencies overlap instead of adding up.
  auto arm = [&](int p) { mbar_expect_tx(bars + (p % NS), tx_bytes); };
  const int box_of_thread = (tid & 31) == 0 ? (NTH - 1 - tid) >> 5 : -1;  // warp 31 -> box 0
  auto issue_box = [&](int p) {
    if (box_of_thread < 0 || box_of_thread >= nbox) return;
    const int sl = p % NS;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tma_load_3d(sm + sl * SLOTE + box_of_thread * BOXE, &maps.m[box_of_thread], bars + sl,
                x0 - RBR_HX, y0 - RBR_HY, p);
  };
  bool failed = false;
  // warp 0 waits for plane p; the barrier that follows publishes it to the CTA
  auto wait = [&](int p) {
    uint64_t *bar = bars + (p % NS);
    const uint32_t par = (uint32_t)((p / NS) & 1);
    if (mbar_try_wait(bar, par)) return;
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, par)) {
      if (globaltimer() - t0 > kWaitNs) {
        failed = true;
        if (err) atomicExch(err, 1);
        return;
      }
    }
  };
  auto zero_x = [&](int p) {
    T *xx = sm + (p % NS) * SLOTE + 5 * BOXE;
    for (int t = tid; t < G::BOX; t += NTH) xx[t] = T(0);
  };
  const bool waiter = tid < 32;

  if (box_of_thread >= 0 && box_of_thread < nbox)
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.m[box_of_thread]))
                 : "memory");
  if (tid == 0) {
    for (int i = 0; i < NS; i++) mbar_init(bars + i, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int p = 0; p < NS - 5 && p < nz; p++) arm(p);
  }
  __syncthreads();
  for (int p = 0; p < NS - 5 && p < nz; p++) issue_box(p);
  if (zero) zero_x(0);
  if (waiter) {
    wait(0);
    if (1 < nz) wait(1);
  }
  __syncthreads();

  int ms = 0;  // s % NS
  for (int s = 0; s < nz + 4; s++) {
#pragma unroll
    for (int u = 0; u < IPT; u++) {
      const int f = iflag[u];
      const int stg = (f >> 1) & 3;
      const int k = s - 2 * stg;
      const int off = ((f >> 5) ^ s) & 1;
      const bool valid = (f & 1) && ((f >> (3 + off)) & 1) && k >= 0 && k < nz;
      if (!valid) continue;
      // ring slots of planes k, k-1, k+1
      int sk = ms - 2 * stg;
      if (sk < 0) sk += NS;
      const int skl = sk == 0 ? NS - 1 : sk - 1, sku = sk == NS - 1 ? 0 : sk + 1;
      const int q = iq[u] + off;
      const T *rec = sm + sk * SLOTE + q;
      T *X = sm + sk * SLOTE + 5 * BOXE + q;
      T v;
      if (stg == 0 && zero) {
        v = rec[4 * BOXE] / rec[0];
      } else {
        const bool lo = k > 0, hi = k + 1 < nz;
        const T *recl = sm + skl * SLOTE + q, *recu = sm + sku * SLOTE + 5 * BOXE + q;
        v = rb_update<T>(rec[0], rec[4 * BOXE], rec[BOXE - 1], X[-1], rec[BOXE], X[1],
                         rec[2 * BOXE - BX], X[-BX], rec[2 * BOXE], X[BX],
                         lo ? recl[3 * BOXE] : T(0), lo ? recl[5 * BOXE] : T(0),
                         hi ? rec[3 * BOXE] : T(0), hi ? recu[0] : T(0));
      }
      X[0] = v;
    }
    if (zero && s + 1 < nz) zero_x(s + 1);
    if (waiter && s + 2 < nz) wait(s + 2);  // for the next step
    // plane s-5 is no longer read after this step: its slot takes plane
    // s+NS-5 (the slot's previous phase completed long ago, so it can be armed)
    if (tid == 0 && s + NS - 5 < nz) arm(s + NS - 5);
    __syncthreads();
    if (s + NS - 5 < nz) issue_box(s + NS - 5);
    if (s >= 4) {  // plane s-4 is final
      int sk = ms - 4;
      if (sk < 0) sk += NS;
      const T *X = sm + sk * SLOTE + 5 * BOXE;
      const long long kz = (long long)nx * ny * (s - 4);
#pragma unroll
      for (int u = 0; u < SPT; u++)
        if (sq[u] >= 0) xout[sg[u] + kz] = X[sq[u]];
    }
    ms = ms == NS - 1 ? 0 : ms + 1;
  }
  if (failed) {
    // a wait gave up: let every copy this CTA issued land before it exits
    for (int p = (nz > NS ? nz - NS : 0); p < nz; p++) wait(p);
  }
}

// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

template <typename T>
bool rbr_fused_eligible(const MGLevel<T> &L) {
  // TMA global strides are multiples of 16 bytes; x stays below 2^31
  return ((long long)L.nx * (long long)sizeof(T)) % 16 == 0 && L.nx >= 1 && L.ny >= 1 &&
         L.nz >= 1 && (long long)L.nx * L.ny < (1LL << 31);
}

template <typename T>
int make_rbr_maps(const MGLevel<T> &L, const T *xin, RbrMaps *out) {
  using G = Geom<T>;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc || !rbr_fused_eligible(L)) return -1;
  memset(out, 0, sizeof(*out));
  const cuuint64_t dims[3] = {(cuuint64_t)L.nx, (cuuint64_t)L.ny, (cuuint64_t)L.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)L.nx * sizeof(T),
                                 (cuuint64_t)L.nx * L.ny * sizeof(T)};
  const cuuint32_t box[3] = {(cuuint32_t)G::BX, (cuuint32_t)G::BY, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  const void *ptr[6] = {L.a[0], L.a[1], L.a[2], L.a[3], L.b, xin};
  const CUtensorMapDataType dt =
      sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  for (int a = 0; a < 6; a++) {
    CUresult r = enc(&out->m[a], dt, 3, const_cast<void *>(ptr[a]), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return -1;
  }
  return 0;
}

template <typename T>
cudaError_t rbr_fused_prepare() {
  return cudaFuncSetAttribute(k_rbr_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Geom<T>::SMEM);
}

template <typename T>
void launch_rbr_fused(const MGLevel<T> &L, const RbrMaps &maps, T *xout, int zero, int *err,
                      cudaStream_t st) {
  using G = Geom<T>;
  dim3 grid((L.nx + G::TX - 1) / G::TX, (L.ny + G::TY - 1) / G::TY);
  k_rbr_tma<T><<<grid, G::NTH, G::SMEM, st>>>(maps, L.nx, L.ny, L.nz, xout, zero, err);
}

#define INST_TMA(T)                                                                     \
  template bool rbr_fused_eligible<T>(const MGLevel<T> &);                               \
  template int make_rbr_maps<T>(const MGLevel<T> &, const T *, RbrMaps *);               \
  template cudaError_t rbr_fused_prepare<T>();                                           \
  template void launch_rbr_fused<T>(const MGLevel<T> &, const RbrMaps &, T *, int, int *, \
                                    cudaStream_t);
INST_TMA(float)
INST_TMA(double)

}  // namespace pfgpu
