// Allocation-free residual entry point (pfgpu_residual_noalloc).
//
// For callers that may not call the CUDA allocator: a host framework that
// reserves its whole device-memory budget at start-up and refuses later
// allocations, or a latency-critical loop where cudaMalloc/cudaFree would
// synchronise the device.  Such a caller passes every input and output as
// device memory; the per-cell scratch the residual needs (relative
// permeability, saturation and their derivatives) and the per-layer dz
// constants live in the file-scope device array below, which every GPU that
// loads this library holds until the process exits.  The layer constants
// travel as kernel arguments, so the call makes no host-to-device copy either.
//
// Limits: at most kMaxCells interior cells and kMaxLayers layers per call.
// Every call on a device shares the one array and leaves the last call's
// values in it, so calls whose kernels overlap on the GPU (different streams,
// no ordering between them) race and corrupt each other's results; order
// them on one stream or synchronise between them.  Each call rewrites every
// scratch entry it reads before reading it, so nothing has to start at zero.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/pfgpu.h"
#include "pfgpu_kernels.h"

using namespace pfgpu;

namespace {

constexpr long long kMaxCells = 262144;  // 2^18 cells, e.g. 64 x 64 x 64 (8 MiB of doubles)
constexpr int kMaxLayers = 1024;
// kr, dkr, S, dS per cell, then z_mult and three per-face constants per layer
constexpr long long kScratchDoubles = 4 * kMaxCells + 4LL * kMaxLayers;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
// device address of g_noalloc_scratch per device, resolved once under the
// mutex (two host threads making their first call on one device at the same
// time both see the one resolved address).  cudaDeviceReset destroys the
// context the address belongs to: a process that resets a device must not
// call pfgpu_residual_noalloc on it again.
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// layer constants of up to kLayerChunk layers, passed by value to k_layers
constexpr int kLayerChunk = 64;
struct LayerChunk {
  int k0, count;
  double zmult[kLayerChunk];
  double zface[3 * kLayerChunk];
};

__global__ void k_layers(LayerChunk c, double *zmult, double *zface) {
  const int t = threadIdx.x;
  if (t < c.count) {
    zmult[c.k0 + t] = c.zmult[t];
    zface[3 * (c.k0 + t)] = c.zface[3 * t];
    zface[3 * (c.k0 + t) + 1] = c.zface[3 * t + 1];
    zface[3 * (c.k0 + t) + 2] = c.zface[3 * t + 2];
  }
}

int fail(int code, const char *fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  pfgpu::record_error(msg);
  return code;
}

// device memory of device `dev` (a buffer of another GPU is rejected: the
// kernels would read it over the peer path or fault), or managed memory
bool on_device(const void *p, int dev) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int pfgpu_residual_noalloc(const pfgpu_desc *desc, const double *perm,
                                      const double *vg_alpha, const double *vg_n,
                                      const double *s_res, const double *s_sat,
                                      const int *bc_type, const double *const *bc_values,
                                      const double *p, const double *p_old,
                                      const double *s_old, double dt, double *f,
                                      void *stream) {
  if (!desc || desc->abi_version != PFGPU_ABI_VERSION)
    return fail(PFGPU_ERR_ARG, "pfgpu_residual_noalloc: null descriptor or ABI mismatch");
  const long long n = (long long)desc->nx * desc->ny * desc->nz;
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1)
    return fail(PFGPU_ERR_ARG, "pfgpu_residual_noalloc: empty grid");
  if (n > kMaxCells || desc->nz > kMaxLayers)
    return fail(PFGPU_ERR_ARG,
                "pfgpu_residual_noalloc: %lld cells / %d layers exceed the static scratch "
                "limit of %lld cells / %d layers",
                n, desc->nz, kMaxCells, kMaxLayers);
  if (!bc_type || !bc_values)
    return fail(PFGPU_ERR_ARG, "pfgpu_residual_noalloc: null boundary tables");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(PFGPU_ERR_CUDA, "pfgpu_residual_noalloc: no usable current device");
  const void *dev_args[] = {perm, p, p_old, s_old, f};
  for (const void *a : dev_args)
    if (!on_device(a, dev))
      return fail(PFGPU_ERR_ARG,
                  "pfgpu_residual_noalloc: inputs and output must be memory of the current "
                  "device %d", dev);
  for (int face = 0; face < 6; face++) {
    if (bc_type[face] != PFGPU_BC_FLUX && bc_type[face] != PFGPU_BC_DIRICHLET)
      return fail(PFGPU_ERR_ARG,
                  "pfgpu_residual_noalloc: face %d: only FluxConst and Dirichlet faces", face);
    if (!on_device(bc_values[face], dev))
      return fail(PFGPU_ERR_ARG,
                  "pfgpu_residual_noalloc: face %d table must be memory of the current device",
                  face);
  }
  const double *vg[] = {vg_alpha, vg_n, s_res, s_sat};
  for (const double *a : vg)
    if (a && !on_device(a, dev))
      return fail(PFGPU_ERR_ARG,
                  "pfgpu_residual_noalloc: per-cell fields must be memory of the current device");

  // set-up, once per device, with that device current: the device address of
  // the scratch array (its host-side name is only a stand-in)
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      void *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return fail(PFGPU_ERR_CUDA, "pfgpu_residual_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<double *>(ptr);
    }
    scratch = g_scratch_ptr[dev];
  }
  double *kr = scratch, *dkr = scratch + kMaxCells, *sat = scratch + 2 * kMaxCells,
         *dsat = scratch + 3 * kMaxCells;
  double *zmult = scratch + 4 * kMaxCells, *zface = zmult + kMaxLayers;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // per-layer constants, as pfgpu_create derives them:
  // 1/(dz mean(z_k, z_k+1)), z_k/(z_k+z_k+1), z_k+1/(z_k+z_k+1)
  const int nz = desc->nz;
  auto zm_at = [&](int k) { return desc->z_mult ? desc->z_mult[k] : 1.0; };
  for (int k0 = 0; k0 < nz; k0 += kLayerChunk) {
    LayerChunk c;
    memset(&c, 0, sizeof(c));
    c.k0 = k0;
    c.count = nz - k0 < kLayerChunk ? nz - k0 : kLayerChunk;
    for (int t = 0; t < c.count; t++) {
      const int k = k0 + t;
      c.zmult[t] = zm_at(k);
      if (k + 1 < nz) {
        const double za = zm_at(k), zb = zm_at(k + 1);
        c.zface[3 * t] = 1.0 / (desc->dz * (0.5 * (za + zb)));
        c.zface[3 * t + 1] = za / (za + zb);
        c.zface[3 * t + 2] = zb / (za + zb);
      }
    }
    k_layers<<<1, kLayerChunk, 0, st>>>(c, zmult, zface);
  }

  DevProblem P;
  memset(&P, 0, sizeof(P));
  P.nx = desc->nx; P.ny = desc->ny; P.nz = desc->nz; P.n = n;
  P.dx = desc->dx; P.dy = desc->dy; P.dz = desc->dz;
  P.gravity = desc->gravity; P.viscosity = desc->viscosity; P.density = desc->density;
  P.porosity = desc->porosity; P.sstorage = desc->specific_storage;
  P.alpha = vg_alpha; P.vgn = vg_n; P.sres = s_res; P.ssat = s_sat;
  P.alpha0 = desc->vg_alpha; P.vgn0 = desc->vg_n; P.sres0 = desc->s_res; P.ssat0 = desc->s_sat;
  P.vg_from_file = desc->vg_from_file;
  P.kx = P.ky = P.kz = perm;
  P.zmult = zmult;
  P.zface = zface;
  P.inv_dx = 1.0 / desc->dx;
  P.inv_dy = 1.0 / desc->dy;
  P.inv_visc = 1.0 / desc->viscosity;
  for (int face = 0; face < 6; face++) {
    P.bc_type[face] = bc_type[face];
    P.bc_val[face] = bc_values[face];
  }
  launch_vg_all(P, p, kr, dkr, sat, dsat, st);
  launch_residual(P, p, p_old, s_old, kr, sat, dt, f, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(PFGPU_ERR_CUDA, "pfgpu_residual_noalloc: launch failed: %s",
                cudaGetErrorString(e));
  return PFGPU_OK;
}
