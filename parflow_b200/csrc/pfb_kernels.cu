// ParFlow binary (PFB) values on the device: the format stores every value
// big-endian, x fastest within each subgrid box (write_parflow_binary.c:74-205,
// read_parflow_binary.c:38-120).  The library packs and byte-swaps a dense
// field in one pass before a single device-to-host copy, and scatters a
// subgrid's raw bytes into the dense field, swapping them, after a single
// host-to-device copy.
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

__device__ __forceinline__ unsigned long long bswap64(unsigned long long v) {
  const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
  return ((unsigned long long)__byte_perm(lo, 0, 0x0123) << 32) |
         (unsigned long long)__byte_perm(hi, 0, 0x0123);
}

__global__ void k_pfb_pack(const double *__restrict__ dense, unsigned long long *__restrict__ out,
                           long long n) {
  pdl_enter();
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    out[c] = bswap64((unsigned long long)__double_as_longlong(dense[c]));
}

// one subgrid box (ix, iy, iz, snx, sny, snz) of an nx x ny x nz grid
__global__ void k_pfb_scatter(const unsigned long long *__restrict__ raw,
                              double *__restrict__ dense, int nx, int ny, int ix, int iy, int iz,
                              int snx, int sny, int snz) {
  pdl_enter();
  const long long n = (long long)snx * sny * snz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % snx);
    const long long r = t / snx;
    const int y = (int)(r % sny), z = (int)(r / sny);
    const long long c = (ix + x) + (long long)nx * ((iy + y) + (long long)ny * (iz + z));
    dense[c] = __longlong_as_double((long long)bswap64(raw[t]));
  }
}

static unsigned grid_1d(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

void launch_pfb_pack(const double *dense, unsigned long long *out, long long n,
                     cudaStream_t st) {
  launch_pdl(k_pfb_pack, dim3(grid_1d(n)), dim3(256), st, dense, out, n);
}
void launch_pfb_scatter(const unsigned long long *raw, double *dense, int nx, int ny, int ix,
                        int iy, int iz, int snx, int sny, int snz, cudaStream_t st) {
  launch_pdl(k_pfb_scatter, dim3(grid_1d((long long)snx * sny * snz)), dim3(256), st, raw, dense,
             nx, ny, ix, iy, iz, snx, sny, snz);
}

}  // namespace pfgpu
