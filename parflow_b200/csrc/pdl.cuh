// Programmatic dependent launch (PDL) helpers shared by the kernel files.
//
// A kernel launched with launch_pdl may have its blocks scheduled while the
// previous kernel in the stream is still draining; it calls pdl_enter()
// first, which waits until that kernel has completed and its writes are
// visible, then lets the next kernel's launch begin.  Kernels launched this
// way keep exact stream order for memory; only launch latency overlaps.
// PFGPU_PDL=0 in the environment turns the attribute off.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>

namespace pfgpu {

__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
#ifndef PFGPU_PDL_LATE_TRIGGER
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// set while capturing a graph whose driver refused programmatic edges
inline bool &pdl_capture_off() {
  static thread_local bool off = false;
  return off;
}

inline bool pdl_on() {
  static const bool on = [] {
    const char *v = getenv("PFGPU_PDL");
    return !(v && *v == '0');
  }();
  return on && !pdl_capture_off();
}

template <typename... KArgs, typename... Args>
inline void launch_pdl_smem(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                            cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = pdl_on() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// one thread-block cluster of cs blocks along x
template <typename... KArgs, typename... Args>
inline void launch_pdl_cluster(void (*kern)(KArgs...), int cs, dim3 block, size_t smem,
                               cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = pdl_on() ? 1 : 0;
  attr[1].id = cudaLaunchAttributeClusterDimension;
  attr[1].val.clusterDim.x = cs;
  attr[1].val.clusterDim.y = 1;
  attr[1].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                       Args... args) {
  launch_pdl_smem(kern, grid, block, 0, st, args...);
}

}  // namespace pfgpu
