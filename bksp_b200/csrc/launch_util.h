// Host-side launch helpers shared by the kernel translation units
// (kernels*.cu): grid sizing for grid-stride kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <utility>

#include "dev_common.cuh"
#include "kernel_api.h"

namespace bk {

// Grid for one thread per work item, capped at the reduction grid cap.
static inline int grid_for(long long work_items) {
  long long g = (work_items + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > kMaxBlocks) g = kMaxBlocks;
  return (int)g;
}

// Blocks of `kernel` (kThreads threads, no dynamic shared memory) that are
// resident on the whole GPU at once, cached per kernel (kernels.cu).
int resident_grid(const void* kernel);

// Grid of a grid-stride streaming kernel over `items` work items (one per
// thread and sweep): exactly one wave of resident blocks, so every block
// gets the same share and no partial second wave idles most of the GPU;
// fewer blocks when the work is smaller.
template <typename K>
static int grid_wave(K* kernel, long long items) {
  const int cap = resident_grid(reinterpret_cast<const void*>(kernel));
  long long g = (items + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// Launch with programmatic stream serialisation (dev_common.cuh:
// pdl_enter): the kernel may be scheduled while its predecessor finishes.
// BKSP_GPU_PDL=0 launches plainly.  Every kernel launched here calls
// pdl_enter() (directly or through skip()) before touching memory.
static inline bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("BKSP_GPU_PDL");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

template <typename... KArgs, typename... Args>
static inline void launch_k(void (*kernel)(KArgs...), int grid, int block,
                            size_t smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  const bool plain = g_plain_scope || g_plain_launches > 0;
  if (g_plain_launches > 0) --g_plain_launches;
  attr[0].val.programmaticStreamSerializationAllowed = (pdl_enabled() && !plain) ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace bk
