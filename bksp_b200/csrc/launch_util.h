// Host-side launch helpers shared by the kernel translation units
// (kernels*.cu): grid sizing for grid-stride kernels.
#pragma once
#include <cuda_runtime.h>

#include "dev_common.cuh"

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

}  // namespace bk
