// Batched solves (bksp_gpu.h): many independent systems in one call.
//
// Host worker threads take systems from a shared counter and run the
// ordinary device solve on each, on the worker's own CUDA stream (the
// library's per-thread stream).  Every system is therefore one CUDA graph
// with its own device-side while loop and convergence flag -- a converged
// system stops, the others keep iterating -- and the GPU runs the graphs
// of different workers concurrently, so small systems share the SMs
// instead of queueing behind each other.  Graph capture and instantiation,
// the host part of a solve, also proceed in parallel.  Results are
// deterministic: each system's arithmetic does not depend on what runs
// beside it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <system_error>
#include <thread>
#include <vector>

#include "capi_internal.h"

using namespace bk;

namespace {

// Run solve_one(i) for i in [0, count) on `workers` host threads (the
// calling thread is one of them) bound to the caller's device; rets[i]
// receives each system's code.
template <typename F>
void run_workers(int count, int workers, const F& solve_one, std::vector<int>& rets) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (workers <= 0) workers = 8;
  workers = std::max(1, std::min(workers, count));
  std::atomic<int> next{0};
  auto work = [&]() {
    cudaSetDevice(dev);
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= count) break;
      rets[i] = solve_one(i);
    }
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < workers; ++w) {
    try {
      pool.emplace_back(work);
    } catch (const std::system_error&) {
      break;   // fewer threads: the remaining workers take their share
    }
  }
  work();
  for (auto& t : pool) t.join();
}

int summarise(const std::vector<int>& rets) {
  int ret = 0;
  for (int r : rets) {
    if (r == INVALID_PARAMETERS) return INVALID_PARAMETERS;
    if (r < 0) ret = NOT_CONVERGED;
  }
  return ret;
}

}  // namespace

extern "C" {

int bksp_gpu_solve_mixed_batch(bksp_gpu_matrix* const* A, const double* const* b,
                               double* const* x, int count,
                               const bksp_gpu_mixed_opts* opts, int workers,
                               bksp_gpu_stats* stats) {
  if (count < 0 || (count > 0 && (!A || !b || !x || !opts))) return INVALID_PARAMETERS;
  for (int i = 0; i < count; ++i)
    if (!A[i] || !b[i] || !x[i]) return INVALID_PARAMETERS;
  if (count == 0) return 0;
  std::vector<int> rets(count, INVALID_PARAMETERS);
  run_workers(count, workers, [&](int i) {
    return bksp_gpu_solve_mixed(A[i], b[i], x[i], opts, nullptr,
                                stats ? &stats[i] : nullptr);
  }, rets);
  return summarise(rets);
}

int bksp_gpu_solve_batch(bksp_gpu_matrix* const* A, int method, int l,
                         const double* const* b, double* const* x, int count,
                         double tol, int max_iter, int workers,
                         bksp_gpu_stats* stats) {
  if (count < 0 || (count > 0 && (!A || !b || !x))) return INVALID_PARAMETERS;
  for (int i = 0; i < count; ++i)
    if (!A[i] || !b[i] || !x[i]) return INVALID_PARAMETERS;
  if (count == 0) return 0;
  std::vector<int> rets(count, INVALID_PARAMETERS);
  run_workers(count, workers, [&](int i) {
    return bksp_gpu_solve(A[i], method, l, b[i], x[i], tol, max_iter, nullptr,
                          stats ? &stats[i] : nullptr);
  }, rets);
  return summarise(rets);
}

}  // extern "C"
