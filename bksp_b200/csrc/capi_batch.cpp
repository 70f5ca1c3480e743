// Batched solves (bksp_gpu.h): many independent systems in one call.
//
// workers >= 0 (default 0 = 8): that many host worker threads take systems
// from a shared counter and run the ordinary device solve on each, on the
// worker's own CUDA stream -- one CUDA graph with its own device-side while
// loop per system, graphs of different workers running concurrently.
//
// workers < 0: one persistent launch.  Every system's solve runs on a host
// thread of its own up to its iteration loop (operator-dependent set-up
// such as the learned preconditioner's values, the initial residual),
// records one iteration of its method and joins a PersistGroup; the
// group's last member launches one cooperative kernel that iterates all
// systems in lockstep with per-system convergence masks
// (kernels_persist.cu).  A system whose iteration has no persistent form,
// and a learned solve's Jacobi retry, run as a graph loop instead.
//
// Either way each system's result does not depend on what runs beside it.
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

// Test hooks and status of this thread's persistent batches.
thread_local long long g_spin_limit = 0;
thread_local int g_absent_cta = -1;
thread_local int g_last_status = 0;
thread_local int g_last_grid = 0;

// One host thread per system, each joined to one persistent group; a
// system whose thread cannot be created withdraws from the group and is
// solved by the calling thread afterwards, outside the group.
template <typename F>
void run_persistent(int count, const F& solve_one, std::vector<int>& rets) {
  int dev = 0;
  cudaGetDevice(&dev);
  PersistGroup grp(count);
  grp.spin_limit = g_spin_limit;
  grp.absent_cta = g_absent_cta;
  auto member = [&](int i) {
    cudaSetDevice(dev);
    persist_group() = &grp;
    rets[i] = solve_one(i);
    if (persist_group() == &grp) {   // ended before its iteration loop
      persist_group() = nullptr;
      try {
        grp.withdraw(Ctx::get().st);
      } catch (const std::exception&) {
        grp.withdraw(nullptr);
      }
    }
  };
  std::vector<std::thread> pool;
  std::vector<int> later;
  for (int i = 1; i < count; ++i) {
    try {
      pool.emplace_back(member, i);
    } catch (const std::system_error&) {
      later.push_back(i);
      grp.withdraw(Ctx::get().st);
    }
  }
  member(0);
  for (auto& t : pool) t.join();
  for (int i : later) rets[i] = solve_one(i);
  g_last_status = grp.status;
  g_last_grid = grp.grid;
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
  auto one = [&](int i) {
    return bksp_gpu_solve_mixed(A[i], b[i], x[i], opts, nullptr,
                                stats ? &stats[i] : nullptr);
  };
  if (workers < 0)
    run_persistent(count, one, rets);
  else
    run_workers(count, workers > 0 ? workers : 8, one, rets);
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
  auto one = [&](int i) {
    return bksp_gpu_solve(A[i], method, l, b[i], x[i], tol, max_iter, nullptr,
                          stats ? &stats[i] : nullptr);
  };
  if (workers < 0)
    run_persistent(count, one, rets);
  else
    run_workers(count, workers > 0 ? workers : 8, one, rets);
  return summarise(rets);
}

void bksp_gpu_persist_debug(long long spin_limit, int absent_cta) {
  g_spin_limit = spin_limit > 0 ? spin_limit : 0;
  g_absent_cta = absent_cta;
}

int bksp_gpu_loop_mode(int mode) {
  try {
    Ctx& cx = Ctx::get();
    const int prev = cx.persistent ? 1 : 0;
    if (mode == 0 || mode == 1) cx.persistent = mode == 1;
    return prev;
  } catch (const std::exception&) {
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

int bksp_gpu_persist_status(int* grid) {
  if (grid) *grid = g_last_grid;
  return g_last_status;
}

}  // extern "C"
