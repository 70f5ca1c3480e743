// Device-side building blocks shared by every kernel of the solver library.
//
// Execution model.  A solve is a fixed sequence of kernel launches per
// iteration (captured once into a CUDA graph).  All scalars of the Krylov
// recurrences live in device memory (`S`, FP64): reduction kernels write
// their dot products there and the LAST block of each reduction runs a
// small scalar "epilogue" (one thread) that advances the recurrence
// (alpha, beta, omega, ...) and performs the convergence test.  No host
// round-trip happens inside an iteration.  Once the convergence test passes
// (or the iteration budget is spent, or a scalar breaks down) the epilogue
// sets `ctl->done`; every kernel checks that flag on entry and returns, so
// extra iterations queued behind the converged one are no-ops and the state
// stays exactly as the converging iteration left it.
//
// Reductions are deterministic: per-thread partial sums over fixed index
// sets, a fixed warp/block tree, per-block partials in global memory and a
// fixed-order final sum in whichever block arrives last.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernel_api.h"

namespace bk {

constexpr int kThreads = 256;            // threads per block, all kernels
constexpr int kWarps = kThreads / 32;
constexpr int kSMs = 148;                // B200
constexpr int kMaxBlocks = kSMs * 8;     // grid cap: 8 resident blocks per SM
constexpr int kMaxDots = 8;              // dots one kernel may produce
static_assert(kMaxBlocks == kGridCap, "grid cap mismatch");

// Solve control block and reduction context (layouts in kernel_api.h).
//   Ctl: done / iter / ret / max_iter / hist_cap / trips / trip_cap / hist_len,
//        tol, hist (per-iteration convergence-test values, or null).
//   Red: per-block partials [kMaxDots][kMaxBlocks], arrival ticket (reset by
//        the last block), scalar slots S, ctl, the S slot receiving dot 0,
//        the epilogue code run by the last block and two epilogue params.
using Ctl = CtlH;
using Red = RedH;
using Cf = CfH;

__device__ __forceinline__ bool finished(const Ctl* c) {
  return *(volatile const int*)&c->done != 0;
}

// Programmatic dependent launch: the solve-loop kernels are launched
// allowed to start while their predecessor in the stream is still running
// (its last CTA's scalar epilogue, typically).  A kernel waits here until
// the predecessor has completed and its memory is visible -- before its
// first access to anything the predecessor may write -- and then lets its
// own successor be scheduled.  Both instructions are no-ops for a launch
// without the attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
// Let the successor be scheduled: kernels with a reduction call this when
// their streaming work is done (finish_reduction), so the successor's launch
// overlaps the last CTA's serial tail; others trigger implicitly at exit.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Entry test of every kernel: the solve has finished, or the launch is
// guarded by a scalar slot that is currently zero (conditional steps such
// as a residual replacement inside a captured iteration).
__device__ __forceinline__ bool skip(const Red& rd) {
  pdl_enter();
  if (finished(rd.ctl)) return true;
  return rd.guard > 0 && *(volatile const double*)(rd.S + rd.guard) == 0.0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Scalar epilogue dispatcher (epilogues.cuh).
static __device__ __noinline__ void run_epilogue(const Red& rd);

// Block-reduce ND per-thread accumulators, publish the block's partials and
// let the last-arriving block finish the sums into S[out..] and run the
// epilogue.  Must be called by every thread of every block of the grid.
template <int ND>
__device__ __forceinline__ void finish_reduction(const double* acc,
                                                 const Red& rd) {
  __shared__ double sh[ND > 0 ? ND : 1][kWarps];
  __shared__ int is_last;
  pdl_trigger();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double v = warp_sum(acc[d]);
    if (lane == 0) sh[d][warp] = v;
  }
  __syncthreads();
  const bool single = gridDim.x == 1;   // one CTA: its sums are the totals
  if (threadIdx.x == 0 && !single) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) s += sh[d][w];
      rd.part[d * kMaxBlocks + blockIdx.x] = s;
    }
    // Release: the partials above are visible to whichever CTA sees this
    // increment complete the count; acquire: the last CTA sees all of them.
    unsigned t;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                 : "=r"(t) : "l"(rd.ticket) : "memory");
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!single && !is_last) return;
  if (!single) __threadfence();
  double tot[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double v = 0.0;
    if (single) {
      if (threadIdx.x < kWarps) v = sh[d][threadIdx.x];
    } else {
      for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads)
        v += __ldcg(rd.part + d * kMaxBlocks + b);
    }
    tot[d] = warp_sum(v);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < ND; ++d) sh[d][warp] = tot[d];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) s += sh[d][w];
      rd.S[rd.out + d] = s;
    }
    if (!single) *rd.ticket = 0u;   // visible to the next kernel at exit
    if (rd.epi) run_epilogue(rd);
  }
}

// Packet types for 16-byte vector memory access.
template <typename T> struct Pack;
template <> struct Pack<double> {
  using V = double2;
  static constexpr int N = 2;
};
template <> struct Pack<float> {
  using V = float4;
  static constexpr int N = 4;
};

template <typename T>
__device__ __forceinline__ void unpack(const typename Pack<T>::V& p, T* e);
template <>
__device__ __forceinline__ void unpack<double>(const double2& p, double* e) {
  e[0] = p.x; e[1] = p.y;
}
template <>
__device__ __forceinline__ void unpack<float>(const float4& p, float* e) {
  e[0] = p.x; e[1] = p.y; e[2] = p.z; e[3] = p.w;
}
template <typename T>
__device__ __forceinline__ typename Pack<T>::V repack(const T* e);
template <>
__device__ __forceinline__ double2 repack<double>(const double* e) {
  return make_double2(e[0], e[1]);
}
template <>
__device__ __forceinline__ float4 repack<float>(const float* e) {
  return make_float4(e[0], e[1], e[2], e[3]);
}

// Rounded arithmetic without FMA contraction, to reproduce the reference's
// CPU operation order where that matters (SpMV row sums, scal).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Coefficient of a linear-combination term, resolved from the scalar slots.
__device__ __forceinline__ double eval_cf(const Cf& c, const double* S) {
  switch (c.op) {
    case 1: return c.k;
    case 2: return c.k * S[c.s];
    case 3: return c.k / S[c.s];
    case 4: return c.k * S[c.s] / S[c.s2];
    case 5: return c.k * S[c.s] * S[c.s2];
    default: return 0.0;
  }
}

}  // namespace bk
