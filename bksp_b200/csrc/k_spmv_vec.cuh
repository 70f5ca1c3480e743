// K1 (vector CSR): a sub-warp of L lanes per row (L = 4, 8, 16 or 32).  Each
// lane loads one stored entry of the row per chunk (the group's loads are
// contiguous, so a warp's column / value loads coalesce across its rows)
// and gathers its x entry, so all of a row's gathers are in flight at once.
// The row's products are then summed by the group's first lane, fetched
// with warp shuffles in entry order: y = ((0 + p_0) + p_1) + ..., without
// FMA -- the reference's dcsrgemm0 order, bit-identical in FP64.
#pragma once
#include "dev_common.cuh"

namespace bk {

template <typename VT, typename XT, int ND, int L>
__global__ void __launch_bounds__(kThreads, 8)
k_spmv_vec(CsrH A, SpmvH<XT> io, Red rd) {
  if (skip(rd)) return;
  const VT* __restrict__ Aval = static_cast<const VT*>(A.val);
  const int lane = threadIdx.x & (L - 1);
  const int gw = (threadIdx.x & 31) / L;                  // group in warp
  const unsigned gmask = (L == 32) ? 0xffffffffu
                                   : (((1u << L) - 1u) << (gw * L));
  const long long gid = ((long long)blockIdx.x * kThreads + threadIdx.x) / L;
  const long long ngroups = (long long)gridDim.x * kThreads / L;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  for (long long r = gid; r < A.n; r += ngroups) {
    const int row = (int)r;
    const int k0 = __ldg(A.rowptr + row), k1 = __ldg(A.rowptr + row + 1);
    XT sum = XT(0);
    for (int base = k0; base < k1; base += L) {
      const int k = base + lane;
      XT p = XT(0);
      if (k < k1) p = mul_rn((XT)__ldg(Aval + k), __ldg(io.x + __ldg(A.col + k)));
      const int cnt = min(L, k1 - base);
#pragma unroll
      for (int q = 0; q < L; ++q) {
        const XT v = __shfl_sync(gmask, p, q, L);
        if (q < cnt) sum = add_rn(sum, v);
      }
    }
    if (lane == 0) {
      XT y = sum, bv = XT(0), w0 = XT(0), w1 = XT(0);
      if (io.b) bv = io.b[row];
      if (io.mode == 1) y = add_rn(bv, -sum);
      io.y[row] = y;
      if (io.y2) io.y2[row] = y;
      if (ND > 0) {
        if (io.w0) w0 = io.w0[row];
        if (io.w1) w1 = io.w1[row];
#pragma unroll
        for (int d = 0; d < ND; ++d)
          acc[d] += (double)spmv_operand(io.dot[d][0], y, bv, w0, w1) *
                    (double)spmv_operand(io.dot[d][1], y, bv, w0, w1);
      }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

}  // namespace bk
