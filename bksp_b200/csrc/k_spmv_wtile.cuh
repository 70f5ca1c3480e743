// K1 (warp tile): the row blocks of k_spmv, but every warp works on its own
// 32 rows -- it streams the 16-byte packs covering its rows' entries (int4
// columns, double2 / float4 values), gathers x, stages the products in its
// slice of the CTA's shared buffer and sums its rows in order, with only a
// __syncwarp between the two phases (one CTA barrier per tile, before the
// buffer is reused).  Summation order is the reference's (left to right, no
// FMA): bit-identical FP64 results.
#pragma once
#include "dev_common.cuh"

namespace bk {

template <typename VT, typename XT, int ND>
__global__ void __launch_bounds__(kThreads, 8)
k_spmv_wtile(CsrH A, SpmvH<XT> io, Red rd) {
  if (skip(rd)) return;
  __shared__ XT prod[kTileNnz + 8];
  const VT* __restrict__ Aval = static_cast<const VT*>(A.val);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x) {
    const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
    const int t0 = __ldg(A.rowptr + r0);
    const int ta0 = t0 & ~3;                    // tile base (smem index 0)
    const bool longrow = r1 - r0 == 1 && __ldg(A.rowptr + r1) - t0 > kTileNnz;
    const int wr0 = r0 + warp * 32;
    if (longrow) {
      // One long row: warp 0 reduces it (warp shuffles), in chunks.
      if (warp == 0) {
        const int k1 = __ldg(A.rowptr + r1);
        XT p = XT(0);
        for (int k = t0 + lane; k < k1; k += 32)
          p = fma_rn((XT)__ldg(Aval + k), __ldg(io.x + __ldg(A.col + k)), p);
        p = sizeof(XT) == 8 ? (XT)warp_sum((double)p) : (XT)warp_sumf((float)p);
        if (lane == 0) {
          XT y = p, bv = XT(0), w0 = XT(0), w1 = XT(0);
          if (io.b) bv = io.b[r0];
          if (io.mode == 1) y = add_rn(bv, -p);
          io.y[r0] = y;
          if (io.y2) io.y2[r0] = y;
          if (ND > 0) {
            if (io.w0) w0 = io.w0[r0];
            if (io.w1) w1 = io.w1[r0];
#pragma unroll
            for (int d = 0; d < ND; ++d)
              acc[d] += (double)spmv_operand(io.dot[d][0], y, bv, w0, w1) *
                        (double)spmv_operand(io.dot[d][1], y, bv, w0, w1);
          }
        }
      }
    } else if (wr0 < r1) {
      const int wr1 = min(wr0 + 32, r1);
      const int k0 = __ldg(A.rowptr + wr0), k1 = __ldg(A.rowptr + wr1);
      const int a0 = k0 & ~3;
      const int npk = (k1 - a0 + 3) >> 2;
      for (int q = lane; q < npk; q += 32) {
        const int kb = a0 + 4 * q;
        const int4 c4 = __ldg(reinterpret_cast<const int4*>(A.col + kb));
        VT v[4];
        load4<VT, XT>(Aval, kb, v);
        const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = kb + e;
          if (k >= k0 && k < k1) prod[k - ta0] = mul_rn((XT)v[e], __ldg(io.x + cc[e]));
        }
      }
      __syncwarp();
      const int row = wr0 + lane;
      if (row < wr1) {
        const int s0 = __ldg(A.rowptr + row) - ta0;
        const int s1 = __ldg(A.rowptr + row + 1) - ta0;
        XT sum = XT(0);
        for (int k = s0; k < s1; ++k) sum = add_rn(sum, prod[k]);
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
    // The next tile's slices can overlap this tile's slices of other
    // warps: the buffer is reused only after every warp has read it.
    __syncthreads();
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

}  // namespace bk
