// K1: CSR sparse matrix-vector product, y = A x, for the single-vector
// methods (reference src/matvec.c:11-53 dcsrgemm0 'n' and, after
// transposition / symmetric expansion at upload, 't' and dcsrsymm0).
//
// Tile kernel.  Rows are pre-partitioned into row blocks of at most
// kTileRows rows and kTileNnz stored entries (a row longer than that is a
// block by itself).  A CTA streams its block's column indices and values
// with 16-byte vector loads (int4 / double2 / float4) through the read-only
// path, gathers x, and stages the products in shared memory; then one
// thread per row sums its products left to right.  The row sum therefore
// uses exactly the reference's order (y = 0; y += a_k x_k, k ascending, no
// FMA contraction), so the FP64 product is bit-identical to dcsrgemm0.
// Long rows are reduced by the whole CTA with warp shuffles.
//
// The epilogue can form a residual (y = b - A x), write a second copy of y,
// and accumulate up to three dot products among {y, b, w0, w1} into the
// solver's scalar slots (finish_reduction), so a following
// "alpha = rho / (r~, A p)" needs no extra pass over memory.
#pragma once
#include "dev_common.cuh"

namespace bk {

// Row-block limits kTileNnz / kTileRows: kernel_api.h.

// A: CsrH (kernel_api.h): rowptr (n + 1), col and val padded to a multiple
// of 4 entries (pad entries: column 0, value 0), rb = nrb + 1 row-block
// starts.  io: SpmvH; dot operand codes 0 = y (result), 1 = b, 2 = w0,
// 3 = w1.

template <typename XT>
__device__ __forceinline__ XT spmv_operand(int code, XT y, XT b, XT w0, XT w1) {
  return code == 0 ? y : code == 1 ? b : code == 2 ? w0 : w1;
}

template <typename VT, typename XT>
__device__ __forceinline__ void load4(const VT* val, int kb, VT (&v)[4]);
template <>
__device__ __forceinline__ void load4<double, double>(const double* val, int kb,
                                                      double (&v)[4]) {
  double2 a = __ldg(reinterpret_cast<const double2*>(val + kb));
  double2 b = __ldg(reinterpret_cast<const double2*>(val + kb + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <>
__device__ __forceinline__ void load4<float, float>(const float* val, int kb,
                                                   float (&v)[4]) {
  float4 a = __ldg(reinterpret_cast<const float4*>(val + kb));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

// VT: matrix value type; XT: vector type (the accumulation type is XT).
template <typename VT, typename XT, int ND>
__global__ void __launch_bounds__(kThreads, 8)
k_spmv(CsrH A, SpmvH<XT> io, Red rd) {
  const VT* __restrict__ Aval = static_cast<const VT*>(A.val);
  if (skip(rd)) return;
  __shared__ XT prod[kTileNnz + 8];
  __shared__ XT wsum[kWarps];
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const int tid = threadIdx.x;

  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x) {
    const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
    const int k0 = __ldg(A.rowptr + r0), k1 = __ldg(A.rowptr + r1);
    // This thread's epilogue operands (b, w0, w1 of its row), loaded now so
    // their latency overlaps the tile's loads instead of following them.
    XT bv = XT(0), w0 = XT(0), w1 = XT(0);
    if (tid < r1 - r0) {
      const int myrow = r0 + tid;
      if (io.b) bv = io.b[myrow];
      if (ND > 0 && io.w0) w0 = io.w0[myrow];
      if (ND > 0 && io.w1) w1 = io.w1[myrow];
    }
    XT sum = XT(0);
    int row = -1;
    if (r1 - r0 == 1 && k1 - k0 > kTileNnz) {
      // One long row: CTA-wide strided sum, warp-shuffle + smem tree.
      XT s = XT(0);
      for (int k = k0 + tid; k < k1; k += kThreads)
        s = fma_rn((XT)__ldg(Aval + k), __ldg(io.x + __ldg(A.col + k)), s);
      s = sizeof(XT) == 8 ? (XT)warp_sum((double)s) : (XT)warp_sumf((float)s);
      if ((tid & 31) == 0) wsum[tid >> 5] = s;
      __syncthreads();
      if (tid == 0) {
        XT t = XT(0);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += wsum[w];
        sum = t;
        row = r0;
      }
      __syncthreads();
    } else {
      const int a0 = k0 & ~3;
      const int npk = (k1 - a0 + 3) >> 2;
      for (int q = tid; q < npk; q += kThreads) {
        const int kb = a0 + 4 * q;
        const int4 c4 = __ldg(reinterpret_cast<const int4*>(A.col + kb));
        VT v[4];
        load4<VT, XT>(Aval, kb, v);
        const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = kb + e;
          if (k >= k0 && k < k1)
            prod[k - a0] = mul_rn((XT)v[e], __ldg(io.x + cc[e]));
        }
      }
      __syncthreads();
      if (tid < r1 - r0) {
        row = r0 + tid;
        const int s0 = __ldg(A.rowptr + row) - a0;
        const int s1 = __ldg(A.rowptr + row + 1) - a0;
        for (int k = s0; k < s1; ++k) sum = add_rn(sum, prod[k]);
      }
      __syncthreads();
    }
    if (row >= 0) {
      if (io.shift != 0.0) sum = add_rn(sum, mul_rn((XT)io.shift, io.x[row]));
      XT y = sum;
      if (io.mode == 1) y = add_rn(bv, -sum);
      io.y[row] = y;
      if (io.y2) io.y2[row] = y;
      if (ND > 0) {
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
