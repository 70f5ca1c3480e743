// Sliced-ELL SpMV (CsrH::sell, kernel_api.h: SellH) for operators without a
// diagonal form: one warp per slice of 32 consecutive rows, one lane per
// row.  A lane walks its row's entries in CSR order, so the row sum keeps
// the reference's order and rounding (y = 0; y += a_k x_k, no FMA) and the
// product is bit-identical to dcsrgemm0 and to the tile kernel.  Entry k of
// the 32 rows sits in 32 consecutive words, so the column and value loads
// of a warp are single coalesced transactions; eight entries' loads (and
// their x gathers) are issued before the first is added, to keep several
// gathers in flight per lane.  Padding (column -1) is skipped, never added.
// Epilogue as the tile kernel (k_spmv.cuh): b - A x, a copy, + shift x,
// up to three dots among {y, b, w0, w1}.
#pragma once
#include "dev_common.cuh"
#include "k_spmv.cuh"

namespace bk {

template <typename VT, typename XT, int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_spmv_sell(CsrH A, SpmvH<XT> io, Red rd) {
  if (skip(rd)) return;
  const int* __restrict__ sptr = A.sell.ptr;
  const int* __restrict__ scol = A.sell.col;
  const VT* __restrict__ sval = static_cast<const VT*>(A.sell.val);
  const XT* __restrict__ x = io.x;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * kThreads) >> 5;
  for (long long sl = gw; sl < A.sell.nslice; sl += nw) {
    const int p0 = __ldg(sptr + sl), p1 = __ldg(sptr + sl + 1);
    const int width = (p1 - p0) >> 5;
    const long long row = sl * 32 + lane;
    const int* cp = scol + p0 + lane;
    const VT* vp = sval + p0 + lane;
    XT sum = XT(0);
    // Eight entries per round: all column and value loads of the round,
    // then all x gathers, then the ordered adds -- one load round trip per
    // round (one per slice for rows of up to eight entries).
    for (int k0 = 0; k0 < width; k0 += 8) {
      int c[8];
      VT v[8];
      XT xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = k0 + u < width;
        c[u] = in ? __ldg(cp + 32 * (k0 + u)) : -1;
        v[u] = in ? __ldg(vp + 32 * (k0 + u)) : VT(0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : XT(0);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) sum = add_rn(sum, mul_rn((XT)v[u], xv[u]));
    }
    if (row < A.n) {
      if (io.shift != 0.0) sum = add_rn(sum, mul_rn((XT)io.shift, x[row]));
      const XT bv = io.b ? io.b[row] : XT(0);
      XT y = sum;
      if (io.mode == 1) y = add_rn(bv, -sum);
      io.y[row] = y;
      if (io.y2) io.y2[row] = y;
      if (ND > 0) {
        const XT w0 = io.w0 ? io.w0[row] : XT(0);
        const XT w1 = io.w1 ? io.w1[row] : XT(0);
#pragma unroll
        for (int d = 0; d < ND; ++d)
          acc[d] += (double)spmv_operand(io.dot[d][0], y, bv, w0, w1) *
                    (double)spmv_operand(io.dot[d][1], y, bv, w0, w1);
      }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// Fill the sliced-ELL arrays from the CSR, one thread per (padded) row:
// the row's entries in CSR order, then column -1 / value 0 up to the
// slice's width.
template <typename VT>
__global__ void k_csr2sell(const int* __restrict__ rowptr, const int* __restrict__ col,
                           const VT* __restrict__ val, int n, int nslice,
                           const int* __restrict__ sptr, int* __restrict__ scol,
                           VT* __restrict__ sval) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (long long)nslice * 32) return;
  const long long sl = r >> 5;
  const int lane = (int)(r & 31);
  const int p0 = sptr[sl];
  const int width = (sptr[sl + 1] - p0) >> 5;
  int k0 = 0, len = 0;
  if (r < n) {
    k0 = rowptr[r];
    len = rowptr[r + 1] - k0;
  }
  for (int k = 0; k < width; ++k) {
    const long long o = (long long)p0 + 32LL * k + lane;
    if (k < len) {
      scol[o] = col[k0 + k];
      sval[o] = val[k0 + k];
    } else {
      scol[o] = -1;
      sval[o] = VT{};
    }
  }
}

}  // namespace bk
