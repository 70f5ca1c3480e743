// K1 (pipelined tile): CSR SpMV with TMA bulk copies.
//
// A persistent CTA walks its row blocks; for each it stages the block's
// column indices and values into shared memory with two 1-D bulk copies
// (cp.async.bulk, mbarrier transaction counting), double-buffered: the copy
// of the next row block is in flight while the current one is summed.  Each
// thread then sums one row from shared memory, gathering x, left to right
// without FMA -- the reference's dcsrgemm0 order, bit-identical in FP64.
// Rows longer than a tile take the CTA-wide path of k_spmv.
//
// Every mbarrier wait is bounded: after kWaitLimit polls the kernel lets
// its copies in flight land (again bounded), records an error in the
// control block (done, ret = -3) and stops.
#pragma once
#include "dev_common.cuh"

namespace bk {

constexpr unsigned kWaitLimit = 1u << 22;
constexpr int kStageEnt = kTileNnz + 8;   // entries per stage buffer

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned cnt) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(cnt) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar,
                                               unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar,
                                              unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// 1-D bulk copy global -> shared, completion counted on `bar`.  Addresses
// 16-byte aligned, size a multiple of 16 bytes.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src,
                                         unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename VT, typename XT, int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_spmv_tma(CsrH A, SpmvH<XT> io, Red rd) {
  if (skip(rd)) return;
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ XT wsum[kWarps];
  __shared__ int abort_flag;
  const VT* __restrict__ Aval = static_cast<const VT*>(A.val);
  int* scol[2];
  VT* sval[2];
  for (int s = 0; s < 2; ++s) {
    unsigned char* base = dsm + s * kStageEnt * (sizeof(int) + sizeof(VT));
    scol[s] = reinterpret_cast<int*>(base);
    sval[s] = reinterpret_cast<VT*>(base + kStageEnt * sizeof(int));
  }
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // Tile of row block `blk`: entries [a0, a1), both multiples of 4.
  auto tile_range = [&](int blk, int& a0, int& a1, bool& longrow) {
    const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
    const int k0 = __ldg(A.rowptr + r0), k1 = __ldg(A.rowptr + r1);
    longrow = (r1 - r0 == 1) && (k1 - k0 > kTileNnz);
    a0 = k0 & ~3;
    a1 = (k1 + 3) & ~3;
    if (a1 < a0 + 4) a1 = a0 + 4;   // never an empty copy (arrays are padded)
  };
  auto issue = [&](int a0, int a1, int s) {
    const unsigned cb = (unsigned)(a1 - a0) * sizeof(int);
    const unsigned vb = (unsigned)(a1 - a0) * sizeof(VT);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[s], cb + vb);
    bulk_g2s(scol[s], A.col + a0, cb, &bar[s]);
    bulk_g2s(sval[s], Aval + a0, vb, &bar[s]);
  };

  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  unsigned phase[2] = {0u, 0u};
  bool pending[2] = {false, false};   // thread 0: a copy in flight per stage
  if (tid == 0 && (int)blockIdx.x < A.nrb) {
    int a0, a1;
    bool lr;
    tile_range(blockIdx.x, a0, a1, lr);
    if (!lr) {
      issue(a0, a1, 0);
      pending[0] = true;
    }
  }

  int it = 0;
  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x, ++it) {
    const int s = it & 1;
    const int nxt = blk + gridDim.x;
    if (tid == 0 && nxt < A.nrb) {
      int n0, n1;
      bool nl;
      tile_range(nxt, n0, n1, nl);
      if (!nl) {
        issue(n0, n1, s ^ 1);
        pending[s ^ 1] = true;
      }
    }
    const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
    int a0, a1;
    bool longrow;
    tile_range(blk, a0, a1, longrow);
    XT sum = XT(0);
    int row = -1;
    if (longrow) {
      const int k0 = __ldg(A.rowptr + r0), k1 = __ldg(A.rowptr + r1);
      XT p = XT(0);
      for (int k = k0 + tid; k < k1; k += kThreads)
        p = fma_rn((XT)__ldg(Aval + k), __ldg(io.x + __ldg(A.col + k)), p);
      p = sizeof(XT) == 8 ? (XT)warp_sum((double)p) : (XT)warp_sumf((float)p);
      if ((tid & 31) == 0) wsum[tid >> 5] = p;
      __syncthreads();
      if (tid == 0) {
        XT t = XT(0);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += wsum[w];
        sum = t;
        row = r0;
      }
    } else {
      unsigned tries = 0;
      while (!mbar_try_wait(&bar[s], phase[s])) {
        if (++tries > kWaitLimit) {
          abort_flag = 1;
          break;
        }
      }
      phase[s] ^= 1u;
      pending[s] = false;
      __syncthreads();   // abort_flag is uniform from here on
      if (!abort_flag && tid < r1 - r0) {
        row = r0 + tid;
        const int s0 = __ldg(A.rowptr + row) - a0;
        const int s1 = __ldg(A.rowptr + row + 1) - a0;
        const int* cs = scol[s];
        const VT* vs = sval[s];
        int k = s0;
        for (; k + 4 <= s1; k += 4) {
          const XT x0 = __ldg(io.x + cs[k]), x1 = __ldg(io.x + cs[k + 1]);
          const XT x2 = __ldg(io.x + cs[k + 2]), x3 = __ldg(io.x + cs[k + 3]);
          sum = add_rn(sum, mul_rn((XT)vs[k], x0));
          sum = add_rn(sum, mul_rn((XT)vs[k + 1], x1));
          sum = add_rn(sum, mul_rn((XT)vs[k + 2], x2));
          sum = add_rn(sum, mul_rn((XT)vs[k + 3], x3));
        }
        for (; k < s1; ++k) sum = add_rn(sum, mul_rn((XT)vs[k], __ldg(io.x + cs[k])));
      }
    }
    __syncthreads();   // stage s fully consumed before it is refilled
    if (abort_flag) break;
    if (row >= 0) {
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
  if (abort_flag) {
    if (tid == 0) {
      for (int q = 0; q < 2; ++q) {
        unsigned tries = 0;
        while (pending[q] && !mbar_try_wait(&bar[q], phase[q]) &&
               ++tries < kWaitLimit) {
        }
      }
      rd.ctl->ret = -3;
      rd.ctl->done = 1;
    }
    return;
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

}  // namespace bk
