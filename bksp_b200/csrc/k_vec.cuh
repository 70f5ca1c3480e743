// K3: fused level-1 kernels -- one pass computing up to kLcMaxOut linear
// combinations of up to kLcMaxIn vectors with scalar-slot coefficients, and
// up to kMaxDots dot products of the results, reduced in FP64 (the
// reference's cblas_daxpy / dscal / dcopy / ddot / dnrm2 sequences, e.g.
// src/bicgstabl.c:60-122, fused per recurrence step).
//
// Terms are applied in input order: the first present term is a rounded
// product, every further term a fused multiply-add -- the rounding of a
// dscal / dcopy followed by FMA-based daxpy calls on the reference's CPU.
// Inputs stream through one at a time with the next two loads in flight,
// so register use grows with the number of outputs and dots, not with the
// number of inputs.
// Operands are streamed as 16-byte packets (double2 / float4); lengths are
// padded to a multiple of 64 and padding entries are zero in every vector.
#pragma once
#include "dev_common.cuh"

namespace bk {

// Input i's packet q (advanced by `off` when i repeats per batch rep).
template <typename T>
__device__ __forceinline__ void load_in(const LcH<T>& d, int i, long long off,
                                        long long q, T* v) {
  const T* p = d.in[i] + ((d.in_rep_mask >> i) & 1u ? off : 0);
  unpack<T>(reinterpret_cast<const typename Pack<T>::V*>(p)[q], v);
}

template <typename T, int MI, int MO, int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_lincomb(const LcH<T> d, Red rd) {
  if (skip(rd)) return;
  using PV = typename Pack<T>::V;
  constexpr int P = Pack<T>::N;
  constexpr int D = 3;   // input packets in flight per thread
  __shared__ T cs[MO][MI];
  __shared__ unsigned pres[MO];
  if (threadIdx.x < MO) {
    unsigned m = 0;
    for (int i = 0; i < MI; ++i)
      if (threadIdx.x < d.nout && i < d.nin && d.c[threadIdx.x][i].op) m |= 1u << i;
    pres[threadIdx.x] = m;
  }
  for (int t = threadIdx.x; t < MO * MI; t += kThreads) {
    const int o = t / MI, i = t % MI;
    cs[o][i] = (o < d.nout && i < d.nin) ? (T)eval_cf(d.c[o][i], rd.S) : T(0);
  }
  __syncthreads();
  unsigned pm[MO];
#pragma unroll
  for (int o = 0; o < MO; ++o) pm[o] = pres[o];

  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < ND; ++k) acc[k] = 0.0;

  const long long npk = d.n / P;
  const long long gstride = (long long)gridDim.x * kThreads;
  for (int rep = 0; rep < d.reps; ++rep) {
    const long long off = (long long)rep * d.stride;
    for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < npk;
         q += gstride) {
      // Inputs are folded into the output accumulators one at a time, in
      // input order, while the loads of the next D - 1 inputs are already
      // in flight (a ring of D packets), so only the outputs, the dot
      // operands and D packets stay live.
      T r[MO][P], da[ND > 0 ? ND : 1][P], db[ND > 0 ? ND : 1][P];
      bool first[MO];
#pragma unroll
      for (int o = 0; o < MO; ++o) first[o] = true;
      T ring[D][P];
#pragma unroll
      for (int i = 0; i < D - 1; ++i)
        if (i < MI && i < d.nin) load_in(d, i, off, q, ring[i]);
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        if (i < d.nin) {
          const int ahead = i + D - 1;
          if (ahead < MI && ahead < d.nin) load_in(d, ahead, off, q, ring[ahead % D]);
          const T* v = ring[i % D];
#pragma unroll
          for (int o = 0; o < MO; ++o) {
            if ((pm[o] >> i) & 1u) {
              const T cf = cs[o][i];
#pragma unroll
              for (int e = 0; e < P; ++e)
                r[o][e] = first[o] ? mul_rn(cf, v[e]) : fma_rn(cf, v[e], r[o][e]);
              first[o] = false;
            }
          }
#pragma unroll
          for (int k = 0; k < ND; ++k) {
            if (d.dot[k][0] == i) {
#pragma unroll
              for (int e = 0; e < P; ++e) da[k][e] = v[e];
            }
            if (d.dot[k][1] == i) {
#pragma unroll
              for (int e = 0; e < P; ++e) db[k][e] = v[e];
            }
          }
        }
      }
#pragma unroll
      for (int o = 0; o < MO; ++o) {
        if (o < d.nout) {
          if (first[o]) {
#pragma unroll
            for (int e = 0; e < P; ++e) r[o][e] = T(0);
          }
          T* p = d.out[o] + ((d.out_rep_mask >> o) & 1u ? off : 0);
          reinterpret_cast<PV*>(p)[q] = repack<T>(r[o]);
#pragma unroll
          for (int k = 0; k < ND; ++k) {
            if (d.dot[k][0] == d.nin + o) {
#pragma unroll
              for (int e = 0; e < P; ++e) da[k][e] = r[o][e];
            }
            if (d.dot[k][1] == d.nin + o) {
#pragma unroll
              for (int e = 0; e < P; ++e) db[k][e] = r[o][e];
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < ND; ++k) {
#pragma unroll
        for (int e = 0; e < P; ++e) acc[k] += (double)da[k][e] * (double)db[k][e];
      }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// All pairwise dot products <v_i, v_j>, i <= j < M, of M vectors in one
// pass (FP64 accumulation), pair (i, j) reduced into S[out + idx] with idx
// running over i, then j >= i.  The one-pass minimal-residual step of
// BiCGSTAB(l) (its Gram matrix of r_0..r_l).
template <typename T, int M>
__global__ void __launch_bounds__(kThreads, (M > 2 ? 2 : 4))
k_gram_vec(const GramH<T> g, Red rd) {
  if (skip(rd)) return;
  using PV = typename Pack<T>::V;
  constexpr int P = Pack<T>::N;
  constexpr int NP = M * (M + 1) / 2;
  double acc[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) acc[q] = 0.0;
  const long long npk = g.n / P;
  const long long stride = (long long)gridDim.x * kThreads;
  // Two packets per thread and sweep: 2 M independent 16-byte loads in
  // flight before the dot products consume them.
  for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < npk;
       q += 2 * stride) {
    const long long q2 = q + stride;
    T v[2][M][P];
#pragma unroll
    for (int i = 0; i < M; ++i) unpack<T>(reinterpret_cast<const PV*>(g.v[i])[q], v[0][i]);
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (q2 < npk) {
        unpack<T>(reinterpret_cast<const PV*>(g.v[i])[q2], v[1][i]);
      } else {
#pragma unroll
        for (int e = 0; e < P; ++e) v[1][i][e] = T(0);
      }
    }
    int idx = 0;
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
      for (int j = i; j < M; ++j) {
        double s = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int e = 0; e < P; ++e) s += (double)v[h][i][e] * (double)v[h][j][e];
        acc[idx++] += s;
      }
  }
  finish_reduction<NP>(acc, rd);
}

}  // namespace bk
