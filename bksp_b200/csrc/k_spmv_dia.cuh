// K1 (diagonal form): y = A x for operators whose stored entries lie on at
// most kDiaMax diagonals (stencil matrices such as the 5- and 7-point
// convection-diffusion operators).  The values are stored diagonal by
// diagonal (nd x stride, zero where a row has no entry on that diagonal)
// with one mask byte per row, so the product streams values with 16-byte
// coalesced loads and needs no column indices (4 bytes fewer per stored
// entry than CSR, against one mask byte per row and the zero fill).
//
// Each thread owns 4 consecutive rows (16-byte value packets per diagonal).
// A row adds its products in ascending diagonal order, which is its
// ascending column order, skipping diagonals its mask does not hold:
// y = 0; y += a_k x_k over the stored entries, k ascending,
// no FMA -- the CSR order of reference src/matvec.c:11-53 (dcsrgemm0), so
// FP64 results are bit-identical to the tile kernel's and the reference's.
// (Only operators whose rows list their columns in ascending order get a
// diagonal form, see runtime.cpp: dia_wanted.)
//
// The x loads depend only on the row index and the offset (bounds checked
// against n), not on the mask, so every load of a thread is independent
// and in flight together; diagonals whose offset is a multiple of the
// 16-byte packet (0, +-nx, +-nx*ny on a grid) read x with vector loads.
// Epilogue as in k_spmv: y = A x or y = b - A x, an optional second copy of
// y, up to three dot products.
#pragma once
#include "dev_common.cuh"
#include "k_spmv.cuh"

namespace bk {

template <int R>
__device__ __forceinline__ unsigned load_mask(const unsigned char* m, int i0);
template <>
__device__ __forceinline__ unsigned load_mask<4>(const unsigned char* m, int i0) {
  return __ldg(reinterpret_cast<const unsigned*>(m + i0));
}

// Four consecutive elements p[i0 .. i0+3] with 16-byte loads (p + i0 16-byte
// aligned): one float4, or two double2.
template <typename T>
__device__ __forceinline__ void load_rows(const T* p, int i0, T (&v)[4]);
template <>
__device__ __forceinline__ void load_rows<float>(const float* p, int i0,
                                                 float (&v)[4]) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(p + i0));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
template <>
__device__ __forceinline__ void load_rows<double>(const double* p, int i0,
                                                  double (&v)[4]) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p + i0));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p + i0 + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <typename T>
__device__ __forceinline__ void store_rows(T* p, int i0, const T (&v)[4]);
template <>
__device__ __forceinline__ void store_rows<float>(float* p, int i0,
                                                  const float (&v)[4]) {
  *reinterpret_cast<float4*>(p + i0) = make_float4(v[0], v[1], v[2], v[3]);
}
template <>
__device__ __forceinline__ void store_rows<double>(double* p, int i0,
                                                   const double (&v)[4]) {
  *reinterpret_cast<double2*>(p + i0) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + i0 + 2) = make_double2(v[2], v[3]);
}

// Rows i0 .. i0+3 of an operand vector: vector loads when all four rows
// exist (vectors of n elements need not be padded), else per-row loads.
template <typename T>
__device__ __forceinline__ void load_opnd(const T* p, int i0, int n, T (&v)[4]) {
  if (i0 + 4 <= n) {
    load_rows<T>(p, i0, v);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = i0 + e < n ? p[i0 + e] : T(0);
  }
}

// x[j0 .. j0+3], zero outside [0, n).  When the diagonal's offset keeps j0
// on a 16-byte packet boundary (offset a multiple of 4 floats / 2 doubles)
// and the four entries exist, vector loads; else per-element loads.
template <typename T>
__device__ __forceinline__ void load_x(const T* __restrict__ x, int j0, int o,
                                       int n, T (&v)[4]) {
  constexpr int P = 16 / (int)sizeof(T);
  if ((o & (P - 1)) == 0 && j0 >= 0 && j0 + 4 <= n) {
    load_rows<T>(x, j0, v);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int j = j0 + e;
      v[e] = (j >= 0 && j < n) ? __ldg(x + j) : T(0);
    }
  }
}

template <typename VT, typename XT, int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_spmv_dia(CsrH A, SpmvH<XT> io, Red rd) {
  constexpr int R = 4;   // rows per thread
  static_assert(sizeof(VT) == sizeof(XT), "one precision per operator");
  if (skip(rd)) return;
  const VT* __restrict__ V = static_cast<const VT*>(A.dia.val);
  const long long stride = A.dia.stride;
  const int nd = A.dia.nd, n = A.n;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const int ngroups = (n + R - 1) / R;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < ngroups;
       g += gridDim.x * kThreads) {
    const int i0 = g * R;
    const unsigned m = load_mask<R>(A.dia.mask, i0);
    XT bv[R], w0[R], w1[R];
    if (io.b) load_opnd<XT>(io.b, i0, n, bv);
    else
#pragma unroll
      for (int e = 0; e < R; ++e) bv[e] = XT(0);
    if (ND > 0 && io.w0) load_opnd<XT>(io.w0, i0, n, w0);
    else
#pragma unroll
      for (int e = 0; e < R; ++e) w0[e] = XT(0);
    if (ND > 0 && io.w1) load_opnd<XT>(io.w1, i0, n, w1);
    else
#pragma unroll
      for (int e = 0; e < R; ++e) w1[e] = XT(0);
    XT sum[R];
#pragma unroll
    for (int e = 0; e < R; ++e) sum[e] = XT(0);
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d) {
      if (d < nd) {
        VT v[R];
        load_rows<VT>(V + d * stride, i0, v);
        const int o = A.dia.off[d];
        XT xv[R];
        load_x<XT>(io.x, i0 + o, o, n, xv);
#pragma unroll
        for (int e = 0; e < R; ++e)
          if ((m >> (8 * e + d)) & 1u) sum[e] = add_rn(sum[e], mul_rn((XT)v[e], xv[e]));
      }
    }
    if (io.shift != 0.0) {   // (A + shift I) x: + shift x_i after the row sum
      XT xo[R];
      load_opnd<XT>(io.x, i0, n, xo);
#pragma unroll
      for (int e = 0; e < R; ++e) sum[e] = add_rn(sum[e], mul_rn((XT)io.shift, xo[e]));
    }
    XT y[R];
#pragma unroll
    for (int e = 0; e < R; ++e) y[e] = io.mode == 1 ? add_rn(bv[e], -sum[e]) : sum[e];
    if (i0 + R <= n) {
      store_rows<XT>(io.y, i0, y);
      if (io.y2) store_rows<XT>(io.y2, i0, y);
    } else {
#pragma unroll
      for (int e = 0; e < R; ++e)
        if (i0 + e < n) {
          io.y[i0 + e] = y[e];
          if (io.y2) io.y2[i0 + e] = y[e];
        }
    }
    if (ND > 0) {
#pragma unroll
      for (int e = 0; e < R; ++e)
        if (i0 + e < n) {
#pragma unroll
          for (int d = 0; d < ND; ++d)
            acc[d] += (double)spmv_operand(io.dot[d][0], y[e], bv[e], w0[e], w1[e]) *
                      (double)spmv_operand(io.dot[d][1], y[e], bv[e], w0[e], w1[e]);
        }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// Diagonal-form product with fused neighbouring updates (kernel_api.h:
// SpmvFuseH).  Same row order and rounding as k_spmv_dia for the product;
// the gathered input x_j = ca xa_j + cb xb_j is formed per element, exactly
// as the row that owns j forms (and stores) it.
template <typename T, int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_spmv_dia_fused(CsrH A, SpmvFuseH<T> f, Red rd) {
  constexpr int R = 4;
  if (skip(rd)) return;
  const T* __restrict__ V = static_cast<const T*>(A.dia.val);
  const long long stride = A.dia.stride;
  const int nd = A.dia.nd, n = A.n;
  const T ca = (T)eval_cf(f.ca, rd.S), cb = f.xb ? (T)eval_cf(f.cb, rd.S) : T(0);
  const T c0 = f.fo ? (T)eval_cf(f.c0, rd.S) : T(0);
  const T c1 = (f.fo && f.f1) ? (T)eval_cf(f.c1, rd.S) : T(0);
  const bool hb = f.xb != nullptr;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const int ngroups = (n + R - 1) / R;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < ngroups;
       g += gridDim.x * kThreads) {
    const int i0 = g * R;
    const unsigned m = load_mask<R>(A.dia.mask, i0);
    T sum[R];
#pragma unroll
    for (int e = 0; e < R; ++e) sum[e] = T(0);
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d) {
      if (d < nd) {
        T v[R];
        load_rows<T>(V + d * stride, i0, v);
        const int o = A.dia.off[d];
        T xa[R], xb[R];
        load_x<T>(f.xa, i0 + o, o, n, xa);
        if (hb) load_x<T>(f.xb, i0 + o, o, n, xb);
#pragma unroll
        for (int e = 0; e < R; ++e) {
          const T xv = hb ? fma_rn(cb, xb[e], mul_rn(ca, xa[e])) : mul_rn(ca, xa[e]);
          if ((m >> (8 * e + d)) & 1u) sum[e] = add_rn(sum[e], mul_rn(v[e], xv));
        }
      }
    }
    // The row's own x, product and second update.
    T xo[R], xa[R], xb[R], fv[R];
    load_opnd<T>(f.xa, i0, n, xa);
    if (hb) load_opnd<T>(f.xb, i0, n, xb);
#pragma unroll
    for (int e = 0; e < R; ++e)
      xo[e] = hb ? fma_rn(cb, xb[e], mul_rn(ca, xa[e])) : mul_rn(ca, xa[e]);
    if (f.fo) {
      T a0[R], a1[R];
      load_opnd<T>(f.f0, i0, n, a0);
      if (f.f1) load_opnd<T>(f.f1, i0, n, a1);
#pragma unroll
      for (int e = 0; e < R; ++e)
        fv[e] = f.f1 ? fma_rn(c1, a1[e], mul_rn(c0, a0[e])) : mul_rn(c0, a0[e]);
    } else {
#pragma unroll
      for (int e = 0; e < R; ++e) fv[e] = T(0);
    }
    if (i0 + R <= n) {
      store_rows<T>(f.y, i0, sum);
      if (f.xe) store_rows<T>(f.xe, i0, xo);
      if (f.fo) store_rows<T>(f.fo, i0, fv);
    } else {
#pragma unroll
      for (int e = 0; e < R; ++e)
        if (i0 + e < n) {
          f.y[i0 + e] = sum[e];
          if (f.xe) f.xe[i0 + e] = xo[e];
          if (f.fo) f.fo[i0 + e] = fv[e];
        }
    }
    if (ND > 0) {
#pragma unroll
      for (int e = 0; e < R; ++e)
        if (i0 + e < n) {
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const int a = f.dot[d][0], b = f.dot[d][1];
            const T u = a == 0 ? sum[e] : a == 1 ? xo[e] : fv[e];
            const T w = b == 0 ? sum[e] : b == 1 ? xo[e] : fv[e];
            acc[d] += (double)u * (double)w;
          }
        }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// Fill the diagonal form from CSR values (and, when mask is given, the row
// masks): one thread per row; a row's columns ascend, so its diagonal index
// only moves forward.
template <typename T>
__global__ void k_csr2dia(CsrH A, const T* __restrict__ val, T* __restrict__ dval,
                          unsigned char* __restrict__ mask) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int k0 = A.rowptr[i], k1 = A.rowptr[i + 1];
  int d = 0;
  unsigned bits = 0;
  for (int k = k0; k < k1; ++k) {
    const int o = A.col[k] - i;
    while (d < A.dia.nd - 1 && A.dia.off[d] < o) ++d;
    if (A.dia.off[d] == o) {
      dval[d * A.dia.stride + i] = val[k];
      bits |= 1u << d;
    }
  }
  if (mask) mask[i] = (unsigned char)bits;
}

}  // namespace bk
