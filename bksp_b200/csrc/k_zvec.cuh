// Complex (double2 = re, im) kernels of the complex solvers (reference
// src/bicg.c, src/bicgstabl.c, src/blbicgstabl.c, src/shbicgstabl.c, which
// call zcsrgemm0 / zcsrgemm1 and the CBLAS z-routines):
//   k_zlc     fused linear combinations with complex coefficients and
//             complex dots (zaxpy / zscal / zcopy chains + zdotc / dznrm2),
//   k_zspmv   CSR product, the reference's row order and rounding,
//   k_zspmm   block product on row-major blocks,
//   k_zblock  block linear combination with s-by-s complex matrices and
//             Gram products (the n-by-s-by-s zgemm calls),
//   k_zshift  the shifted method's per-shift vector updates.
// Reductions finish through finish_reduction / their own block-major
// partials, so the scalar epilogues (zepilogues.cuh) run as for the real
// solvers.
#pragma once
#include "dev_common.cuh"
#include "solver_defs.h"
#include "zkernel_api.h"
#include "zepi_block_cta.cuh"

namespace bk {

// Complex products without FMA contraction: the reference's C99 complex
// multiply (re = ac - bd, im = ad + bc, each product rounded) and add.
__device__ __forceinline__ double2 zmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 zadd_rn(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
// y + c x with FMAs (linear combinations; not a parity-critical order).
__device__ __forceinline__ double2 zfma(double2 c, double2 x, double2 y) {
  y.x = fma(c.x, x.x, fma(-c.y, x.y, y.x));
  y.y = fma(c.x, x.y, fma(c.y, x.x, y.y));
  return y;
}
__device__ __forceinline__ double2 zmul_f(double2 c, double2 x) {
  return make_double2(fma(c.x, x.x, -c.y * x.y), fma(c.x, x.y, c.y * x.x));
}
// Accumulate one term of a complex dot: conj(u) v (cj) or u v.  The
// imaginary part's two products are rounded separately and subtracted, so a
// vector's dot with itself has an imaginary part of exactly zero.
__device__ __forceinline__ void zdot_acc(double2 u, double2 v, bool cj,
                                         double& re, double& im) {
  if (cj) {
    re = fma(u.x, v.x, fma(u.y, v.y, re));
    im += __dsub_rn(__dmul_rn(u.x, v.y), __dmul_rn(u.y, v.x));
  } else {
    re = fma(u.x, v.x, fma(-u.y, v.y, re));
    im += __dadd_rn(__dmul_rn(u.x, v.y), __dmul_rn(u.y, v.x));
  }
}

// Coefficient of a complex term from the scalar slots.
__device__ __forceinline__ double2 eval_zcf(const ZCfH& c, const double* S) {
  if (c.op == 1) return make_double2(c.kr, c.ki);
  if (c.op == 2) {
    const double re = S[c.s], im = c.conj ? -S[c.s + 1] : S[c.s + 1];
    return make_double2(c.kr * re - c.ki * im, c.kr * im + c.ki * re);
  }
  return make_double2(0.0, 0.0);
}

// ------------------------------------------------------------- k_zlc
// Grid-stride over reps x n, one element per thread and sweep.  All of an
// element's inputs are loaded before the first is used (MI bounds the
// inputs, MO the outputs, both compile-time so the operands stay in
// registers and the loads are in flight together); every output then adds
// its terms in input order.  The operand pointers and the coefficients are
// staged in shared memory first; the dots are reduced as kZDots pairs
// (unused ones are zero).
template <int MI, int MO>
__global__ void __launch_bounds__(kThreads)
k_zlc(ZLcH a, Red rd) {
  if (skip(rd)) return;
  __shared__ double2 cs[kZLcOut][kZLcIn];
  __shared__ const double2* ip[kZLcIn];
  __shared__ double2* op[kZLcOut];
  __shared__ unsigned used[kZLcOut];
  __shared__ int dcode[kZDots][2];
  __shared__ int dconj[kZDots];
  const int t = threadIdx.x;
  if (t < kZLcOut * kZLcIn) {
    const int o = t / kZLcIn, i = t % kZLcIn;
    cs[o][i] = (o < a.nout && i < a.nin) ? eval_zcf(a.c[o][i], rd.S)
                                         : make_double2(0.0, 0.0);
  }
  if (t < kZLcIn) ip[t] = t < a.nin ? a.in[t] : nullptr;
  if (t < kZLcOut) {
    op[t] = t < a.nout ? a.out[t] : nullptr;
    unsigned m = 0;
    if (t < a.nout)
      for (int i = 0; i < a.nin; ++i)
        if (a.c[t][i].op) m |= 1u << i;
    used[t] = m;
  }
  if (t < kZDots) {
    dcode[t][0] = t < a.nd ? a.dot[t][0] : -1;
    dcode[t][1] = t < a.nd ? a.dot[t][1] : -1;
    dconj[t] = a.dconj[t];
  }
  __syncthreads();
  double acc[2 * kZDots];
#pragma unroll
  for (int d = 0; d < 2 * kZDots; ++d) acc[d] = 0.0;
  const long long n = a.n;
  const int nin = a.nin, nout = a.nout, nd = a.nd;
  const unsigned irep = a.in_rep_mask, orep = a.out_rep_mask;
  const long long step = (long long)gridDim.x * kThreads;
  // Up to two elements per thread and sweep (narrow combinations): all of
  // both elements' input loads are in flight together.
  constexpr int UN = MI <= 8 ? 2 : 1;
  for (int rep = 0; rep < a.reps; ++rep) {
    const long long ioff = rep * a.stride;
    for (long long e0 = (long long)blockIdx.x * kThreads + t; e0 < n; e0 += step * UN) {
      double2 v[UN][MI];
#pragma unroll
      for (int q = 0; q < UN; ++q) {
        const long long e = e0 + q * step;
#pragma unroll
        for (int i = 0; i < MI; ++i)
          v[q][i] = (i < nin && e < n)
                        ? __ldg(ip[i] + (((irep >> i) & 1u) ? ioff : 0) + e)
                        : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int q = 0; q < UN; ++q) {
        const long long e = e0 + q * step;
        if (e >= n) break;
        double2 y[MO];
#pragma unroll
        for (int o = 0; o < MO; ++o) {
          y[o] = make_double2(0.0, 0.0);
          if (o < nout) {
            const unsigned u = used[o];
            bool any = false;
#pragma unroll
            for (int i = 0; i < MI; ++i) {
              if ((u >> i) & 1u) {
                y[o] = any ? zfma(cs[o][i], v[q][i], y[o]) : zmul_f(cs[o][i], v[q][i]);
                any = true;
              }
            }
            op[o][(((orep >> o) & 1u) ? ioff : 0) + e] = y[o];
          }
        }
#pragma unroll
        for (int d = 0; d < kZDots; ++d) {
          if (d < nd) {
            double2 du = make_double2(0.0, 0.0), dv = du;
            const int c0 = dcode[d][0], c1 = dcode[d][1];
#pragma unroll
            for (int i = 0; i < MI; ++i) {
              if (c0 == i) du = v[q][i];
              if (c1 == i) dv = v[q][i];
            }
#pragma unroll
            for (int o = 0; o < MO; ++o) {
              if (c0 == 100 + o) du = y[o];
              if (c1 == 100 + o) dv = y[o];
            }
            zdot_acc(du, dv, dconj[d] != 0, acc[2 * d], acc[2 * d + 1]);
          }
        }
      }
    }
  }
  if (nd > 0 || rd.epi) finish_reduction<2 * kZDots>(acc, rd);
}

// ----------------------------------------------------------- k_zspmv
// Complex CSR product on the row blocks of the real tile kernel (at most
// kTileRows rows and kTileNnz entries per block; col and val padded to a
// multiple of 4 entries).  A CTA streams its block's columns (int4) and
// values (double2), gathers x and stages the products a_k x_k (the
// reference's complex multiply, no FMA) in shared memory; one thread per row
// then adds them left to right from zero, src/matvec.c:55-72's order, so the
// product is bit-identical to zcsrgemm0 'n' (and, on the conjugated
// transpose built at upload, to 't').  A row longer than kTileNnz is summed
// by the whole CTA in strided order instead.
__device__ __forceinline__ double2 zspmv_operand(int code, double2 y, double2 b,
                                                 double2 w0) {
  return code == 0 ? y : code == 1 ? b : w0;
}

template <int ND>
__global__ void __launch_bounds__(kThreads, 4)
k_zspmv(CsrH A, ZSpmvH io, Red rd) {
  const double2* __restrict__ val = static_cast<const double2*>(A.val);
  if (skip(rd)) return;
  __shared__ double2 prod[kTileNnz];
  __shared__ double2 wsum[kWarps];
  double acc[ND > 0 ? 2 * ND : 1];
#pragma unroll
  for (int d = 0; d < 2 * ND; ++d) acc[d] = 0.0;
  const int tid = threadIdx.x;
  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x) {
    const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
    const int k0 = __ldg(A.rowptr + r0), k1 = __ldg(A.rowptr + r1);
    double2 bv = make_double2(0.0, 0.0), w0 = make_double2(0.0, 0.0);
    if (tid < r1 - r0) {
      if (io.b) bv = io.b[r0 + tid];
      if (ND > 0 && io.w0) w0 = io.w0[r0 + tid];
    }
    double2 sum = make_double2(0.0, 0.0);
    int row = -1;
    if (r1 - r0 == 1 && k1 - k0 > kTileNnz) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = k0 + tid; k < k1; k += kThreads)
        s = zfma(__ldg(val + k), __ldg(io.x + __ldg(A.col + k)), s);
      s.x = warp_sum(s.x);
      s.y = warp_sum(s.y);
      if ((tid & 31) == 0) wsum[tid >> 5] = s;
      __syncthreads();
      if (tid == 0) {
        double2 t = make_double2(0.0, 0.0);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t = zadd_rn(t, wsum[w]);
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
        const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = kb + e;
          if (k >= k0 && k < k1)
            prod[k - a0] = zmul_rn(__ldg(val + k), __ldg(io.x + cc[e]));
        }
      }
      __syncthreads();
      if (tid < r1 - r0) {
        row = r0 + tid;
        const int s0 = __ldg(A.rowptr + row) - a0;
        const int s1 = __ldg(A.rowptr + row + 1) - a0;
        for (int k = s0; k < s1; ++k) sum = zadd_rn(sum, prod[k]);
      }
      __syncthreads();
    }
    if (row >= 0) {
      // mode 1: tmp = -(A x) then tmp += 1 b (src/bicg.c:108-111): one
      // rounded addition per component.
      double2 y = sum;
      if (io.mode == 1) y = make_double2(__dadd_rn(bv.x, -sum.x), __dadd_rn(bv.y, -sum.y));
      io.y[row] = y;
      if (io.y2) io.y2[row] = y;
#pragma unroll
      for (int d = 0; d < ND; ++d)
        zdot_acc(zspmv_operand(io.dot[d][0], y, bv, w0),
                 zspmv_operand(io.dot[d][1], y, bv, w0), io.dconj[d] != 0,
                 acc[2 * d], acc[2 * d + 1]);
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<2 * ND>(acc, rd);
}

// Complex sliced-ELL product (CsrH::sell with double2 values): one warp
// per 32-row slice, one lane per row walking its entries in CSR order with
// the reference's complex multiply and add, so the result equals k_zspmv's
// (and zcsrgemm0's) bit for bit; coalesced column/value loads, eight
// entries' gathers in flight per lane, padding (column -1) skipped.
template <int ND>
__global__ void __launch_bounds__(kThreads, 3)
k_zspmv_sell(CsrH A, ZSpmvH io, Red rd) {
  if (skip(rd)) return;
  const int* __restrict__ sptr = A.sell.ptr;
  const int* __restrict__ scol = A.sell.col;
  const double2* __restrict__ sval = static_cast<const double2*>(A.sell.val);
  const double2* __restrict__ x = io.x;
  double acc[ND > 0 ? 2 * ND : 1];
#pragma unroll
  for (int d = 0; d < 2 * ND; ++d) acc[d] = 0.0;
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * kThreads) >> 5;
  const double2 z0 = make_double2(0.0, 0.0);
  for (long long sl = gw; sl < A.sell.nslice; sl += nw) {
    const int p0 = __ldg(sptr + sl), p1 = __ldg(sptr + sl + 1);
    const int width = (p1 - p0) >> 5;
    const long long row = sl * 32 + lane;
    const int* cp = scol + p0 + lane;
    const double2* vp = sval + p0 + lane;
    double2 sum = z0;
    for (int k0 = 0; k0 < width; k0 += 8) {   // eight entries per round
      int c[8];
      double2 v[8], xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = k0 + u < width;
        c[u] = in ? __ldg(cp + 32 * (k0 + u)) : -1;
        v[u] = in ? __ldg(vp + 32 * (k0 + u)) : z0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : z0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) sum = zadd_rn(sum, zmul_rn(v[u], xv[u]));
    }
    if (row < A.n) {
      const double2 bv = io.b ? io.b[row] : z0;
      double2 y = sum;
      if (io.mode == 1) y = make_double2(__dadd_rn(bv.x, -sum.x), __dadd_rn(bv.y, -sum.y));
      io.y[row] = y;
      if (io.y2) io.y2[row] = y;
      if (ND > 0) {
        const double2 w0 = io.w0 ? io.w0[row] : z0;
#pragma unroll
        for (int d = 0; d < ND; ++d)
          zdot_acc(zspmv_operand(io.dot[d][0], y, bv, w0),
                   zspmv_operand(io.dot[d][1], y, bv, w0), io.dconj[d] != 0,
                   acc[2 * d], acc[2 * d + 1]);
      }
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<2 * ND>(acc, rd);
}

// ----------------------------------------------------------- k_zspmm
// Y = beta C + alpha A X on row-major complex blocks, one thread per
// (row, column), s <= 16 columns per row group: y = beta c, then
// y += (alpha a_k) x_k entry by entry (src/matvec.c:174-191's order and
// rounding; alpha = +-1 and beta in {0, 1} make those factors exact).
__global__ void __launch_bounds__(kThreads, 4)
k_zspmm(CsrH A, ZSpmmH a, Red rd) {
  if (skip(rd)) return;
  const double2* __restrict__ val = static_cast<const double2*>(A.val);
  const int lane = threadIdx.x & 15;
  const long long grp = ((long long)blockIdx.x * kThreads + threadIdx.x) >> 4;
  const long long ngrp = ((long long)gridDim.x * kThreads) >> 4;
  const int s = a.s;
  if (lane < s) {
    for (long long row = grp; row < A.n; row += ngrp) {
      const long long o = row * s + lane;
      double2 y = make_double2(0.0, 0.0);
      if (a.beta) y = a.C[o];
      const int k0 = __ldg(A.rowptr + row), k1 = __ldg(A.rowptr + row + 1);
      for (int k = k0; k < k1; ++k) {
        double2 av = __ldg(val + k);
        if (a.alpha < 0) av = make_double2(-av.x, -av.y);
        y = zadd_rn(y, zmul_rn(av, __ldg(a.X + (long long)__ldg(A.col + k) * s + lane)));
      }
      a.Y[o] = y;
    }
  }
  if (rd.epi) {
    double none[1] = {0.0};
    finish_reduction<0>(none, rd);
  }
}

// ---------------------------------------------------------- k_zblock
// Tiles of 16 rows; thread (r, c) = (t / 16, t % 16) handles element (r, c)
// of each tile, and entry (r, c) of each Gram product.  Matrix terms
// in[i] M use the s-by-s complex matrix staged in shared memory once per
// CTA; every output adds its terms in input order.
constexpr int kZBlkRows = 16;

__device__ __forceinline__ void zblk_finish(const double* g, int ng, int s,
                                            const double* dd, int nd,
                                            const short* gslot, const Red& rd);

__global__ void __launch_bounds__(kThreads, 3)
k_zblock(ZBlkH a, Red rd) {
  if (skip(rd)) return;
  __shared__ double2 tile[6][kZBlkRows][17];
  __shared__ double2 mat[2][256];
  __shared__ double2 cs[2][4];
  __shared__ int mi[2][4];
  const int s = a.s;
  const int t = threadIdx.x, r = t >> 4, c = t & 15;
  if (t == 0) {
    int nm = 0;
    for (int o = 0; o < 2; ++o)
      for (int i = 0; i < 4; ++i)
        mi[o][i] = (o < a.nout && i < a.nin && a.c[o][i].op && a.mslot[o][i] >= 0 && nm < 2)
                       ? nm++ : -1;
  }
  if (t < 8) {
    const int o = t >> 2, i = t & 3;
    cs[o][i] = (o < a.nout && i < a.nin) ? eval_zcf(a.c[o][i], rd.S) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int o = 0; o < a.nout; ++o)
    for (int i = 0; i < a.nin; ++i)
      if (mi[o][i] >= 0)
        for (int q = t; q < s * s; q += kThreads)
          mat[mi[o][i]][q] = make_double2(rd.S[a.mslot[o][i] + 2 * q],
                                          rd.S[a.mslot[o][i] + 2 * q + 1]);
  __syncthreads();
  double g[4] = {0.0, 0.0, 0.0, 0.0};
  double dd[4] = {0.0, 0.0, 0.0, 0.0};
  const long long ntiles = (a.n + kZBlkRows - 1) / kZBlkRows;
  // The next tile's inputs are loaded into registers while the current
  // tile is computed, so a tile's global loads overlap the previous one's
  // work.
  double2 pre[4];
  auto fetch = [&](long long tl) {
    const long long row = tl * kZBlkRows + r;
    const bool ok = c < s && row < a.n && tl < ntiles;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      pre[i] = (i < a.nin && ok) ? a.in[i][row * s + c] : make_double2(0.0, 0.0);
  };
  fetch(blockIdx.x);
  for (long long tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
    const long long row = tl * kZBlkRows + r;
    const bool valid = c < s && row < a.n;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (i < a.nin) tile[i][r][c] = pre[i];
    __syncthreads();
    fetch(tl + gridDim.x);
    for (int o = 0; o < a.nout; ++o) {
      double2 y = make_double2(0.0, 0.0);
      bool first = true;
      for (int i = 0; i < a.nin; ++i) {
        if (!a.c[o][i].op) continue;
        double2 term;
        if (mi[o][i] >= 0) {
          const double2* M = mat[mi[o][i]];
          double2 z = make_double2(0.0, 0.0);
          for (int b = 0; b < s; ++b) z = zfma(tile[i][r][b], M[b * s + (c < s ? c : 0)], z);
          term = zmul_f(cs[o][i], z);
        } else {
          term = zmul_f(cs[o][i], tile[i][r][c]);
        }
        y = first ? term : make_double2(y.x + term.x, y.y + term.y);
        first = false;
      }
      if (valid) a.out[o][row * s + c] = y;
      tile[4 + o][r][c] = valid ? y : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int q = 0; q < a.ng; ++q) {
      const int u = a.gram[q][0], v = a.gram[q][1];
      const int tu = u < a.nin ? u : 4 + (u - a.nin);
      const int tv = v < a.nin ? v : 4 + (v - a.nin);
      if (r < s && c < s)
        for (int k = 0; k < kZBlkRows; ++k)
          zdot_acc(tile[tu][k][r], tile[tv][k][c], a.gconj[q] != 0, g[2 * q], g[2 * q + 1]);
    }
    for (int d = 0; d < a.nd; ++d) {
      const int u = a.dot[d][0], v = a.dot[d][1];
      const int tu = u < a.nin ? u : 4 + (u - a.nin);
      const int tv = v < a.nin ? v : 4 + (v - a.nin);
      zdot_acc(tile[tu][r][c], tile[tv][r][c], true, dd[2 * d], dd[2 * d + 1]);
    }
    __syncthreads();
  }
  if (a.ng > 0 || a.nd > 0 || rd.epi) zblk_finish(g, a.ng, s, dd, a.nd, a.gslot, rd);
}

// Deterministic grid reduction of the Gram entries (thread t owns entry t
// of each Gram) and the Frobenius dots, in two levels as blk_finish does
// (the last block of each group of kRedGroup blocks sums its group in
// block order, the last group block the group sums in group order):
// block-major partials of kZBlkPart doubles per block; the last block
// writes the sums to the slots and runs the epilogue.
__device__ __forceinline__ void zblk_finish(const double* g, int ng, int s,
                                            const double* dd, int nd,
                                            const short* gslot, const Red& rd) {
  __shared__ double wsum[4][kWarps];
  __shared__ int is_last;
  const int t = threadIdx.x;
  const int nb = gridDim.x;
  const int grp = blockIdx.x / kRedGroup;
  const int b0 = grp * kRedGroup;
  const int gn = min(kRedGroup, nb - b0);
  const int ngrp = (nb + kRedGroup - 1) / kRedGroup;
  double* gpart = rd.part + (long long)kGridCap * kZBlkPart;
  unsigned* gticket = reinterpret_cast<unsigned*>(rd.part + red2_ticket_offset(kZBlkPart));
  double* mine = rd.part + (long long)blockIdx.x * kZBlkPart;
  for (int q = 0; q < ng; ++q) {
    mine[q * 512 + 2 * t] = g[2 * q];
    mine[q * 512 + 2 * t + 1] = g[2 * q + 1];
  }
  for (int d = 0; d < 2 * nd; ++d) {
    const double v = warp_sum(dd[d]);
    if ((t & 31) == 0) wsum[d][t >> 5] = v;
  }
  __syncthreads();
  if (t == 0) {
    for (int d = 0; d < 2 * nd; ++d) {
      double v = 0.0;
      for (int w = 0; w < kWarps; ++w) v += wsum[d][w];
      mine[1024 + d] = v;
    }
    __threadfence();
    is_last = atomicAdd(gticket + grp, 1u) == (unsigned)gn - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // Level 1: this group's blocks.
  const double* gp = rd.part + (long long)b0 * kZBlkPart;
  double* gout = gpart + (long long)grp * kZBlkPart;
  for (int q = 0; q < ng; ++q) {
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int b = 0; b < kRedGroup; ++b)
      if (b < gn) {
        re += __ldcg(gp + (long long)b * kZBlkPart + q * 512 + 2 * t);
        im += __ldcg(gp + (long long)b * kZBlkPart + q * 512 + 2 * t + 1);
      }
    gout[q * 512 + 2 * t] = re;
    gout[q * 512 + 2 * t + 1] = im;
  }
  if (t < 2 * nd) {
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < kRedGroup; ++b)
      if (b < gn) v += __ldcg(gp + (long long)b * kZBlkPart + 1024 + t);
    gout[1024 + t] = v;
  }
  __syncthreads();
  if (t == 0) {
    gticket[grp] = 0u;
    __threadfence();
    is_last = atomicAdd(rd.ticket, 1u) == (unsigned)ngrp - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // Level 2: the groups.
  const int r = t >> 4, c = t & 15;
  for (int q = 0; q < ng; ++q) {
    double re = 0.0, im = 0.0;
#pragma unroll 8
    for (int k = 0; k < ngrp; ++k) {
      re += __ldcg(gpart + (long long)k * kZBlkPart + q * 512 + 2 * t);
      im += __ldcg(gpart + (long long)k * kZBlkPart + q * 512 + 2 * t + 1);
    }
    if (r < s && c < s) {
      rd.S[gslot[q] + 2 * (r * s + c)] = re;
      rd.S[gslot[q] + 2 * (r * s + c) + 1] = im;
    }
  }
  if (t < 2 * nd) {
    double v = 0.0;
#pragma unroll 8
    for (int k = 0; k < ngrp; ++k) v += __ldcg(gpart + (long long)k * kZBlkPart + 1024 + t);
    rd.S[rd.out + t] = v;
  }
  __syncthreads();
  if (t == 0) {
    *rd.ticket = 0u;
    __threadfence();
  }
  // s-by-s algebra on all threads; the scalar epilogues on one
  if (rd.epi && !run_zblock_epilogue_cta(rd, t) && t == 0) run_epilogue(rd);
}

// ---------------------------------------------------------- k_zshift
// All shifts in one pass over the elements (ZShiftH's modes): each thread
// loads the seed residuals it needs for element e once and updates every
// shift's vectors at e.  The per-shift coefficients are staged in shared
// memory (kZMaxShifts entries; mode 2 also kBlMaxL x-coefficients per
// shift).
__global__ void __launch_bounds__(kThreads, 2)
k_zshift(ZShiftH a, Red rd) {
  if (skip(rd)) return;
  __shared__ double2 c0[kZMaxShifts], c1[kZMaxShifts], c2[kZMaxShifts],
      c3[kZMaxShifts];
  __shared__ double2 cx[kZMaxShifts * kBlMaxL];
  __shared__ double2 om[kBlMaxL];
  const double* S = rd.S;
  const int ns = a.ns, l = a.l, j = a.j;
  auto ld2 = [&](int slot) { return make_double2(S[slot], S[slot + 1]); };
  for (int k = threadIdx.x; k < ns; k += kThreads) {
    if (a.mode == 0) {
      c0[k] = ld2(kZShCb + 2 * k);
      c1[k] = ld2(kZShCr + 2 * k);
      c2[k] = ld2(kZShCq + 2 * k);
      c3[k] = ld2(kZShAlpha + 2 * k);
    } else if (a.mode == 1) {
      c0[k] = ld2(kZShCs + 2 * k);
      c1[k] = ld2(kZShCn + 2 * k);
      const double2 sg = ld2(kZShSigma + 2 * k);
      c2[k] = make_double2(-sg.x, -sg.y);
    } else {
      c0[k] = ld2(kZShCp + 2 * k);
      for (int i = 0; i < l; ++i) cx[k * kBlMaxL + i] = ld2(kZShCx + 2 * (k * kBlMaxL + i));
    }
  }
  if (threadIdx.x < l) {
    const double2 w = ld2(kZOmega + 2 * threadIdx.x);
    om[threadIdx.x] = make_double2(-w.x, -w.y);
  }
  __syncthreads();
  const long long np = a.np;
  const long long vs = (long long)(l + 1) * np;   // one shift's P block
  const long long step = (long long)gridDim.x * kThreads;
  for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < np; e += step) {
    double2 rv[kBlMaxL + 1];
#pragma unroll
    for (int i = 0; i <= kBlMaxL; ++i) {
      const bool need = a.mode == 0 ? i <= j : a.mode == 1 ? i == j : i < l;
      rv[i] = need ? __ldg(a.R + i * np + e) : make_double2(0.0, 0.0);
    }
    for (int k = 0; k < ns; ++k) {
      double2* P = a.P + k * vs + e;
      double2* X = a.X + k * np + e;
      if (a.mode == 0) {           // src/shbicgstabl.c:429-441
        double2 p0 = make_double2(0.0, 0.0);
#pragma unroll
        for (int i = 0; i <= kBlMaxL; ++i) {
          if (i <= j) {
            const double2 v = zfma(c1[k], rv[i], zmul_f(c0[k], P[i * np]));
            P[i * np] = v;
            if (i == 0) p0 = v;
          }
        }
        double2 rj = make_double2(0.0, 0.0);
#pragma unroll
        for (int i = 0; i <= kBlMaxL; ++i)
          if (i == j) rj = rv[i];
        P[(j + 1) * np] = zmul_f(c2[k], rj);
        *X = zfma(c3[k], p0, *X);
      } else if (a.mode == 1) {    // :455-463
        double2 rj = make_double2(0.0, 0.0);
#pragma unroll
        for (int i = 0; i <= kBlMaxL; ++i)
          if (i == j) rj = rv[i];
        const double2 t = zfma(c1[k], rj, P[(j + 1) * np]);
        P[(j + 1) * np] = zfma(c2[k], P[j * np], zmul_f(c0[k], t));
      } else {                     // :545-556
        double2 x = *X;
#pragma unroll
        for (int i = 0; i < kBlMaxL; ++i)
          if (i < l) x = zfma(cx[k * kBlMaxL + i], rv[i], x);
        *X = x;
        double2 p = P[0];
        for (int i = 1; i <= l; ++i) p = zfma(om[i - 1], P[i * np], p);
        P[0] = zmul_f(c0[k], p);
      }
    }
  }
  if (rd.epi) {
    double none[1] = {0.0};
    finish_reduction<0>(none, rd);
  }
}

}  // namespace bk
