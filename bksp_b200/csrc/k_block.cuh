// Block (multiple right-hand side) kernels: K2 SpMM and K4/K5 fused block
// linear combination + Gram products, for the block methods (reference
// src/blcg.c, src/blbicgstab.c, src/blbicgstabl.c, which call mkl_dcsrmm /
// dcsrgemm1 and n-by-s-by-s cblas_dgemm).
//
// Blocks are n-by-s, s <= 16, stored ROW-major in HBM (row i's s values
// contiguous, 128 bytes at s = 16), so one sparse row gathers whole
// 128-byte rows of X.  s-by-s coefficient matrices live in the scalar slots
// (row-major, M[b][c] at S[slot + b * s + c]).
#pragma once
#include "dev_common.cuh"
#include "epi_block_cta.cuh"

namespace bk {

constexpr int kBlkS = 16;           // max block width
constexpr int kBlkTileRows = 32;    // rows per tile of the block kernel
constexpr int kBlkSub = kBlkTileRows / (kThreads / kBlkS);   // rows per thread
// Tile row stride: a multiple of two elements, so a row's entries can be
// read two at a time (double2 / float2), and not of 16, so the two rows a
// warp reads at once fall in different banks.
constexpr int kBlkTileStride = kBlkS + 2;
template <typename T> struct Pair;
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<float> { using V = float2; };

// ------------------------------------------------------------------ SpMM
// Y = alpha * A X  (mode 0), Y = C + alpha * A X  (mode 1), with the
// reference's per-entry rounding (y += (alpha a_k) x_k, no FMA).  Optional
// Frobenius dots (Y, W) and (Y, Y) into S[out], S[out + 1].
// T = value and block element type (double: the reference-parity path;
// float: the inner solves of the mixed-precision block methods, dots still
// accumulated in FP64).
template <typename T>
struct SpmmArgs {
  const T* X;
  T* Y;
  const T* C;
  const T* W;
  double alpha;
  int mode, s, nd, prec;
};

template <typename T, int ND>
__global__ void __launch_bounds__(kThreads, 8)
k_spmm(CsrH A, SpmmArgs<T> a, Red rd) {
  if (skip(rd)) return;
  const T* __restrict__ val = static_cast<const T*>(A.val);
  const int lane = threadIdx.x & (kBlkS - 1);
  const int grp = (blockIdx.x * kThreads + threadIdx.x) / kBlkS;
  const int ngrp = gridDim.x * kThreads / kBlkS;
  const int s = a.s;
  const T alpha = (T)a.alpha;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  for (int row = grp; row < A.n; row += ngrp) {
    if (lane < s) {
      T y = T(0);
      const int k0 = __ldg(A.rowptr + row), k1 = __ldg(A.rowptr + row + 1);
      for (int k = k0; k < k1; ++k) {
        const T av = mul_rn(alpha, __ldg(val + k));
        y = add_rn(y, mul_rn(av, __ldg(a.X + (long long)__ldg(A.col + k) * s + lane)));
      }
      const long long o = (long long)row * s + lane;
      if (a.mode == 1) y = add_rn(a.C[o], y);
      a.Y[o] = y;
      if (ND > 0) acc[0] += (double)y * (double)a.W[o];
      if (ND > 1) acc[1] += (double)y * (double)y;
    }
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// SpMM on the diagonal form (stencil operators): each row's s values are
// handled by s / V threads with 16-byte loads and stores (V = 2 doubles or
// 4 floats per thread), the row's diagonal value loaded once per diagonal
// and shared by those threads; entries in ascending diagonal (= column)
// order with the reference's rounding (y += (alpha a_k) x_k), so the
// result equals k_spmm's.  Needs s % V == 0 and 16-byte aligned blocks.
template <typename T> struct Vec16;
template <> struct Vec16<double> { using V = double2; static constexpr int N = 2; };
template <> struct Vec16<float> { using V = float4; static constexpr int N = 4; };

template <typename T, int ND>
__global__ void __launch_bounds__(kThreads, 3)
k_spmm_dia(CsrH A, SpmmArgs<T> a, Red rd) {
  if (skip(rd)) return;
  using PV = typename Vec16<T>::V;
  constexpr int VN = Vec16<T>::N;
  const T* __restrict__ V = static_cast<const T*>(A.dia.val);
  const long long stride = A.dia.stride;
  const int s = a.s, nd = A.dia.nd, n = A.n;
  const int tpr = s / VN;                       // threads per row
  const int rows_per_pass = kThreads / tpr;
  const int q = threadIdx.x % tpr, rloc = threadIdx.x / tpr;
  const bool active = rloc < rows_per_pass;     // kThreads % tpr leftovers idle
  const T alpha = (T)a.alpha;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  for (long long row = (long long)blockIdx.x * rows_per_pass + rloc; active && row < n;
       row += (long long)gridDim.x * rows_per_pass) {
    const unsigned m = __ldg(A.dia.mask + row);
    T y[VN];
#pragma unroll
    for (int e = 0; e < VN; ++e) y[e] = T(0);
    // Every diagonal's value and X segment are loaded before the first is
    // used (a row index clamped into range where the row lacks the
    // diagonal: a valid address whose value is then not used), so all of a
    // row's loads are in flight together; the adds keep ascending diagonal
    // order and only the stored entries enter.
    T av[kDiaMax];
    PV xp[kDiaMax];
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d) {
      if (d < nd) {
        long long j = row + A.dia.off[d];
        j = j < 0 ? 0 : (j >= n ? n - 1 : j);
        av[d] = __ldg(V + d * stride + row);
        xp[d] = __ldg(reinterpret_cast<const PV*>(a.X + j * s) + q);
      }
    }
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d) {
      if (d < nd && ((m >> d) & 1u)) {
        const T avd = mul_rn(alpha, av[d]);
        T xv[VN];
        unpack<T>(xp[d], xv);
#pragma unroll
        for (int e = 0; e < VN; ++e) y[e] = add_rn(y[e], mul_rn(avd, xv[e]));
      }
    }
    const long long o = row * s + q * VN;
    if (a.mode == 1) {
      T cv[VN];
      unpack<T>(reinterpret_cast<const PV*>(a.C + o)[0], cv);
#pragma unroll
      for (int e = 0; e < VN; ++e) y[e] = add_rn(cv[e], y[e]);
    }
    reinterpret_cast<PV*>(a.Y + o)[0] = repack<T>(y);
    if (ND > 0) {
      T wv[VN];
      unpack<T>(reinterpret_cast<const PV*>(a.W + o)[0], wv);
#pragma unroll
      for (int e = 0; e < VN; ++e) acc[0] += (double)y[e] * (double)wv[e];
    }
    if (ND > 1)
#pragma unroll
      for (int e = 0; e < VN; ++e) acc[1] += (double)y[e] * (double)y[e];
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

// ---------------------------------------------- block linear combination
// out[o] = sum_i term(o, i) with term = c * in[i] (scalar) or
// c * in[i] * M (M s-by-s from slots, optionally transposed); then up to
// two Gram products G_g = U_g^T V_g (U, V among [in..., out...]) written to
// S[gslot_g + a * s + b], and up to two Frobenius dots.
template <typename T>
struct BlkArgs {
  const T* in[4];
  T* out[2];
  CfH c[2][4];
  short mslot[2][4];     // >= 0: matrix term
  unsigned char trans[2][4];
  int nin, nout, s;
  long long n;           // rows (padded)
  int ng;
  unsigned char gram[2][2];
  short gslot[2];
  int nd;
  unsigned char dot[2][2];
  int prec;
};

__device__ __forceinline__ void blk_finish(const double* g, int ng, int s,
                                           const double* dd, int nd,
                                           const short* gslot, const Red& rd,
                                           double* stage);

// Scalar slots a block epilogue may touch: the common and recurrence
// slots below the first s-by-s cell and the cells kBkG1 .. kBkScr2.  The
// last CTA stages them in shared memory for the epilogue (its s-by-s
// algebra is a long dependent chain of loads and stores; in shared memory
// each costs tens of cycles instead of an L2 round trip) and writes them
// back afterwards.
constexpr int kBlkEpiSlots = bk_cell(19);

template <typename T>
struct BlkSmem {
  T tile[6][kBlkTileRows][kBlkTileStride];
  T mat[2][4][kBlkS * kBlkS];
  T cs[2][4];
};
template <typename T>
constexpr size_t blk_smem_bytes() {
  return sizeof(BlkSmem<T>) > sizeof(double) * kBlkEpiSlots
             ? sizeof(BlkSmem<T>) : sizeof(double) * kBlkEpiSlots;
}

// Terms are formed in T (the block's element type); Gram products and dots
// accumulate in FP64 either way.  Two CTAs per SM (128 registers, no
// spills): measured ~10 % faster than three (80 registers) and ~20 % faster
// than four (64 registers, the tile loop spilling).
template <typename T>
__global__ void __launch_bounds__(kThreads, 2)
k_block(BlkArgs<T> a, Red rd) {
  if (skip(rd)) return;
  // The tiles and matrices share their storage with the epilogue's staged
  // slots (used only after the last tile).
  __shared__ __align__(16) unsigned char raw[blk_smem_bytes<T>()];
  BlkSmem<T>& sm = *reinterpret_cast<BlkSmem<T>*>(raw);
  auto& tile = sm.tile;
  auto& mat = sm.mat;
  auto& cs = sm.cs;
  const int s = a.s;
  const int t = threadIdx.x;
  const int r = t / kBlkS, c = t % kBlkS;   // tile element of this thread
  for (int q = t; q < 2 * 4; q += kThreads) {
    const int o = q / 4, i = q % 4;
    cs[o][i] = (o < a.nout && i < a.nin) ? (T)eval_cf(a.c[o][i], rd.S) : T(0);
  }
  // s-by-s matrices zero-padded to kBlkS x kBlkS (row stride kBlkS): with
  // the tile's columns >= s zero as well, the products below run over all
  // kBlkS terms without a per-term predicate (the padded terms add
  // fma(0, 0, z) = z).
  for (int o = 0; o < a.nout; ++o)
    for (int i = 0; i < a.nin; ++i)
      if (a.mslot[o][i] >= 0)
        for (int q = t; q < kBlkS * kBlkS; q += kThreads) {
          const int b = q / kBlkS, cc = q % kBlkS;
          const int src = a.trans[o][i] ? cc * s + b : b * s + cc;
          mat[o][i][q] = (b < s && cc < s) ? (T)rd.S[a.mslot[o][i] + src] : T(0);
        }
  __syncthreads();
  double gacc[2] = {0.0, 0.0};
  double dacc[2] = {0.0, 0.0};
  // Tiles of kBlkTileRows rows; thread (r, c) handles rows r + 16 k of the
  // tile (k < kBlkSub), column c: all of a tile's loads are issued before
  // its first use.
  const long long ntiles = (a.n + kBlkTileRows - 1) / kBlkTileRows;
  // The next tile's inputs are loaded into registers while the current tile
  // is computed, so each tile's global loads overlap the previous tile's
  // work instead of starting after it.
  T pre[4][kBlkSub];
  auto fetch = [&](long long tl) {
    const long long row0 = tl * kBlkTileRows;
#pragma unroll
    for (int k = 0; k < kBlkSub; ++k) {
      const int rr = r + (kThreads / kBlkS) * k;
      const long long row = row0 + rr;
      const bool valid = c < s && row < a.n && tl < ntiles;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        pre[i][k] = (i < a.nin && valid) ? a.in[i][row * s + c] : T(0);
    }
  };
  fetch(blockIdx.x);
  for (long long tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
    const long long row0 = tl * kBlkTileRows;
#pragma unroll
    for (int k = 0; k < kBlkSub; ++k) {
      const int rr = r + (kThreads / kBlkS) * k;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (i < a.nin) tile[i][rr][c] = pre[i][k];
    }
    __syncthreads();
    fetch(tl + gridDim.x);
    // Outputs: for each term the s-by-s matrix column c is read once into
    // registers and serves all kBlkSub rows of this thread; every element's
    // terms are accumulated in input order, as before.
    // (Both loops are unrolled to their bounds so that every term's
    // parameters and matrices are addressed statically.)
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      if (o >= a.nout) break;
      T y[kBlkSub];
      bool first = true;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (i >= a.nin) break;
        const CfH& cf = a.c[o][i];
        if (!cf.op) continue;
        if (a.mslot[o][i] >= 0) {
          T mc[kBlkS];
#pragma unroll
          for (int b = 0; b < kBlkS; ++b) mc[b] = mat[o][i][b * kBlkS + c];
#pragma unroll
          for (int k = 0; k < kBlkSub; ++k) {
            const int rr = r + (kThreads / kBlkS) * k;
            T z = T(0);
#pragma unroll
            for (int b = 0; b < kBlkS; b += 2) {
              const typename Pair<T>::V x2 =
                  *reinterpret_cast<const typename Pair<T>::V*>(&tile[i][rr][b]);
              z = fma_rn(x2.x, mc[b], z);
              z = fma_rn(x2.y, mc[b + 1], z);
            }
            const T term = cs[o][i] * z;
            y[k] = first ? term : add_rn(y[k], term);
          }
        } else {
#pragma unroll
          for (int k = 0; k < kBlkSub; ++k) {
            const int rr = r + (kThreads / kBlkS) * k;
            y[k] = first ? mul_rn(cs[o][i], tile[i][rr][c])
                         : fma_rn(cs[o][i], tile[i][rr][c], y[k]);
          }
        }
        first = false;
      }
      if (first) {
#pragma unroll
        for (int k = 0; k < kBlkSub; ++k) y[k] = T(0);
      }
#pragma unroll
      for (int k = 0; k < kBlkSub; ++k) {
        const int rr = r + (kThreads / kBlkS) * k;
        const long long row = row0 + rr;
        const bool valid = c < s && row < a.n;
        if (valid) a.out[o][row * s + c] = y[k];
        tile[4 + o][rr][c] = valid ? y[k] : T(0);
      }
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      if (g >= a.ng) break;
      // thread (r, c) accumulates G[r][c] = sum_rows U[row][r] V[row][c]
      const int u = a.gram[g][0], v = a.gram[g][1];
      const int tu = u < a.nin ? u : 4 + (u - a.nin);
      const int tv = v < a.nin ? v : 4 + (v - a.nin);
      if (r < s && c < s) {
        double z = gacc[g];
#pragma unroll 8
        for (int q = 0; q < kBlkTileRows; ++q)
          z = fma_rn((double)tile[tu][q][r], (double)tile[tv][q][c], z);
        gacc[g] = z;
      }
    }
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      if (d >= a.nd) break;
      const int u = a.dot[d][0], v = a.dot[d][1];
      const int tu = u < a.nin ? u : 4 + (u - a.nin);
      const int tv = v < a.nin ? v : 4 + (v - a.nin);
#pragma unroll
      for (int k = 0; k < kBlkSub; ++k) {
        const int rr = r + (kThreads / kBlkS) * k;
        dacc[d] = fma_rn((double)tile[tu][rr][c], (double)tile[tv][rr][c], dacc[d]);
      }
    }
    __syncthreads();
  }
  if (a.ng > 0 || a.nd > 0 || rd.epi)
    blk_finish(gacc, a.ng, s, dacc, a.nd, a.gslot, rd, reinterpret_cast<double*>(raw));
}

// Deterministic reduction of per-thread Gram entries (thread t owns entry t
// of each Gram) and Frobenius dots across the grid, in two levels: the
// last block of each group of kRedGroup blocks sums its group's partials
// in block order, the last such group block sums the group sums in group
// order, writes them to the scalar slots and runs the epilogue.  (One
// level over all the grid's partials was a long chain of dependent
// batches of L2 loads on one SM; two levels need a handful.)  Partials: block b's
// kBlkPart values contiguous (Grams at q * 256, dots at 512), so writes
// and reads are coalesced.
__device__ __forceinline__ void blk_finish(const double* g, int ng, int s,
                                           const double* dd, int nd,
                                           const short* gslot, const Red& rd,
                                           double* stage) {
  __shared__ double wsum[2][kWarps];
  __shared__ int is_last;
  constexpr int kBlkPart = 514;
  const int t = threadIdx.x;
  const int nb = gridDim.x;
  const int grp = blockIdx.x / kRedGroup;
  const int b0 = grp * kRedGroup;
  const int gn = min(kRedGroup, nb - b0);
  const int ngrp = (nb + kRedGroup - 1) / kRedGroup;
  double* gpart = rd.part + (long long)kGridCap * kBlkPart;
  unsigned* gticket = reinterpret_cast<unsigned*>(rd.part + red2_ticket_offset(kBlkPart));
  double* mine = rd.part + (long long)blockIdx.x * kBlkPart;
#pragma unroll
  for (int q = 0; q < 2; ++q)
    if (q < ng) mine[q * 256 + t] = g[q];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    if (d >= nd) break;
    const double v = warp_sum(dd[d]);
    if ((t & 31) == 0) wsum[d][t >> 5] = v;
  }
  __syncthreads();
  if (t == 0) {
    for (int d = 0; d < nd; ++d) {
      double v = 0.0;
      for (int w = 0; w < kWarps; ++w) v += wsum[d][w];
      mine[512 + d] = v;
    }
    __threadfence();
    is_last = atomicAdd(gticket + grp, 1u) == (unsigned)gn - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // Level 1: this group's blocks.
  const double* gp = rd.part + (long long)b0 * kBlkPart;
  double* gout = gpart + (long long)grp * kBlkPart;
  for (int q = 0; q < ng; ++q) {
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < kRedGroup; ++b)
      if (b < gn) v += __ldcg(gp + (long long)b * kBlkPart + q * 256 + t);
    gout[q * 256 + t] = v;
  }
  if (t < nd) {
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < kRedGroup; ++b)
      if (b < gn) v += __ldcg(gp + (long long)b * kBlkPart + 512 + t);
    gout[512 + t] = v;
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
  const int r = t / kBlkS, c = t % kBlkS;
  for (int q = 0; q < ng; ++q) {
    double v = 0.0;
#pragma unroll 16
    for (int k = 0; k < ngrp; ++k) v += __ldcg(gpart + (long long)k * kBlkPart + q * 256 + t);
    if (r < s && c < s) rd.S[gslot[q] + r * s + c] = v;
  }
  if (t < nd) {
    double v = 0.0;
#pragma unroll 16
    for (int k = 0; k < ngrp; ++k) v += __ldcg(gpart + (long long)k * kBlkPart + 512 + t);
    rd.S[rd.out + t] = v;
  }
  __syncthreads();
  if (t == 0) *rd.ticket = 0u;
  if (rd.epi) {
    for (int q = t; q < kBlkEpiSlots; q += kThreads) stage[q] = __ldcg(rd.S + q);
    __syncthreads();
    Red local = rd;
    local.S = stage;
    // s-by-s algebra on all threads; the scalar epilogues on one
    if (!run_block_epilogue_cta(local, t) && t == 0) run_epilogue(local);
    __syncthreads();
    for (int q = t; q < kBlkEpiSlots; q += kThreads) rd.S[q] = stage[q];
  }
  if (t == 0) __threadfence();
}

}  // namespace bk
