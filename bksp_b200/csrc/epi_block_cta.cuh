// The block methods' s-by-s epilogues run by every thread of the last CTA
// of a block-kernel launch instead of by one thread.  Each s-by-s result
// entry (or, for the triangular solves, each column) is owned by one
// thread and formed with the same operations in the same order as the
// one-thread forms in epi_block.cuh, so the results are bit-identical to
// them; the steps that depend on one another (a factorisation column, a
// pivot) are separated by __syncthreads().
//
// Every helper is called by all threads of the block with the same
// arguments, reads operands that are visible to all threads on entry and
// ends with a __syncthreads(), so its outputs are visible on return.  The
// operands live in the staged slot copy in shared memory.  Requires
// blockDim.x >= s * s (256 threads, s <= 16).
#pragma once
#include "epilogues.cuh"

namespace bk {

__device__ __forceinline__ void cm_copy(const double* A, double* B, int s, int t) {
  if (t < s * s) B[t] = A[t];
  __syncthreads();
}

__device__ __forceinline__ void cm_eye(double* A, int s, int t) {
  if (t < s * s) A[t] = t / s == t % s ? 1.0 : 0.0;
  __syncthreads();
}

__device__ __forceinline__ void cm_zero(double* A, int s, int t) {
  if (t < s * s) A[t] = 0.0;
  __syncthreads();
}

// B = -A entry by entry (B may be A).
__device__ __forceinline__ void cm_neg(const double* A, double* B, int s, int t) {
  if (t < s * s) B[t] = -A[t];
  __syncthreads();
}

// B = f * A entry by entry (B may be A).
__device__ __forceinline__ void cm_scale(const double* A, double f, double* B,
                                         int s, int t) {
  if (t < s * s) B[t] = f * A[t];
  __syncthreads();
}

// C = A * B (C distinct from A and B): thread i * s + j forms C[i][j].
__device__ __forceinline__ void cm_mul(const double* A, const double* B,
                                       double* C, int s, int t) {
  if (t < s * s) {
    const int i = t / s, j = t % s;
    double z = 0.0;
    for (int k = 0; k < s; ++k) z = fma(A[i * s + k], B[k * s + j], z);
    C[t] = z;
  }
  __syncthreads();
}

// dm_lu by the block.  At step k every thread finds the pivot itself (the
// same scan, so the same row), then row k and the pivot row are swapped,
// the multipliers f_i = a_ik / a_kk formed once (thread i, into shared
// memory) and the trailing entries updated (thread (i, j), i > k, j >= k;
// j = k stores f_i).
__device__ __forceinline__ bool cm_lu(double* A, double* piv, int s, int t) {
  __shared__ double fcol[16];
  bool ok = true;
  for (int k = 0; k < s; ++k) {
    int p = k;
    double best = fabs(A[k * s + k]);
    for (int i = k + 1; i < s; ++i)
      if (fabs(A[i * s + k]) > best) { best = fabs(A[i * s + k]); p = i; }
    __syncthreads();                 // column k read by all before the swap
    if (t == 0) piv[k] = (double)p;
    if (p != k && t < s) {
      const double x = A[k * s + t];
      A[k * s + t] = A[p * s + t];
      A[p * s + t] = x;
    }
    __syncthreads();
    const double d = A[k * s + k];
    if (d == 0.0) { ok = false; continue; }
    if (t > k && t < s) fcol[t] = A[t * s + k] / d;
    __syncthreads();
    if (t < s * s) {
      const int i = t / s, j = t % s;
      if (i > k && j > k) A[i * s + j] = fma(-fcol[i], A[k * s + j], A[i * s + j]);
      else if (i > k && j == k) A[i * s + k] = fcol[i];
    }
    __syncthreads();
  }
  __syncthreads();
  return ok;
}

// dm_lu_solve by the block: B's columns are independent, thread j solves
// column j exactly as the one-thread form does.
__device__ __forceinline__ void cm_lu_solve(const double* LU, const double* piv,
                                            double* B, int s, int m, int t) {
  if (t < m) {
    const int j = t;
    for (int k = 0; k < s; ++k) {
      const int p = (int)piv[k];
      if (p != k) {
        const double x = B[k * m + j];
        B[k * m + j] = B[p * m + j];
        B[p * m + j] = x;
      }
    }
    for (int i = 1; i < s; ++i) {
      double z = B[i * m + j];
      for (int k = 0; k < i; ++k) z = fma(-LU[i * s + k], B[k * m + j], z);
      B[i * m + j] = z;
    }
    for (int i = s - 1; i >= 0; --i) {
      double z = B[i * m + j];
      for (int k = i + 1; k < s; ++k) z = fma(-LU[i * s + k], B[k * m + j], z);
      B[i * m + j] = z / LU[i * s + i];
    }
  }
  __syncthreads();
}

__device__ __forceinline__ bool cm_inv(double* A, double* piv, double* Ainv,
                                       int s, int t) {
  const bool ok = cm_lu(A, piv, s, t);
  cm_eye(Ainv, s, t);
  cm_lu_solve(A, piv, Ainv, s, s, t);
  return ok;
}

// dm_chol by the block: for column j, thread j forms the pivot and thread
// i > j the entry R[j][i] (both from rows 0 .. j-1 of R only).
__device__ __forceinline__ bool cm_chol(const double* G, double* R, int s,
                                        double shift, int t) {
  __shared__ double piv_d;
  if (t < s * s) R[t] = 0.0;
  __syncthreads();
  for (int j = 0; j < s; ++j) {
    double z = 0.0;
    if (t == j) {
      double d = G[j * s + j] + shift;
      for (int k = 0; k < j; ++k) d = fma(-R[k * s + j], R[k * s + j], d);
      piv_d = d;
    } else if (t > j && t < s) {
      z = G[j * s + t];
      for (int k = 0; k < j; ++k) z = fma(-R[k * s + j], R[k * s + t], z);
    }
    __syncthreads();
    const double d = piv_d;
    if (!(d > 0.0)) return false;    // every thread sees the same pivot
    const double rjj = sqrt(d);
    if (t == j) R[j * s + j] = rjj;
    else if (t > j && t < s) R[j * s + t] = z / rjj;
    __syncthreads();
  }
  return true;
}

// dm_triinv by the block: the columns of R^-1 are independent, thread j
// forms column j.
__device__ __forceinline__ void cm_triinv(const double* R, double* Ri, int s,
                                          int t) {
  if (t < s * s) Ri[t] = 0.0;
  __syncthreads();
  if (t < s) {
    const int j = t;
    Ri[j * s + j] = 1.0 / R[j * s + j];
    for (int i = j - 1; i >= 0; --i) {
      double z = 0.0;
      for (int k = i + 1; k <= j; ++k) z = fma(R[i * s + k], Ri[k * s + j], z);
      Ri[i * s + j] = -z / R[i * s + i];
    }
  }
  __syncthreads();
}

// qr_pass by the block (the shift is formed by every thread the same way).
static __device__ bool cqr_pass(double* S, int pass, int t) {
  const int s = (int)S[kBkS];
  double* G = S + kBkG1;
  double* Rp = S + kBkScr;
  double shift = 0.0;
  if (pass == 1) {
    double tr = 0.0;
    for (int i = 0; i < s; ++i) tr += G[i * s + i];
    const double m = S[kBkRows];
    const double u = S[kBkU] > 0.0 ? S[kBkU] : 1.1102230246251565e-16;
    shift = 11.0 * (m * s + s * (s + 1.0)) * u * tr;
  }
  if (!cm_chol(G, Rp, s, shift, t)) return false;
  cm_triinv(Rp, S + kBkRinv, s, t);
  if (pass == 1) {
    cm_copy(Rp, S + kBkR, s, t);
  } else {
    cm_mul(Rp, S + kBkR, S + kBkScr2, s, t);
    cm_copy(S + kBkScr2, S + kBkR, s, t);
  }
  return true;
}

static __device__ void cqr_post(const Red& rd, int action, int t) {
  double* S = rd.S;
  const int s = (int)S[kBkS];
  switch (action) {
    case QR_POST_BCG:        // src/blcg.c:95-105
      cm_copy(S + kBkR, S + kBkBeta, s, t);
      cm_mul(S + kBkBeta, S + kBkC, S + kBkScr, s, t);
      cm_copy(S + kBkScr, S + kBkC, s, t);
      if (t == 0) conv_check(rd, dm_fro(S + kBkC, s) / S[kFnb]);
      break;
    case QR_POST_BCG_INIT:   // src/blcg.c:58, :61-63
      cm_copy(S + kBkR, S + kBkC, s, t);
      cm_eye(S + kBkBeta, s, t);
      break;
    case QR_POST_BBL_INIT:   // src/blbicgstabl.c:88
      cm_copy(S + kBkR, S + kBkXi, s, t);
      break;
    case QR_POST_BBL_T:      // src/blbicgstabl.c:135-148
      cm_copy(S + kBkR, S + kBkT, s, t);
      cm_copy(S + kBkXi, S + kBkXiOld, s, t);
      cm_mul(S + kBkT, S + kBkXiOld, S + kBkXi, s, t);
      cm_copy(S + kBkT, S + kBkScr, s, t);
      cm_inv(S + kBkScr, S + kBkPiv, S + kBkTinv, s, t);
      cm_mul(S + kBkAlpha, S + kBkTinv, S + kBkATinv, s, t);
      break;
    default:
      break;
  }
}

// The block-algebra epilogue codes, by all threads of the last CTA.
// Returns false (before touching anything) for every other code, which
// the caller then runs on one thread.
static __device__ __noinline__ bool run_block_epilogue_cta(const Red& rd, int t) {
  double* S = rd.S;
  const double* D = S + rd.out;
  const int l = (int)S[kL];
  const int s = (int)S[kBkS];
  switch (rd.epi) {
    case E_QR1:
    case E_QR2:
    case E_QR3: {
      const int pass = rd.epi == E_QR1 ? 1 : rd.epi == E_QR2 ? 2 : 3;
      if (!cqr_pass(S, pass, t)) {
        if (t == 0) fail_divergence(rd);
      } else if (pass == 3) {
        cqr_post(rd, rd.a0, t);
      }
      return true;
    }
    case E_BCG_INIT: {       // src/blcg.c:60, then the first pass of myqr (:58)
      if (t == 0) S[kFnb] = sqrt(D[0]);
      __syncthreads();
      if (!cqr_pass(S, 1, t) && t == 0) fail_divergence(rd);
      return true;
    }
    case E_BCG_ALPHA:        // src/blcg.c:78-86
      cm_copy(S + kBkG1, S + kBkLU, s, t);
      cm_inv(S + kBkLU, S + kBkPiv, S + kBkAlpha, s, t);
      cm_mul(S + kBkAlpha, S + kBkC, S + kBkTmp, s, t);
      return true;
    case E_BBS_ALPHA:        // src/blbicgstab.c:185-189
      cm_copy(S + kBkG1, S + kBkLU, s, t);
      cm_lu(S + kBkLU, S + kBkPiv, s, t);
      cm_copy(S + kBkG2, S + kBkAlpha, s, t);
      cm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkAlpha, s, s, t);
      return true;
    case E_BBS_BETA:         // src/blbicgstab.c:212-214, :226-229
      cm_neg(S + kBkG1, S + kBkBeta, s, t);
      cm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkBeta, s, s, t);
      if (t == 0) conv_check(rd, sqrt(D[0]) / S[kFnb]);
      return true;
    case E_BBL_INIT: {       // src/blbicgstabl.c:31-38, :67-76, :93, :88
      if (t == 0) {
        S[kFnb] = sqrt(D[0]);
        for (int i = 0; i <= l; ++i) S[kBlOmega + i] = 0.0;
        S[kBlOmega + l] = 1.0;
      }
      cm_zero(S + kBkAlpha, s, t);
      cm_eye(S + kBkGam0, s, t);
      // :98  gamma0 = -omega[l] gamma0 of the first iteration
      cm_scale(S + kBkGam0, -S[kBlOmega + l], S + kBkGam0, s, t);
      if (!cqr_pass(S, 1, t) && t == 0) fail_divergence(rd);
      return true;
    }
    case E_BBL_BETA:         // src/blbicgstabl.c:102-108
      cm_copy(S + kBkG1, S + kBkGam1, s, t);
      cm_copy(S + kBkGam0, S + kBkLU, s, t);
      cm_lu(S + kBkLU, S + kBkPiv, s, t);
      cm_copy(S + kBkGam1, S + kBkTmp, s, t);
      cm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkTmp, s, s, t);
      cm_mul(S + kBkAlpha, S + kBkTmp, S + kBkBeta, s, t);
      cm_neg(S + kBkBeta, S + kBkBeta, s, t);
      cm_copy(S + kBkGam1, S + kBkGam0, s, t);
      return true;
    case E_BBL_ALPHA:        // src/blbicgstabl.c:121-124
      cm_copy(S + kBkG1, S + kBkLU, s, t);
      cm_lu(S + kBkLU, S + kBkPiv, s, t);
      cm_copy(S + kBkGam1, S + kBkAlpha, s, t);
      cm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkAlpha, s, s, t);
      return true;
    case E_BBL_CHECK: {      // src/blbicgstabl.c:209-212, then :98
      if (t == 0) conv_check(rd, dm_fro(S + kBkXi, s) / S[kFnb]);
      const double f = -S[kBlOmega + l];
      cm_scale(S + kBkGam0, f, S + kBkGam0, s, t);
      return true;
    }
    default:
      return false;
  }
}

}  // namespace bk
