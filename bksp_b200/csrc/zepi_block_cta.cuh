// The complex block method's s-by-s epilogues (Cholesky-QR passes and
// Block BiCGSTAB(l)'s small systems, src/blbicgstabl.c:326-457 and
// src/myqr.c:41-76) run by every thread of the last CTA of a complex
// block-kernel launch instead of by one thread.  Each result entry (or,
// for the triangular solves, each column) is owned by one thread and
// formed with the same operations in the same order as the one-thread
// forms in zepi_block.cuh; the dependent steps are separated by
// __syncthreads(), which also makes the global slot writes of one thread
// visible to the others of the block.
//
// Every helper is called by all threads of the block with the same
// arguments and ends with a __syncthreads().  Requires blockDim.x >= s * s.
#pragma once
#include "epi_common.cuh"
#include "zepi_block.cuh"

namespace bk {

__device__ __forceinline__ void zcm_copy(const double* A, double* B, int s, int t) {
  for (int q = t; q < 2 * s * s; q += blockDim.x) B[q] = A[q];
  __syncthreads();
}

// C = A B (C distinct from A and B): thread i * s + j forms C[i][j].
__device__ __forceinline__ void zcm_mul(const double* A, const double* B,
                                        double* C, int s, int t) {
  if (t < s * s) {
    const int i = t / s, j = t % s;
    zc z = zmk(0.0);
    for (int k = 0; k < s; ++k) z = zadd(z, zmul(zm_get(A, s, i, k), zm_get(B, s, k, j)));
    zm_set(C, s, i, j, z);
  }
  __syncthreads();
}

// zm_lu by the block: every thread scans for the pivot itself, then the
// swap, the trailing update (thread (i, j), i, j > k) and the multipliers.
__device__ __forceinline__ bool zcm_lu(double* A, double* piv, int s, int t) {
  bool ok = true;
  for (int k = 0; k < s; ++k) {
    int p = k;
    double best = zabs2(zm_get(A, s, k, k));
    for (int i = k + 1; i < s; ++i) {
      const double v = zabs2(zm_get(A, s, i, k));
      if (v > best) { best = v; p = i; }
    }
    __syncthreads();                 // column k read by all before the swap
    if (t == 0) piv[k] = (double)p;
    if (p != k && t < s) {
      const zc x = zm_get(A, s, k, t);
      zm_set(A, s, k, t, zm_get(A, s, p, t));
      zm_set(A, s, p, t, x);
    }
    __syncthreads();
    const zc d = zm_get(A, s, k, k);
    if (d.re == 0.0 && d.im == 0.0) { ok = false; continue; }
    if (t < s * s) {
      const int i = t / s, j = t % s;
      if (i > k && j > k) {
        const zc f = zdiv(zm_get(A, s, i, k), d);
        zm_set(A, s, i, j, zsub(zm_get(A, s, i, j), zmul(f, zm_get(A, s, k, j))));
      }
    }
    __syncthreads();
    if (t > k && t < s) zm_set(A, s, t, k, zdiv(zm_get(A, s, t, k), d));
    __syncthreads();
  }
  __syncthreads();
  return ok;
}

// zm_lu_solve by the block: thread j solves column j.
__device__ __forceinline__ void zcm_lu_solve(const double* LU, const double* piv,
                                             double* B, int s, int t) {
  if (t < s) {
    const int j = t;
    for (int k = 0; k < s; ++k) {
      const int p = (int)piv[k];
      if (p != k) {
        const zc x = zm_get(B, s, k, j);
        zm_set(B, s, k, j, zm_get(B, s, p, j));
        zm_set(B, s, p, j, x);
      }
    }
    for (int i = 1; i < s; ++i) {
      zc z = zm_get(B, s, i, j);
      for (int k = 0; k < i; ++k) z = zsub(z, zmul(zm_get(LU, s, i, k), zm_get(B, s, k, j)));
      zm_set(B, s, i, j, z);
    }
    for (int i = s - 1; i >= 0; --i) {
      zc z = zm_get(B, s, i, j);
      for (int k = i + 1; k < s; ++k) z = zsub(z, zmul(zm_get(LU, s, i, k), zm_get(B, s, k, j)));
      zm_set(B, s, i, j, zdiv(z, zm_get(LU, s, i, i)));
    }
  }
  __syncthreads();
}

// zm_chol by the block: for column j, thread j forms the (real) pivot and
// thread i > j the entry R[j][i].
__device__ __forceinline__ bool zcm_chol(const double* G, double* R, int s,
                                         double shift, int t) {
  __shared__ double piv_d;
  for (int q = t; q < 2 * s * s; q += blockDim.x) R[q] = 0.0;
  __syncthreads();
  for (int j = 0; j < s; ++j) {
    zc z = zmk(0.0);
    if (t == j) {
      double d = zm_get(G, s, j, j).re + shift;
      for (int k = 0; k < j; ++k) d -= zabs2(zm_get(R, s, k, j));
      piv_d = d;
    } else if (t > j && t < s) {
      z = zm_get(G, s, j, t);
      for (int k = 0; k < j; ++k)
        z = zsub(z, zmul(zconj(zm_get(R, s, k, j)), zm_get(R, s, k, t)));
    }
    __syncthreads();
    const double d = piv_d;
    if (!(d > 0.0)) return false;    // every thread sees the same pivot
    const double rjj = sqrt(d);
    if (t == j) zm_set(R, s, j, j, zmk(rjj));
    else if (t > j && t < s) zm_set(R, s, j, t, zscal(1.0 / rjj, z));
    __syncthreads();
  }
  return true;
}

// zm_triinv by the block: thread j forms column j of R^-1.
__device__ __forceinline__ void zcm_triinv(const double* R, double* Ri, int s,
                                           int t) {
  for (int q = t; q < 2 * s * s; q += blockDim.x) Ri[q] = 0.0;
  __syncthreads();
  if (t < s) {
    const int j = t;
    zm_set(Ri, s, j, j, zinv(zm_get(R, s, j, j)));
    for (int i = j - 1; i >= 0; --i) {
      zc z = zmk(0.0);
      for (int k = i + 1; k <= j; ++k) z = zadd(z, zmul(zm_get(R, s, i, k), zm_get(Ri, s, k, j)));
      zm_set(Ri, s, i, j, zneg(zdiv(z, zm_get(R, s, i, i))));
    }
  }
  __syncthreads();
}

// One complex Cholesky-QR pass (the one-thread zqr_pass) by the block.
static __device__ bool zcqr_pass(double* S, int pass, int t) {
  const int s = (int)S[kZBkS];
  const double* G = S + kZBkG1;
  double* Rp = S + kZBkScr;
  double shift = 0.0;
  if (pass == 1) {
    double tr = 0.0;
    for (int i = 0; i < s; ++i) tr += zm_get(G, s, i, i).re;
    shift = 11.0 * (S[kZBkRows] * s + s * (s + 1.0)) * 1.1102230246251565e-16 * tr;
  }
  if (!zcm_chol(G, Rp, s, shift, t)) return false;
  zcm_triinv(Rp, S + kZBkRinv, s, t);
  if (pass == 1) {
    zcm_copy(Rp, S + kZBkR, s, t);
  } else {
    zcm_mul(Rp, S + kZBkR, S + kZBkG2, s, t);
    zcm_copy(S + kZBkG2, S + kZBkR, s, t);
  }
  return true;
}

static __device__ void zcqr_post(double* S, int action, int t) {
  const int s = (int)S[kZBkS];
  switch (action) {
    case ZQR_POST_INIT:      // src/blbicgstabl.c:326
      zcm_copy(S + kZBkR, S + kZBkXi, s, t);
      break;
    case ZQR_POST_T:         // :376-390
      zcm_copy(S + kZBkR, S + kZBkT, s, t);
      zcm_copy(S + kZBkXi, S + kZBkXiOld, s, t);
      zcm_mul(S + kZBkT, S + kZBkXiOld, S + kZBkXi, s, t);
      zcm_triinv(S + kZBkT, S + kZBkTinv, s, t);
      zcm_mul(S + kZBkAlpha, S + kZBkTinv, S + kZBkATinv, s, t);
      break;
    default:
      break;
  }
}

// The complex block-algebra epilogue codes, by all threads of the last CTA.
// Returns false (before touching anything) for every other code, which the
// caller then runs on one thread.
static __device__ __noinline__ bool run_zblock_epilogue_cta(const Red& rd, int t) {
  double* S = rd.S;
  const int D = rd.out;
  const int l = (int)S[kL];
  const int s = (int)S[kZBkS];
  switch (rd.epi) {
    case EZ_QR1:
    case EZ_QR2:
    case EZ_QR3: {
      const int pass = rd.epi == EZ_QR1 ? 1 : rd.epi == EZ_QR2 ? 2 : 3;
      if (!zcqr_pass(S, pass, t)) {
        if (t == 0) fail_divergence(rd);
      } else if (pass == 3) {
        zcqr_post(S, rd.a0, t);
      }
      return true;
    }
    case EZ_BB_INIT:         // src/blbicgstabl.c:333, zqreco pass 1 (:326)
      if (t == 0) S[kFnb] = sqrt(S[D]);
      __syncthreads();
      if (!zcqr_pass(S, 1, t) && t == 0) fail_divergence(rd);
      return true;
    case EZ_BB_BETA:         // :343-349
      zcm_copy(S + kZBkG1, S + kZBkGam1, s, t);
      zcm_copy(S + kZBkGam0, S + kZBkLU, s, t);
      if (!zcm_lu(S + kZBkLU, S + kZBkPiv, s, t)) {
        if (t == 0) fail_divergence(rd);
        return true;
      }
      zcm_copy(S + kZBkGam1, S + kZBkScr, s, t);
      zcm_lu_solve(S + kZBkLU, S + kZBkPiv, S + kZBkScr, s, t);
      zcm_mul(S + kZBkAlpha, S + kZBkScr, S + kZBkBeta, s, t);
      zcm_copy(S + kZBkGam1, S + kZBkGam0, s, t);
      return true;
    case EZ_BB_ALPHA:        // :362-365
      zcm_copy(S + kZBkG1, S + kZBkLU, s, t);
      if (!zcm_lu(S + kZBkLU, S + kZBkPiv, s, t)) {
        if (t == 0) fail_divergence(rd);
        return true;
      }
      zcm_copy(S + kZBkGam1, S + kZBkAlpha, s, t);
      zcm_lu_solve(S + kZBkLU, S + kZBkPiv, S + kZBkAlpha, s, t);
      return true;
    case EZ_BB_CHECK: {      // :454-457, then :338-339 of the next iteration
      if (t == 0) conv_check(rd, zm_fro(S + kZBkXi, s) / S[kFnb]);
      const zc m = zneg(zld(S, kZOmega + 2 * (l - 1)));
      double* g0 = S + kZBkGam0;
      if (t < s * s) {
        const zc v = zmul(m, zc{g0[2 * t], g0[2 * t + 1]});
        g0[2 * t] = v.re;
        g0[2 * t + 1] = v.im;
      }
      __syncthreads();
      return true;
    }
    default:
      return false;
  }
}

}  // namespace bk
