// Complex scalar arithmetic and small dense complex s-by-s algebra for the
// scalar epilogues of the complex solvers (one thread; s <= 16).  Replaces
// the reference's LAPACKE_zgesv / zgetrf / zgetri calls on s-by-s blocks
// (src/blbicgstabl.c:346, 365, 389-390) and the R side of zqreco
// (src/myqr.c:41-76).  Matrices are row-major (re, im) pairs:
// M[i][j] = (M[2 (i s + j)], M[2 (i s + j) + 1]).
#pragma once
#include <cuda_runtime.h>

namespace bk {

struct zc {
  double re, im;
};

__device__ __forceinline__ zc zmk(double re, double im = 0.0) { return zc{re, im}; }
__device__ __forceinline__ zc zadd(zc a, zc b) { return zc{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ zc zsub(zc a, zc b) { return zc{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ zc zneg(zc a) { return zc{-a.re, -a.im}; }
__device__ __forceinline__ zc zconj(zc a) { return zc{a.re, -a.im}; }
__device__ __forceinline__ zc zscal(double k, zc a) { return zc{k * a.re, k * a.im}; }
__device__ __forceinline__ zc zmul(zc a, zc b) {
  return zc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ double zabs2(zc a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ double zabs(zc a) { return hypot(a.re, a.im); }
// a / b by Smith's algorithm (R. L. Smith, "Algorithm 116: Complex
// division", CACM 5(8), 1962): scale by the larger component of b so that
// no intermediate overflows for representable quotients.
__device__ __forceinline__ zc zdiv(zc a, zc b) {
  if (fabs(b.re) >= fabs(b.im)) {
    if (b.re == 0.0 && b.im == 0.0) return zc{a.re / 0.0, a.im / 0.0};
    const double r = b.im / b.re, d = b.re + b.im * r;
    return zc{(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  const double r = b.re / b.im, d = b.re * r + b.im;
  return zc{(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
__device__ __forceinline__ zc zinv(zc b) { return zdiv(zc{1.0, 0.0}, b); }
__device__ __forceinline__ bool zfinite(zc a) { return isfinite(a.re) && isfinite(a.im); }

// Slot pairs.
__device__ __forceinline__ zc zld(const double* S, int k) { return zc{S[k], S[k + 1]}; }
__device__ __forceinline__ void zst(double* S, int k, zc z) { S[k] = z.re; S[k + 1] = z.im; }

// ---------------------------------------------------------- s-by-s matrices
__device__ __forceinline__ zc zm_get(const double* A, int s, int i, int j) {
  return zc{A[2 * (i * s + j)], A[2 * (i * s + j) + 1]};
}
__device__ __forceinline__ void zm_set(double* A, int s, int i, int j, zc z) {
  A[2 * (i * s + j)] = z.re;
  A[2 * (i * s + j) + 1] = z.im;
}

__device__ __forceinline__ void zm_copy(const double* A, double* B, int s) {
  for (int q = 0; q < 2 * s * s; ++q) B[q] = A[q];
}

__device__ __forceinline__ void zm_eye(double* A, int s) {
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) zm_set(A, s, i, j, zmk(i == j ? 1.0 : 0.0));
}

// C = A B (C distinct from A and B).
__device__ __forceinline__ void zm_mul(const double* A, const double* B,
                                       double* C, int s) {
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) {
      zc z = zmk(0.0);
      for (int k = 0; k < s; ++k) z = zadd(z, zmul(zm_get(A, s, i, k), zm_get(B, s, k, j)));
      zm_set(C, s, i, j, z);
    }
}

// In-place LU with partial pivoting on |a_ik| (P A = L U; piv[k] = row
// swapped into k, as doubles).  False on an exactly zero pivot.
__device__ __forceinline__ bool zm_lu(double* A, double* piv, int s) {
  bool ok = true;
  for (int k = 0; k < s; ++k) {
    int p = k;
    double best = zabs2(zm_get(A, s, k, k));
    for (int i = k + 1; i < s; ++i) {
      const double v = zabs2(zm_get(A, s, i, k));
      if (v > best) { best = v; p = i; }
    }
    piv[k] = (double)p;
    if (p != k)
      for (int j = 0; j < s; ++j) {
        const zc t = zm_get(A, s, k, j);
        zm_set(A, s, k, j, zm_get(A, s, p, j));
        zm_set(A, s, p, j, t);
      }
    const zc d = zm_get(A, s, k, k);
    if (d.re == 0.0 && d.im == 0.0) { ok = false; continue; }
    for (int i = k + 1; i < s; ++i) {
      const zc f = zdiv(zm_get(A, s, i, k), d);
      zm_set(A, s, i, k, f);
      for (int j = k + 1; j < s; ++j)
        zm_set(A, s, i, j, zsub(zm_get(A, s, i, j), zmul(f, zm_get(A, s, k, j))));
    }
  }
  return ok;
}

// B <- A^-1 B for an LU from zm_lu; B is s-by-s.
__device__ __forceinline__ void zm_lu_solve(const double* LU, const double* piv,
                                            double* B, int s) {
  for (int k = 0; k < s; ++k) {
    const int p = (int)piv[k];
    if (p != k)
      for (int j = 0; j < s; ++j) {
        const zc t = zm_get(B, s, k, j);
        zm_set(B, s, k, j, zm_get(B, s, p, j));
        zm_set(B, s, p, j, t);
      }
  }
  for (int j = 0; j < s; ++j) {
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
}

// Upper-triangular R with real positive diagonal and R^H R = G + shift I
// (Cholesky of a Hermitian G).  False if a pivot is not positive.
__device__ __forceinline__ bool zm_chol(const double* G, double* R, int s,
                                        double shift) {
  for (int q = 0; q < 2 * s * s; ++q) R[q] = 0.0;
  for (int j = 0; j < s; ++j) {
    double d = zm_get(G, s, j, j).re + shift;
    for (int k = 0; k < j; ++k) d -= zabs2(zm_get(R, s, k, j));
    if (!(d > 0.0)) return false;
    const double rjj = sqrt(d);
    zm_set(R, s, j, j, zmk(rjj));
    for (int i = j + 1; i < s; ++i) {
      zc z = zm_get(G, s, j, i);
      for (int k = 0; k < j; ++k)
        z = zsub(z, zmul(zconj(zm_get(R, s, k, j)), zm_get(R, s, k, i)));
      zm_set(R, s, j, i, zscal(1.0 / rjj, z));
    }
  }
  return true;
}

// Ri = R^-1 for upper-triangular R.
__device__ __forceinline__ void zm_triinv(const double* R, double* Ri, int s) {
  for (int q = 0; q < 2 * s * s; ++q) Ri[q] = 0.0;
  for (int j = 0; j < s; ++j) {
    zm_set(Ri, s, j, j, zinv(zm_get(R, s, j, j)));
    for (int i = j - 1; i >= 0; --i) {
      zc z = zmk(0.0);
      for (int k = i + 1; k <= j; ++k) z = zadd(z, zmul(zm_get(R, s, i, k), zm_get(Ri, s, k, j)));
      zm_set(Ri, s, i, j, zneg(zdiv(z, zm_get(R, s, i, i))));
    }
  }
}

__device__ __forceinline__ double zm_fro(const double* A, int s) {
  double z = 0.0;
  for (int q = 0; q < 2 * s * s; ++q) z = fma(A[q], A[q], z);
  return sqrt(z);
}

}  // namespace bk
