// Small dense s-by-s algebra of the block methods, run inside the scalar
// epilogues (one thread; s <= 16, so a factorisation is a few thousand
// flops).  Replaces the reference's LAPACKE_dgetrf / dgetri / dgesv /
// dgetrs calls on s-by-s blocks (src/blcg.c:81-82, src/blbicgstab.c:69,94,
// src/blbicgstabl.c:105,124,147-148) and the R factor side of myqr
// (src/myqr.c).  All matrices row-major: M[i][j] = M[i * s + j].
#pragma once

namespace bk {

__device__ __forceinline__ void dm_copy(const double* A, double* B, int s) {
  for (int q = 0; q < s * s; ++q) B[q] = A[q];
}

__device__ __forceinline__ void dm_eye(double* A, int s) {
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) A[i * s + j] = i == j ? 1.0 : 0.0;
}

// C = A * B (C distinct from A and B).
__device__ __forceinline__ void dm_mul(const double* A, const double* B,
                                       double* C, int s) {
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) {
      double z = 0.0;
      for (int k = 0; k < s; ++k) z = fma(A[i * s + k], B[k * s + j], z);
      C[i * s + j] = z;
    }
}

// In-place LU with partial pivoting, P A = L U (piv[k] = row swapped into
// k at step k, stored as doubles).  Returns false on an exactly zero pivot.
__device__ __forceinline__ bool dm_lu(double* A, double* piv, int s) {
  bool ok = true;
  for (int k = 0; k < s; ++k) {
    int p = k;
    double best = fabs(A[k * s + k]);
    for (int i = k + 1; i < s; ++i)
      if (fabs(A[i * s + k]) > best) { best = fabs(A[i * s + k]); p = i; }
    piv[k] = (double)p;
    if (p != k)
      for (int j = 0; j < s; ++j) {
        const double t = A[k * s + j];
        A[k * s + j] = A[p * s + j];
        A[p * s + j] = t;
      }
    const double d = A[k * s + k];
    if (d == 0.0) { ok = false; continue; }
    for (int i = k + 1; i < s; ++i) {
      const double f = A[i * s + k] / d;
      A[i * s + k] = f;
      for (int j = k + 1; j < s; ++j) A[i * s + j] = fma(-f, A[k * s + j], A[i * s + j]);
    }
  }
  return ok;
}

// B <- A^-1 B for an LU from dm_lu; B is s-by-m row-major.
__device__ __forceinline__ void dm_lu_solve(const double* LU, const double* piv,
                                            double* B, int s, int m) {
  for (int k = 0; k < s; ++k) {
    const int p = (int)piv[k];
    if (p != k)
      for (int j = 0; j < m; ++j) {
        const double t = B[k * m + j];
        B[k * m + j] = B[p * m + j];
        B[p * m + j] = t;
      }
  }
  for (int j = 0; j < m; ++j) {
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
}

// Ainv = A^-1 (A is overwritten by its LU; piv scratch of s doubles).
__device__ __forceinline__ bool dm_inv(double* A, double* piv, double* Ainv,
                                       int s) {
  const bool ok = dm_lu(A, piv, s);
  dm_eye(Ainv, s);
  dm_lu_solve(A, piv, Ainv, s, s);
  return ok;
}

// Upper-triangular R with R^T R = G + shift I (Cholesky).  Returns false if
// a pivot is not positive.
__device__ __forceinline__ bool dm_chol(const double* G, double* R, int s,
                                        double shift) {
  for (int q = 0; q < s * s; ++q) R[q] = 0.0;
  for (int j = 0; j < s; ++j) {
    double d = G[j * s + j] + shift;
    for (int k = 0; k < j; ++k) d = fma(-R[k * s + j], R[k * s + j], d);
    if (!(d > 0.0)) return false;
    const double rjj = sqrt(d);
    R[j * s + j] = rjj;
    for (int i = j + 1; i < s; ++i) {
      double z = G[j * s + i];
      for (int k = 0; k < j; ++k) z = fma(-R[k * s + j], R[k * s + i], z);
      R[j * s + i] = z / rjj;
    }
  }
  return true;
}

// Ri = R^-1 for upper-triangular R.
__device__ __forceinline__ void dm_triinv(const double* R, double* Ri, int s) {
  for (int q = 0; q < s * s; ++q) Ri[q] = 0.0;
  for (int j = 0; j < s; ++j) {
    Ri[j * s + j] = 1.0 / R[j * s + j];
    for (int i = j - 1; i >= 0; --i) {
      double z = 0.0;
      for (int k = i + 1; k <= j; ++k) z = fma(R[i * s + k], Ri[k * s + j], z);
      Ri[i * s + j] = -z / R[i * s + i];
    }
  }
}

__device__ __forceinline__ double dm_fro(const double* A, int s) {
  double z = 0.0;
  for (int q = 0; q < s * s; ++q) z = fma(A[q], A[q], z);
  return sqrt(z);
}

}  // namespace bk
