// Host-visible interface of the complex (double _Complex) kernels: plain
// structs shared by kernels_z.cu and the complex drivers (zsolvers.cpp).
//
// Complex data in HBM: vectors are arrays of double2 (re, im), padded to a
// multiple of 64 elements like the real vectors; n-by-s blocks are stored
// row-major (row i's s values contiguous, s <= 16).  A complex scalar of a
// recurrence occupies two consecutive FP64 slots S[k] (re), S[k + 1] (im).
#pragma once

#include <cuda_runtime.h>

#include "kernel_api.h"

namespace bk {

// Coefficient of one complex linear-combination term:
//   op 1: k                      (k = kr + i ki)
//   op 2: k * z(S[s])            (conj: k * conj(z(S[s])))
struct ZCfH {
  short op, s, conj, pad;
  double kr, ki;
};
static inline ZCfH zcf_const(double kr, double ki = 0.0) {
  ZCfH c{}; c.op = 1; c.kr = kr; c.ki = ki; return c;
}
static inline ZCfH zcf_slot(short s, double k = 1.0) {
  ZCfH c{}; c.op = 2; c.s = s; c.kr = k; return c;
}
static inline ZCfH zcf_conj(short s, double k = 1.0) {
  ZCfH c{}; c.op = 2; c.s = s; c.conj = 1; c.kr = k; return c;
}

constexpr int kZLcIn = 20;
constexpr int kZLcOut = 6;
constexpr int kZDots = 4;

// out[o] = sum_i c[o][i] in[i] over n complex elements, repeated `reps`
// times with the operands flagged in the rep masks advanced by `stride`
// elements per repetition; then up to kZDots complex dots among
// [in..., out...] (operand codes: input index, or 100 + output index):
// dconj = 1: sum conj(u) v (zdotc), 0: sum u v.  Dot d is written to
// S[out + 2d] (re) and S[out + 2d + 1] (im).
struct ZLcH {
  const double2* in[kZLcIn];
  double2* out[kZLcOut];
  ZCfH c[kZLcOut][kZLcIn];
  long long n, stride;
  int nin, nout, reps, nd;
  unsigned in_rep_mask, out_rep_mask;
  unsigned char dot[kZDots][2];
  unsigned char dconj[kZDots];
};

// Complex CSR product y = A x (mode 0) or y = b - A x (mode 1) on the row
// blocks of the tile kernel, optional copy y2, up to three complex dots
// among {0: y, 1: b, 2: w0} written like ZLcH's.  The operator's values
// (CsrH::val) are double2.
struct ZSpmvH {
  const double2* x;
  double2* y;
  double2* y2;
  const double2* b;
  const double2* w0;
  int mode, nd;
  unsigned char dot[3][2];
  unsigned char dconj[3];
};

// Complex SpMM on row-major n-by-s blocks: Y = beta C + alpha A X with
// alpha = +-1 and beta in {0, 1} (the reference's zcsrgemm1 order:
// y = beta c, then y += (alpha a_k) x_k entry by entry).
struct ZSpmmH {
  const double2* X;
  double2* Y;
  const double2* C;
  int s, alpha, beta;
};

// Complex block linear combination on row-major n-by-s blocks:
//   out[o] = sum_i term(o, i),  term = c * in[i]  or  in[i] * M
// (M an s-by-s complex matrix from the slots, row-major pairs, at most two
// matrix terms per launch), then up to two Gram products
//   G_g = U_g^T V_g  (gconj 0)  or  U_g^H V_g  (gconj 1)
// written to S[gslot_g + 2 (a s + b)] and up to two Frobenius dots
// (zdotc) to S[out + 2d].
struct ZBlkH {
  const double2* in[4];
  double2* out[2];
  ZCfH c[2][4];
  short mslot[2][4];   // >= 0: matrix term
  int nin, nout, s;
  long long n;         // rows
  int ng;
  unsigned char gram[2][2];
  unsigned char gconj[2];
  short gslot[2];
  int nd;
  unsigned char dot[2][2];
};
constexpr int kZBlkPart = 1028;   // per-block partials: 2 Grams x 512 + 2 dots x 2

// All-shift updates of the complex shifted BiCGSTAB(l) (kernels_z.cu).
// Per shift k (ns shifts, vectors ps[k][i] = P + (k (l+1) + i) np):
//   mode 0 (BiCG step j):   ps_i = cb_k ps_i + cr_k r_i (i <= j),
//                           ps_{j+1} = cq_k r_j,  x_k += ca_k ps_0
//   mode 1 (after r_{j+1}): ps_{j+1} = cs_k (ps_{j+1} + cn_k r_j) - sig_k ps_j
//   mode 2 (MR update):     x_k += sum_{i<l} cx_{k,i} r_i,
//                           ps_0 = cp_k (ps_0 - sum_{i=1..l} om_{i-1} ps_i)
// Coefficients are complex slot pairs in per-shift arrays (index k).
struct ZShiftH {
  double2* P;          // shift direction vectors, ns x (l + 1) x np
  double2* X;          // shifted solutions, ns x np
  const double2* R;    // seed residuals r_0..r_l, (l + 1) x np
  long long np;
  int ns, l, j, mode;
};

// Launch entry points (kernels_z.cu).  Each throws CudaError on failure.
void launch_zlc(const ZLcH& d, const RedH& rd, cudaStream_t st);
void launch_zspmv(const CsrH& A, const ZSpmvH& io, const RedH& rd,
                  cudaStream_t st);
void launch_zspmm(const CsrH& A, const ZSpmmH& a, const RedH& rd,
                  cudaStream_t st);
void launch_zblock(const ZBlkH& a, const RedH& rd, cudaStream_t st);
void launch_zshift(const ZShiftH& a, const RedH& rd, cudaStream_t st);
// Fill a complex sliced-ELL copy from the device CSR (sptr from the host).
void launch_csr2sell_z(const int* rowptr, const int* col, const double2* val,
                       int n, int nslice, const int* sptr, int* scol,
                       double2* sval, cudaStream_t st);

}  // namespace bk
