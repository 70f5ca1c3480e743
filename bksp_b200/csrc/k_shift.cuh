// K9: fused all-shift update of the shifted methods (reference
// src/shbicg.c:78-96 and src/shbicgstabl.c:111-153, 202-237, which update
// each shift's p and x vectors with separate BLAS-1 calls per shift).
// One thread owns element i: it loads the seed vectors' entries once and
// updates p_k and x_k of every shift k, so each shift vector moves through
// HBM exactly once per step.  Per-shift coefficients come from the scalar
// slots (computed by the epilogues) and are staged in shared memory.
#pragma once
#include "dev_common.cuh"
#include "solver_defs.h"

namespace bk {

// Modes:
//   0  shifted BiCG:            x += a p;  p_k = -b_k p_k + r / pi_k;
//                               x_k += a_k p_k
//   1  shifted BiCGSTAB(l), BiCG step j (before the r update):
//                               x += a p_0;  p_k[i] = -b_k p_k[i] + r[i] / (pi_k th_k),
//                               i <= j;  p_k[j+1] = r[j] / pi_k;  x_k += a_k p_k[0]
//   2  same, after r_{j+1} = A r_j:
//                               p_k[j+1] = (p_k[j+1] - r[j] / pin_k) / (th_k a_k) - s_k p_k[j]
//   3  shifted BiCGSTAB(l), update (before the seed r0 update):
//                               x_k += sum_i cx_k[i] r[i];
//                               p_k[0] = (p_k[0] - w[l-1] p_k[l] - sum_{i<l} w[i-1] p_k[i]) / psi_k
// PT: storage type of the shift vectors p_k (double, or float in the
// mixed-precision shifted solve, where they are the bulk of the traffic);
// every update is computed in FP64 and rounded to PT when stored.  The seed
// vectors and x_k are always FP64.
template <typename PT>
struct ShiftArgs {
  const double* r;   // seed r[0..l] (stride np)
  const double* p;   // seed p[0..l]
  double* x;         // seed x
  double* xs;        // x_k at xs + k * np
  PT* ps;            // p_k[i] at ps + (k * (l + 1) + i) * np
  long long np;
  int ns, l, j, mode;
};

template <int MODE, typename PT>
__global__ void __launch_bounds__(kThreads, 4)
k_shift(ShiftArgs<PT> a, Red rd) {
  if (skip(rd)) return;
  __shared__ double c0[kMaxShifts], c1[kMaxShifts], c2[kMaxShifts],
      c3[kMaxShifts], c4[kMaxShifts];
  __shared__ double cx[kMaxShifts][kBlMaxL];
  __shared__ double om[kBlMaxL];
  const double* S = rd.S;
  const int ns = a.ns, l = a.l, j = a.j;
  for (int k = threadIdx.x; k < ns; k += kThreads) {
    if (MODE == 0 || MODE == 1) {
      c0[k] = -S[kShBeta + k];
      c1[k] = MODE == 0 ? 1.0 / S[kShPi + k]
                        : 1.0 / (S[kShPi + k] * S[kShTheta + k]);
      c2[k] = S[kShAlpha + k];
      c3[k] = 1.0 / S[kShPi + k];
    } else if (MODE == 2) {
      c0[k] = -1.0 / S[kShPiNew + k];
      c1[k] = 1.0 / (S[kShTheta + k] * S[kShAlpha + k]);
      c2[k] = -S[kShSigma + k];
    } else {
      for (int i = 0; i < l; ++i) cx[k][i] = S[kShCx + k * 8 + i];
      c4[k] = S[kShPsiInv + k];
    }
  }
  if (MODE == 3 && threadIdx.x < l) om[threadIdx.x] = S[kBlOmega + threadIdx.x];
  const double alpha = MODE == 0 ? S[kShAlphaS] : S[kBlAlpha];
  __syncthreads();
  const long long np = a.np;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < np;
       i += (long long)gridDim.x * kThreads) {
    double r[kBlMaxL + 1];
    if (MODE == 0) {
      r[0] = a.r[i];
      a.x[i] = fma_rn(alpha, a.p[i], a.x[i]);
      // Four shifts per pass: their loads are in flight together (one
      // shift at a time left the kernel bound by load latency).
#pragma unroll 4
      for (int k = 0; k < ns; ++k) {
        PT* pk = a.ps + (long long)k * np;
        const double pv = (double)(PT)fma_rn(c1[k], r[0], mul_rn(c0[k], (double)pk[i]));
        pk[i] = (PT)pv;
        double* xk = a.xs + (long long)k * np;
        xk[i] = fma_rn(c2[k], pv, xk[i]);
      }
    } else if (MODE == 1) {
      for (int q = 0; q <= j; ++q) r[q] = a.r[q * np + i];
      a.x[i] = fma_rn(alpha, a.p[i], a.x[i]);
      // Four shifts per pass: their loads are in flight together (one
      // shift at a time left the kernel bound by load latency).
#pragma unroll 4
      for (int k = 0; k < ns; ++k) {
        PT* pk = a.ps + (long long)k * (l + 1) * np;
        double p0 = 0.0;
        for (int q = 0; q <= j; ++q) {
          const double pv =
              (double)(PT)fma_rn(c1[k], r[q], mul_rn(c0[k], (double)pk[q * np + i]));
          pk[q * np + i] = (PT)pv;
          if (q == 0) p0 = pv;
        }
        pk[(j + 1) * np + i] = (PT)mul_rn(r[j], c3[k]);
        double* xk = a.xs + (long long)k * np;
        xk[i] = fma_rn(c2[k], p0, xk[i]);
      }
    } else if (MODE == 2) {
      const double rj = a.r[j * np + i];
      // Four shifts per pass: their loads are in flight together (one
      // shift at a time left the kernel bound by load latency).
#pragma unroll 4
      for (int k = 0; k < ns; ++k) {
        PT* pk = a.ps + (long long)k * (l + 1) * np;
        double v = fma_rn(c0[k], rj, (double)pk[(j + 1) * np + i]);
        v = mul_rn(v, c1[k]);
        pk[(j + 1) * np + i] = (PT)fma_rn(c2[k], (double)pk[j * np + i], v);
      }
    } else {
      for (int q = 0; q < l; ++q) r[q] = a.r[q * np + i];
      // Four shifts per pass: their loads are in flight together (one
      // shift at a time left the kernel bound by load latency).
#pragma unroll 4
      for (int k = 0; k < ns; ++k) {
        PT* pk = a.ps + (long long)k * (l + 1) * np;
        double* xk = a.xs + (long long)k * np;
        double xv = fma_rn(cx[k][0], r[0], xk[i]);
        double p0 = fma_rn(-om[l - 1], (double)pk[l * np + i], (double)pk[i]);
        for (int q = 1; q < l; ++q) {
          p0 = fma_rn(-om[q - 1], (double)pk[q * np + i], p0);
          xv = fma_rn(cx[k][q], r[q], xv);
        }
        xk[i] = xv;
        pk[i] = (PT)mul_rn(p0, c4[k]);
      }
    }
  }
  if (rd.epi) {
    double none[1] = {0.0};
    finish_reduction<0>(none, rd);
  }
}

}  // namespace bk
