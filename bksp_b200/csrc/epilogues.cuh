// Scalar epilogues: the per-iteration scalar work of each Krylov method,
// run by one thread of the last block of the reduction that produced its
// inputs (see finish_reduction).  Each case restates the scalar statements
// of the cited reference lines; vector work lives in the launching kernels.
#pragma once
#include "dev_common.cuh"
#include "solver_defs.h"
#include "epi_block.cuh"
#include "epi_common.cuh"

namespace bk {


__device__ __forceinline__ void bl_back_substitution(double* S, int l) {
  // src/bicgstabl.c:93-109
  double* om = S + kBlOmega;
  const double* omd = S + kBlOmegaD;
  double* omdd = S + kBlOmegaDD;
  const double* tau = S + kBlTau;
  om[l] = omd[l];
  for (int j = l - 1; j > 0; --j) {
    double t = 0.0;
    for (int i = j + 1; i <= l; ++i) t += tau[j * l + i] * om[i];
    om[j] = omd[j] - t;
  }
  for (int j = 1; j < l; ++j) {
    double t = 0.0;
    for (int i = j + 1; i < l; ++i) t += tau[j * l + i] * om[i + 1];
    omdd[j] = om[j + 1] + t;
  }
}

// Shifted BiCGSTAB(l) helpers (src/shbicgstabl.c, src/util_shift.c).
__device__ __forceinline__ void horner_shift(const double* gamma, int l,
                                             double sigma, double* out) {
  // The reference's dhorner (src/util_shift.c:5-27), step for step.
  out[l] = -gamma[l - 1];
  for (int i = l - 1; i > 0; --i) out[i] = -sigma * out[i + 1] - gamma[i - 1];
  out[0] = -sigma * out[1] + 1.0;
  for (int i = 1; i < l; ++i)
    for (int j = l - 1; j >= i; --j) out[j] += -sigma * out[j + 1];
  for (int i = 1; i <= l; ++i) out[i] = -out[i] / out[0];
}

__device__ __forceinline__ double binom(int n, int r) {
  if (n < 0 || r < 0 || n < r) return 0.0;
  double c = 1.0;
  for (int q = 1; q <= r; ++q) c = c * (double)(n - r + q) / (double)q;
  return c;
}

__device__ __forceinline__ double ipow(double x, int p) {
  double y = 1.0;
  for (int q = 0; q < p; ++q) y *= x;
  return y;
}

// End of the MR part of shifted BiCGSTAB(l): seed omega, omega'' and the
// per-shift update coefficients (src/shbicgstabl.c:175-227).
static __device__ void shl_mr_finish(double* S, int l, int ns) {
  double* om = S + kBlOmega;
  const double* omd = S + kBlOmegaD;
  double* omdd = S + kBlOmegaDD;
  const double* tau = S + kBlTau;
  om[l - 1] = omd[l - 1];
  for (int j = l - 2; j >= 0; --j) {
    double t = 0.0;
    for (int i = j + 1; i < l; ++i) t += tau[j * l + i] * om[i];
    om[j] = omd[j] - t;
  }
  for (int j = 0; j < l - 1; ++j) {
    double t = 0.0;
    for (int i = j + 1; i < l - 1; ++i) t += tau[j * l + i] * om[i + 1];
    omdd[j] = om[j + 1] + t;
  }
  for (int k = 0; k < ns; ++k) {
    const double sg = S[kShSigma + k];
    double h[kBlMaxL + 1], oms[kBlMaxL], omsd[kBlMaxL], omsdd[kBlMaxL];
    horner_shift(om, l, sg, h);
    const double psi = h[0];
    for (int i = 0; i < l; ++i) oms[i] = h[i + 1];
    const double e = S[kShTheta + k] * S[kShPi + k];
    S[kShTheta + k] = S[kShTheta + k] * psi;
    for (int j = 0; j < l; ++j) {
      double t = 0.0;
      for (int i = j; i < l; ++i) t += ipow(sg, i - j) * binom(i, j) * oms[i];
      omsd[j] = t;
    }
    for (int j = 0; j < l - 1; ++j) {
      double t = 0.0;
      for (int i = j + 1; i < l - 1; ++i) t += tau[j * l + i] * omsd[i + 1];
      omsdd[j] = omsd[j + 1] + t;
    }
    double* cx = S + kShCx + k * 8;
    cx[0] = omsd[0] / e;
    for (int i = 1; i < l; ++i) cx[i] = omsdd[i - 1] / e;
    S[kShPsiInv + k] = 1.0 / psi;
  }
}

// pi_new / beta_k / alpha_k of every shift after a seed alpha (shared by
// shifted BiCG, src/shbicg.c:78-88, and shifted BiCGSTAB(l), :111-121).
__device__ __forceinline__ void shift_scalars(double* S, int ns, double alpha,
                                              double beta) {
  const double aold = S[kShAlphaOld];
  for (int k = 0; k < ns; ++k) {
    const double pi = S[kShPi + k], po = S[kShPiOld + k];
    const double pn = (1.0 + alpha * S[kShSigma + k]) * pi +
                      alpha * beta / aold * (po - pi);
    S[kShPiNew + k] = pn;
    S[kShBeta + k] = (po / pi) * (po / pi) * beta;
    S[kShAlpha + k] = pi / pn * alpha;
  }
}

__device__ __forceinline__ void shift_rotate(double* S, int ns) {
  for (int k = 0; k < ns; ++k) {
    S[kShPiOld + k] = S[kShPi + k];
    S[kShPi + k] = S[kShPiNew + k];
  }
}

// One Cholesky-QR pass on the Gram matrix in kBkG1: R_pass with
// R^T R = G (+ shift), kBkRinv = R^-1, kBkR = R_pass * kBkR (kBkR = R_pass
// for the first pass).  The first pass is shifted (shifted CholeskyQR3,
// Fukaya et al. 2020), so the three passes together give Q R = V with
// orthonormal Q to rounding for any numerically full-rank V.
static __device__ bool qr_pass(double* S, int pass) {
  const int s = (int)S[kBkS];
  double* G = S + kBkG1;
  double* Rp = S + kBkScr;
  double shift = 0.0;
  if (pass == 1) {
    double tr = 0.0;
    for (int i = 0; i < s; ++i) tr += G[i * s + i];
    const double m = S[kBkRows];
    // unit roundoff of the data: FP64 blocks, or FP32 blocks (mixed solves)
    const double u = S[kBkU] > 0.0 ? S[kBkU] : 1.1102230246251565e-16;
    shift = 11.0 * (m * s + s * (s + 1.0)) * u * tr;
  }
  if (!dm_chol(G, Rp, s, shift)) return false;
  dm_triinv(Rp, S + kBkRinv, s);
  if (pass == 1) {
    dm_copy(Rp, S + kBkR, s);
  } else {
    dm_mul(Rp, S + kBkR, S + kBkScr2, s);
    dm_copy(S + kBkScr2, S + kBkR, s);
  }
  return true;
}

static __device__ void qr_post(const Red& rd, int action) {
  double* S = rd.S;
  const int s = (int)S[kBkS];
  switch (action) {
    case QR_POST_BCG:        // src/blcg.c:95-105
      dm_copy(S + kBkR, S + kBkBeta, s);
      dm_mul(S + kBkBeta, S + kBkC, S + kBkScr, s);
      dm_copy(S + kBkScr, S + kBkC, s);
      conv_check(rd, dm_fro(S + kBkC, s) / S[kFnb]);
      break;
    case QR_POST_BCG_INIT:   // src/blcg.c:58, :61-63
      dm_copy(S + kBkR, S + kBkC, s);
      dm_eye(S + kBkBeta, s);
      break;
    case QR_POST_BBL_INIT:   // src/blbicgstabl.c:88
      dm_copy(S + kBkR, S + kBkXi, s);
      break;
    case QR_POST_BBL_T:      // src/blbicgstabl.c:135-148
      dm_copy(S + kBkR, S + kBkT, s);
      dm_copy(S + kBkXi, S + kBkXiOld, s);
      dm_mul(S + kBkT, S + kBkXiOld, S + kBkXi, s);
      dm_copy(S + kBkT, S + kBkScr, s);
      dm_inv(S + kBkScr, S + kBkPiv, S + kBkTinv, s);
      dm_mul(S + kBkAlpha, S + kBkTinv, S + kBkATinv, s);
      break;
    default:
      break;
  }
}


// One-pass minimal-residual step of BiCGSTAB(l): the modified Gram-Schmidt
// quantities of src/bicgstabl.c:84-91 (tau_ij, sigma_j, omega'_j) from the
// Gram matrix G_ij = <r_i, r_j> by an LDL^T recurrence (equal in exact
// arithmetic), the omega / omega'' back substitution, and the update
// coefficients mapped from the orthogonalised r'_j back onto r_j
// (r' = r U^-1 with U unit upper, U_ij = tau_ij).
// Compile-time degree L: the Gram entries are loaded once (independent
// loads) and the whole recurrence runs in registers, so the one thread's
// dependent chain pays register latency, not a memory round trip per step.
template <int L>
static __device__ __noinline__ void blf_mr_t(double* S) {
  constexpr int M = L + 1;
  double g[M][M];
#pragma unroll
  for (int i = 0; i < M; ++i)
#pragma unroll
    for (int j = i; j < M; ++j) {
      const double v = S[kGramOut + i * M - i * (i - 1) / 2 + (j - i)];
      g[i][j] = v;
      g[j][i] = v;
    }
  double tau[M][M], sig[M], h[M], omd[M], om[M], omdd[M], cr[M], cx[M];
#pragma unroll
  for (int j = 1; j <= L; ++j) {
#pragma unroll
    for (int i = 1; i < j; ++i) {
      double t = g[i][j];
#pragma unroll
      for (int k = 1; k < i; ++k) t -= tau[k][i] * sig[k] * tau[k][j];
      tau[i][j] = t / sig[i];
    }
    double sj = g[j][j];
#pragma unroll
    for (int k = 1; k < j; ++k) sj -= tau[k][j] * tau[k][j] * sig[k];
    sig[j] = sj;
    double hj = g[0][j];
#pragma unroll
    for (int i = 1; i < j; ++i) hj -= tau[i][j] * h[i];
    h[j] = hj;
    omd[j] = hj / sj;
  }
  // src/bicgstabl.c:93-109 (bl_back_substitution) on the register copies.
  om[L] = omd[L];
#pragma unroll
  for (int j = L - 1; j > 0; --j) {
    double t = 0.0;
#pragma unroll
    for (int i = j + 1; i <= L; ++i) t += tau[j][i] * om[i];
    om[j] = omd[j] - t;
  }
#pragma unroll
  for (int j = 1; j < L; ++j) {
    double t = 0.0;
#pragma unroll
    for (int i = j + 1; i < L; ++i) t += tau[j][i] * om[i + 1];
    omdd[j] = om[j + 1] + t;
  }
#pragma unroll
  for (int j = 1; j <= L; ++j) {
    cr[j] = omd[j];
    cx[j] = j < L ? omdd[j] : 0.0;
  }
#pragma unroll
  for (int i = L - 1; i >= 1; --i)
#pragma unroll
    for (int j = i + 1; j <= L; ++j) {
      cr[i] -= tau[i][j] * cr[j];
      cx[i] -= tau[i][j] * cx[j];
    }
#pragma unroll
  for (int j = 1; j <= L; ++j) {
#pragma unroll
    for (int i = 1; i < j; ++i) S[kBlTau + i * L + j] = tau[i][j];
    S[kBlSigma + j] = sig[j];
    S[kBlOmegaD + j] = omd[j];
    S[kBlOmega + j] = om[j];
    if (j < L) S[kBlOmegaDD + j] = omdd[j];
    S[kBlfCr + j] = cr[j];
    S[kBlfCx + j] = cx[j];
  }
}

static __device__ void blf_mr(double* S, int l) {
  switch (l) {
    case 1: blf_mr_t<1>(S); break;
    case 2: blf_mr_t<2>(S); break;
    case 3: blf_mr_t<3>(S); break;
    case 4: blf_mr_t<4>(S); break;
    case 5: blf_mr_t<5>(S); break;
    case 6: blf_mr_t<6>(S); break;
    case 7: blf_mr_t<7>(S); break;
    default: blf_mr_t<8>(S); break;
  }
}

__device__ __forceinline__ void bl_beta0(double* S, int l, double g1) {
  // src/bicgstabl.c:57 gamma0 = -omega[l] gamma0, then :60-62 for j = 0.
  const double g0 = -S[kBlOmega + l] * S[kBlG0];
  S[kBlBeta] = -S[kBlAlpha] * g1 / g0;
  S[kBlG0] = g1;
  S[kBlG1] = g1;
}


static __device__ __noinline__ void run_epilogue(const Red& rd) {
  double* S = rd.S;
  const double* D = S + rd.out;
  const int l = (int)S[kL];
  switch (rd.epi) {
    case E_SET_FNB:
      S[kFnb] = sqrt(D[0]);
      break;
    // ---------------- CG, src/cg.c
    case E_CG_INIT:          // :29-30
      S[kFnb] = sqrt(D[0]);
      S[kRdotOld] = D[1];
      break;
    case E_CG_ALPHA:         // :39
      S[kAlpha] = S[kRdotOld] / D[0];
      break;
    case E_CG_CHECK: {       // :48-50, :56-59
      const double rdot = D[0];
      S[kBeta] = rdot / S[kRdotOld];
      S[kRdotOld] = rdot;
      conv_check(rd, sqrt(rdot) / S[kFnb]);
      break;
    }
    // ---------------- CR, src/cr.c
    case E_CR_INIT1:         // :34
      S[kFnb] = sqrt(D[0]);
      break;
    case E_CR_INIT2:         // :33, then :39 for the first iteration
      S[kRdotOld] = D[0];
      S[kAlpha] = S[kRdotOld] / D[1];
      break;
    case E_CR_SAVE_RR:
      S[kRR] = D[0];
      break;
    case E_CR_BETA: {        // :51-53
      const double rdot = D[0];
      S[kBeta] = rdot / S[kRdotOld];
      S[kRdotOld] = rdot;
      break;
    }
    case E_CR_CHECK:         // :64-67, then :39 of the next iteration
      conv_check(rd, sqrt(S[kRR]) / S[kFnb]);
      S[kAlpha] = S[kRdotOld] / D[0];
      break;
    // ---------------- BiCG, src/bicg.c
    case E_BICG_INIT:        // :28-29
      S[kFnb] = sqrt(D[0]);
      S[kRdotOld] = D[1];
      break;
    case E_BICG_ALPHA:       // :42
      S[kAlpha] = S[kRdotOld] / D[0];
      break;
    case E_BICG_CHECK: {     // :54-56, :66-69
      const double rdot = D[0];
      S[kBeta] = rdot / S[kRdotOld];
      S[kRdotOld] = rdot;
      conv_check(rd, sqrt(D[1]) / S[kFnb]);
      break;
    }
    // ---------------- BiCGSTAB, src/bicgstab.c
    case E_BS_INIT:          // :29-30
      S[kFnb] = sqrt(D[0]);
      S[kRho] = D[1];
      break;
    case E_BS_ALPHA:         // :36
      S[kAlpha] = S[kRho] / D[0];
      break;
    case E_BS_OMEGA:         // :43
      S[kOmega1] = D[0] / D[1];
      break;
    case E_BS_CHECK: {       // :51-53, :59-62
      const double rn = D[0];
      S[kBeta] = S[kAlpha] / S[kOmega1] * rn / S[kRho];
      S[kRho] = rn;
      conv_check(rd, sqrt(D[1]) / S[kFnb]);
      break;
    }
    // ---------------- BiCGSTAB(l), src/bicgstabl.c
    case E_BL_INIT0:         // :39, :51, alpha = 0, gamma0 = 1
      S[kFnb] = sqrt(D[0]);
      S[kBlAlpha] = 0.0;
      S[kBlG0] = 1.0;
      S[kBlOmega + l] = 1.0;
      break;
    case E_BL_BETA0:         // :57, :60-62 (j = 0)
      bl_beta0(S, l, D[0]);
      break;
    case E_BL_ALPHA:         // :71
      S[kBlAlpha] = S[kBlG1] / D[0];
      break;
    case E_BL_BETA: {        // :60-62 (j > 0)
      const double g1 = D[0];
      S[kBlBeta] = -S[kBlAlpha] * g1 / S[kBlG0];
      S[kBlG0] = g1;
      S[kBlG1] = g1;
      break;
    }
    case E_BL_TAU:           // :86
      S[kBlTau + rd.a0 * l + rd.a1] = D[0] / S[kBlSigma + rd.a0];
      break;
    case E_BL_SIG:           // :89-90
      S[kBlSigma + rd.a1] = D[0];
      S[kBlOmegaD + rd.a1] = D[1] / D[0];
      if (rd.a1 == l) bl_back_substitution(S, l);
      break;
    case E_BLF_MR:           // :84-109 in one pass (see blf_mr)
      blf_mr(S, l);
      break;
    case E_BL_CHECK:         // :122-125, then :57-62 of the next iteration
      conv_check(rd, sqrt(D[0]) / S[kFnb]);
      if (!rd.ctl->done) bl_beta0(S, l, D[1]);
      break;
    // ---------------- mixed-precision BiCGSTAB(l) (no reference counterpart;
    // the BiCG / MR scalar steps are the E_BL_* cases above)
    case E_MX_INIT: {        // r64 = b - A x0: D0 = (r, r), D1 = (b, b)
      S[kFnb] = sqrt(D[1]);
      const double t = sqrt(D[0]) / S[kFnb];
      S[kMxTrue] = t;
      S[kMxLastRep] = t;
      S[kMxSinceRep] = 0.0;
      S[kMxReps] = 0.0;
      S[kMxDoRep] = 0.0;
      if (t <= S[kMxTarget]) {
        rd.ctl->done = 1;
        rd.ctl->ret = rd.ctl->iter;
      } else if (!isfinite(t)) {
        rd.ctl->done = 1;
        rd.ctl->ret = kDivergence;
      }
      break;
    }
    case E_MX_INIT2:         // r0 = p0 = rs = fl(r64): D0 = (rs, r0)
      S[kBlAlpha] = 0.0;
      S[kBlG0] = 1.0;
      S[kBlOmega + l] = 1.0;
      bl_beta0(S, l, D[0]);
      break;
    case E_MX_CHECK: {       // after the update: D0 = (r0, r0), D1 = (rs, r0)
      Ctl* c = rd.ctl;
      const double rec = sqrt(D[0]) / S[kFnb];
      S[kErr] = rec;
      if (c->hist && c->hist_len < c->hist_cap) c->hist[c->hist_len] = rec;
      c->hist_len++;
      if (!isfinite(rec)) {
        c->done = 1;
        c->ret = kDivergence;
        break;
      }
      S[kMxSinceRep] += 1.0;
      const bool rep = rec <= S[kMxTarget] ||
                       rec < S[kMxDelta] * S[kMxLastRep] ||
                       S[kMxSinceRep] >= S[kMxPeriod];
      // The replacement block runs as a conditional node of the captured
      // iteration when there is one (only then are its kernels launched).
      if (c->use_cond)
        cudaGraphSetConditional((cudaGraphConditionalHandle)c->cond, rep ? 1u : 0u);
      if (rep) {
        S[kMxDoRep] = 1.0;   // the replacement block decides convergence
      } else {
        S[kMxDoRep] = 0.0;
        bl_beta0(S, l, D[1]);
        c->iter++;
        if (c->iter >= c->max_iter) {
          c->done = 1;
          c->ret = kNotConverged;
        }
      }
      break;
    }
    case E_MX_TRUE: {        // r64 = b - A x64 after accumulation: D0 = (r, r)
      Ctl* c = rd.ctl;
      const double t = sqrt(D[0]) / S[kFnb];
      S[kMxTrue] = t;
      S[kMxLastRep] = t;
      S[kMxSinceRep] = 0.0;
      S[kMxReps] += 1.0;
      if (t <= S[kMxTarget]) {
        c->done = 1;
        c->ret = c->iter;
      } else if (!isfinite(t)) {
        c->done = 1;
        c->ret = kDivergence;
      } else {
        c->iter++;
        if (c->iter >= c->max_iter) {
          c->done = 1;
          c->ret = kNotConverged;
        }
      }
      break;
    }
    case E_MX_REBETA:        // r0 = fl(r64) replaced: D0 = (rs, r0)
      S[kMxDoRep] = 0.0;
      bl_beta0(S, l, D[0]);
      break;
    // ---------------- mixed-precision preconditioned CG (no reference
    // counterpart; the recurrence is src/cg.c:35-54 with z = M r).
    // E_MCG_RES's a0: 0 = (r, z) comes later (E_MCG_BETA), else it is
    // D[a0 - 1] of this reduction.
    case E_MCG_RHO0:         // after r = fl(r64), z = M r: D0 = (r, z)
      S[kRho] = D[0];
      break;
    case E_MCG_ALPHA:        // q = A p: D0 = (p, q)
      S[kAlpha] = S[kRho] / D[0];
      break;
    case E_MCG_RES: {        // after y += alpha p, r -= alpha q: D0 = (r, r)
      Ctl* c = rd.ctl;
      const double rec = sqrt(D[0]) / S[kFnb];
      S[kErr] = rec;
      if (c->hist && c->hist_len < c->hist_cap) c->hist[c->hist_len] = rec;
      c->hist_len++;
      if (!isfinite(rec)) {
        c->done = 1;
        c->ret = kDivergence;
        break;
      }
      S[kMxSinceRep] += 1.0;
      const bool rep = rec <= S[kMxTarget] ||
                       rec < S[kMxDelta] * S[kMxLastRep] ||
                       S[kMxSinceRep] >= S[kMxPeriod];
      if (c->use_cond)   // a1: which of the body's conditional nodes
        cudaGraphSetConditional(
            (cudaGraphConditionalHandle)(rd.a1 ? c->cond_alt : c->cond), rep ? 1u : 0u);
      S[kMxDoRep] = rep ? 1.0 : 0.0;
      if (!rep) {
        if (rd.a0) {   // (r, z) in D[a0 - 1] (z = r: D0; fused M r: D1)
          const double rz = D[rd.a0 - 1];
          S[kBeta] = rz / S[kRho];
          S[kRho] = rz;
        }
        c->iter++;
        if (c->iter >= c->max_iter) {
          c->done = 1;
          c->ret = kNotConverged;
        }
      }
      break;
    }
    case E_MCG_BETA:         // z = M r (or the replaced r): D0 = (r, z)
      S[kMxDoRep] = 0.0;
      S[kBeta] = D[0] / S[kRho];
      S[kRho] = D[0];
      break;
    // ---------------- shifted BiCG, src/shbicg.c
    case E_SHB_INIT: {       // :27-46; then rho / beta of iteration 0 (:52-53)
      const int ns = (int)S[kNs];
      S[kFnb] = sqrt(D[0]);
      S[kShAlphaOld] = 1.0;
      S[kShRhoOld] = 1.0;
      for (int k = 0; k < ns; ++k) {
        S[kShPi + k] = 1.0;
        S[kShPiOld + k] = 1.0;
      }
      S[kShRho] = D[1];
      S[kShBetaS] = -S[kShRho] / S[kShRhoOld];
      break;
    }
    case E_SHB_ALPHA: {      // :72, :78-88
      const double alpha = S[kShRho] / D[0];
      S[kShAlphaS] = alpha;
      shift_scalars(S, (int)S[kNs], alpha, S[kShBetaS]);
      break;
    }
    case E_SHB_CHECK: {      // :105-115, then :52-53 of the next iteration
      const int ns = (int)S[kNs];
      S[kShAlphaOld] = S[kShAlphaS];
      S[kShRhoOld] = S[kShRho];
      shift_rotate(S, ns);
      conv_check(rd, sqrt(D[1]) / S[kFnb]);
      S[kShRho] = D[0];
      S[kShBetaS] = -S[kShRho] / S[kShRhoOld];
      break;
    }
    // ---------------- shifted BiCGSTAB(l), src/shbicgstabl.c
    case E_SHL_INIT: {       // :25, :39-43, :60-66; then :88-92 (m = 0, j = 0)
      const int ns = (int)S[kNs];
      S[kFnb] = sqrt(D[0]);
      S[kBlAlpha] = 0.0;
      S[kShAlphaOld] = 1.0;
      S[kShRhoOld] = 1.0;
      for (int i = 0; i < l; ++i) S[kBlOmega + i] = 0.0;
      S[kBlOmega + l - 1] = 1.0;
      for (int k = 0; k < ns; ++k) {
        S[kShPi + k] = 1.0;
        S[kShPiOld + k] = 1.0;
        S[kShTheta + k] = 1.0;
      }
      S[kShRhoOld] = -S[kBlOmega + l - 1] * S[kShRhoOld];
      S[kShRho] = D[1];
      S[kBlBeta] = S[kBlAlpha] * S[kShRho] / S[kShRhoOld];
      break;
    }
    case E_SHL_BETA:         // :91 (j > 0); beta after the rotation below
      S[kShRhoNext] = D[0];
      break;
    case E_SHL_ALPHA:        // :105, :111-121
      S[kBlAlpha] = S[kShRho] / D[0];
      shift_scalars(S, (int)S[kNs], S[kBlAlpha], S[kBlBeta]);
      break;
    case E_SHL_ROTATE:       // :156-161, then :91-92 of step j + 1 (a0 = 1)
      S[kShAlphaOld] = S[kBlAlpha];
      S[kShRhoOld] = S[kShRho];
      shift_rotate(S, (int)S[kNs]);
      if (rd.a0) {
        S[kShRho] = S[kShRhoNext];
        S[kBlBeta] = S[kBlAlpha] * S[kShRho] / S[kShRhoOld];
      }
      break;
    case E_SHL_TAU:          // :168
      S[kBlTau + rd.a0 * l + rd.a1] = D[0] / S[kBlSigma + rd.a0];
      break;
    case E_SHL_SIG:          // :171-172, then :175-227 after the last one
      S[kBlSigma + rd.a1] = D[0];
      S[kBlOmegaD + rd.a1] = D[1] / D[0];
      if (rd.a1 == l - 1) shl_mr_finish(S, l, (int)S[kNs]);
      break;
    case E_SHL_CHECK:        // :244-247, then :88-92 of the next iteration
      conv_check(rd, sqrt(D[0]) / S[kFnb]);
      if (!rd.ctl->done) {
        S[kShRhoOld] = -S[kBlOmega + l - 1] * S[kShRhoOld];
        S[kShRho] = D[1];
        S[kBlBeta] = S[kBlAlpha] * S[kShRho] / S[kShRhoOld];
      }
      break;
    // ---------------- Cholesky-QR passes
    case E_QR1:
      if (!qr_pass(S, 1)) fail_divergence(rd);
      break;
    case E_QR2:
      if (!qr_pass(S, 2)) fail_divergence(rd);
      break;
    case E_QR3:
      if (!qr_pass(S, 3)) fail_divergence(rd);
      else qr_post(rd, rd.a0);
      break;
    // ---------------- Block CG, src/blcg.c
    case E_BCG_INIT:         // :60 ||B||_F, then the first pass of myqr (:58)
      S[kFnb] = sqrt(D[0]);
      if (!qr_pass(S, 1)) fail_divergence(rd);
      break;
    case E_BCG_ALPHA: {      // :78-86  alpha = (P^T A P)^-1, tmp = alpha C
      const int s = (int)S[kBkS];
      dm_copy(S + kBkG1, S + kBkLU, s);
      dm_inv(S + kBkLU, S + kBkPiv, S + kBkAlpha, s);
      dm_mul(S + kBkAlpha, S + kBkC, S + kBkTmp, s);
      break;
    }
    // ---------------- Block BiCGSTAB, src/blbicgstab.c
    case E_BBS_INIT:         // :175
      S[kFnb] = sqrt(D[0]);
      break;
    case E_BBS_ALPHA: {      // :185-189  alpha = (Rs^T V)^-1 (Rs^T R)
      const int s = (int)S[kBkS];
      dm_copy(S + kBkG1, S + kBkLU, s);
      dm_lu(S + kBkLU, S + kBkPiv, s);
      dm_copy(S + kBkG2, S + kBkAlpha, s);
      dm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkAlpha, s, s);
      break;
    }
    case E_BBS_OMEGA:        // :200-201
      S[kOmega1] = D[0] / D[1];
      break;
    case E_BBS_BETA: {       // :212-214, :226-229
      const int s = (int)S[kBkS];
      for (int q = 0; q < s * s; ++q) S[kBkBeta + q] = -S[kBkG1 + q];
      dm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkBeta, s, s);
      conv_check(rd, sqrt(D[0]) / S[kFnb]);
      break;
    }
    // ---------------- Block BiCGSTAB(l), src/blbicgstabl.c
    case E_BBL_INIT: {       // :31-38, :67-76, :93 and the first myqr pass (:88)
      const int s = (int)S[kBkS];
      S[kFnb] = sqrt(D[0]);
      for (int q = 0; q < s * s; ++q) S[kBkAlpha + q] = 0.0;
      dm_eye(S + kBkGam0, s);
      for (int i = 0; i <= l; ++i) S[kBlOmega + i] = 0.0;
      S[kBlOmega + l] = 1.0;
      // :98  gamma0 = -omega[l] gamma0 of the first iteration
      for (int q = 0; q < s * s; ++q) S[kBkGam0 + q] *= -S[kBlOmega + l];
      if (!qr_pass(S, 1)) fail_divergence(rd);
      break;
    }
    case E_BBL_BETA: {       // :102-108  beta = -alpha gamma0^-1 gamma1
      const int s = (int)S[kBkS];
      dm_copy(S + kBkG1, S + kBkGam1, s);
      dm_copy(S + kBkGam0, S + kBkLU, s);
      dm_lu(S + kBkLU, S + kBkPiv, s);
      dm_copy(S + kBkGam1, S + kBkTmp, s);
      dm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkTmp, s, s);
      dm_mul(S + kBkAlpha, S + kBkTmp, S + kBkBeta, s);
      for (int q = 0; q < s * s; ++q) S[kBkBeta + q] = -S[kBkBeta + q];
      dm_copy(S + kBkGam1, S + kBkGam0, s);
      break;
    }
    case E_BBL_ALPHA: {      // :121-124  alpha = (Rs^T P_{j+1})^-1 gamma1
      const int s = (int)S[kBkS];
      dm_copy(S + kBkG1, S + kBkLU, s);
      dm_lu(S + kBkLU, S + kBkPiv, s);
      dm_copy(S + kBkGam1, S + kBkAlpha, s);
      dm_lu_solve(S + kBkLU, S + kBkPiv, S + kBkAlpha, s, s);
      break;
    }
    case E_BBL_CHECK: {      // :209-212, then :98 of the next iteration
      const int s = (int)S[kBkS];
      const double err = dm_fro(S + kBkXi, s) / S[kFnb];
      conv_check(rd, err);
      for (int q = 0; q < s * s; ++q) S[kBkGam0 + q] *= -S[kBlOmega + l];
      break;
    }
    default:
      break;
  }
}

}  // namespace bk
