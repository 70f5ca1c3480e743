// Scalar epilogues: the per-iteration scalar work of each Krylov method,
// run by one thread of the last block of the reduction that produced its
// inputs (see finish_reduction).  Each case restates the scalar statements
// of the cited reference lines; vector work lives in the launching kernels.
#pragma once
#include "dev_common.cuh"
#include "solver_defs.h"

namespace bk {

// Convergence test shared by every method: `error < tol` passes (the
// reference's `if (error < tol) break;`), a non-finite error is a breakdown,
// otherwise the iteration index advances until max_iter.
__device__ __forceinline__ void conv_check(const Red& rd, double err) {
  Ctl* c = rd.ctl;
  rd.S[kErr] = err;
  if (c->hist && c->hist_len < c->hist_cap) c->hist[c->hist_len] = err;
  c->hist_len++;
  const int it = c->iter;
  if (err < c->tol) {
    c->done = 1;
    c->ret = it;
  } else if (!isfinite(err)) {
    c->done = 1;
    c->ret = kDivergence;
  } else {
    c->iter = it + 1;
    if (it + 1 >= c->max_iter) {
      c->done = 1;
      c->ret = kNotConverged;
    }
  }
}

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

__device__ __forceinline__ void bl_beta0(double* S, int l, double g1) {
  // src/bicgstabl.c:57 gamma0 = -omega[l] gamma0, then :60-62 for j = 0.
  const double g0 = -S[kBlOmega + l] * S[kBlG0];
  S[kBlBeta] = -S[kBlAlpha] * g1 / g0;
  S[kBlG0] = g1;
  S[kBlG1] = g1;
}

static __device__ void run_epilogue(const Red& rd) {
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
    default:
      break;
  }
}

}  // namespace bk
