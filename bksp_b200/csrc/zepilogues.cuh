// Scalar epilogues of the complex solvers (zbicg, zbicgstabl, zshbicgstabl,
// zblbicgstabl), run like the real ones by one thread of the last block of
// the reduction that produced their inputs.  Complex scalars live in slot
// pairs (solver_defs.h); dot d of the reduction is zld(S, out + 2 d).  Each
// case restates the cited reference statements.  The complex kernels'
// translation unit (kernels_z.cu) includes this file in place of
// epilogues.cuh, so its run_epilogue dispatches the complex codes only.
#pragma once
#include "epi_common.cuh"
#include "zepi_block.cuh"

namespace bk {

// Shared by zbicgstabl's BiCG part (src/bicgstabl.c:190-192):
// beta = -alpha gamma1 / gamma0, gamma0 = gamma1.
__device__ __forceinline__ void zbl_beta(double* S, zc g1) {
  const zc g0 = zld(S, kZG0);
  zst(S, kZBeta, zneg(zdiv(zmul(zld(S, kZAlpha), g1), g0)));
  zst(S, kZG0, g1);
  zst(S, kZG1, g1);
}

// zbicgstabl's omega / omega'' back substitution, src/bicgstabl.c:228-244
// (degree l, omega[1..l]).
__device__ __forceinline__ void zbl_back_substitution(double* S, int l) {
  auto om = [&](int i) { return zld(S, kZOmega + 2 * i); };
  auto tau = [&](int i) { return zld(S, kZTau + 2 * i); };
  zst(S, kZOmega + 2 * l, zld(S, kZOmegaD + 2 * l));
  for (int j = l - 1; j > 0; --j) {
    zc t = zmk(0.0);
    for (int i = j + 1; i <= l; ++i) t = zadd(t, zmul(tau(i * l + j), om(i)));
    zst(S, kZOmega + 2 * j, zsub(zld(S, kZOmegaD + 2 * j), t));
  }
  for (int j = 1; j < l; ++j) {
    zc t = zmk(0.0);
    for (int i = j + 1; i < l; ++i) t = zadd(t, zmul(tau(i * l + j), om(i + 1)));
    zst(S, kZOmegaDD + 2 * j, zadd(om(j + 1), t));
  }
}

// The reference's zhorner (src/util_shift.c:28-50) on omega[0..l-1].
__device__ __forceinline__ void zhorner_shift(const double* S, int l, zc sigma,
                                              zc* out) {
  auto g = [&](int i) { return zld(S, kZOmega + 2 * i); };
  out[l] = zneg(g(l - 1));
  for (int i = l - 1; i > 0; --i) out[i] = zsub(zneg(zmul(sigma, out[i + 1])), g(i - 1));
  out[0] = zadd(zneg(zmul(sigma, out[1])), zmk(1.0));
  for (int i = 1; i < l; ++i)
    for (int j = l - 1; j >= i; --j) out[j] = zsub(out[j], zmul(sigma, out[j + 1]));
  for (int i = 1; i <= l; ++i) out[i] = zneg(zdiv(out[i], out[0]));
}

__device__ __forceinline__ zc zpow_int(zc z, int e) {
  zc r = zmk(1.0);
  for (int q = 0; q < e; ++q) r = zmul(r, z);
  return r;
}

__device__ __forceinline__ double binom_d(int n, int r) {
  double c = 1.0;
  for (int q = 1; q <= r; ++q) c = c * (n - r + q) / q;
  return c;
}

// Complex Cholesky-QR pass on the Hermitian Gram V^H V in kZBkG1: the
// factor of this pass to kZBkScr, its inverse to kZBkRinv, the accumulated
// R (R_pass ... R_1) to kZBkR.  Pass 1 is shifted by 11 (m s + s (s + 1))
// u tr(G) (shifted Cholesky-QR3).
__device__ __forceinline__ bool zqr_pass(double* S, int pass) {
  const int s = (int)S[kZBkS];
  const double* G = S + kZBkG1;
  double* Rp = S + kZBkScr;
  double shift = 0.0;
  if (pass == 1) {
    double tr = 0.0;
    for (int i = 0; i < s; ++i) tr += zm_get(G, s, i, i).re;
    shift = 11.0 * (S[kZBkRows] * s + s * (s + 1.0)) * 1.1102230246251565e-16 * tr;
  }
  if (!zm_chol(G, Rp, s, shift)) return false;
  zm_triinv(Rp, S + kZBkRinv, s);
  if (pass == 1) {
    zm_copy(Rp, S + kZBkR, s);
  } else {
    zm_mul(Rp, S + kZBkR, S + kZBkG2, s);
    zm_copy(S + kZBkG2, S + kZBkR, s);
  }
  return true;
}

__device__ __forceinline__ void zqr_post(double* S, int action) {
  const int s = (int)S[kZBkS];
  switch (action) {
    case ZQR_POST_INIT:      // src/blbicgstabl.c:326: xi = R of V0
      zm_copy(S + kZBkR, S + kZBkXi, s);
      break;
    case ZQR_POST_T:         // :376-390: t = R, xi_old = xi, xi = t xi, t^-1
      zm_copy(S + kZBkR, S + kZBkT, s);
      zm_copy(S + kZBkXi, S + kZBkXiOld, s);
      zm_mul(S + kZBkT, S + kZBkXiOld, S + kZBkXi, s);
      zm_triinv(S + kZBkT, S + kZBkTinv, s);
      zm_mul(S + kZBkAlpha, S + kZBkTinv, S + kZBkATinv, s);
      break;
    default:
      break;
  }
}

// Shifted BiCGSTAB(l), src/shbicgstabl.c:416-442: per-shift scalars of BiCG
// step j and the coefficients of the all-shift kernel's modes 0 and 1.
__device__ __forceinline__ void zsh_shift_step(double* S, zc alpha, zc beta) {
  const int ns = (int)S[kNs];
  const zc alpha_old = zld(S, kZAlphaOld);
  const zc ab = zdiv(zmul(alpha, beta), alpha_old);
  for (int k = 0; k < ns; ++k) {
    const zc sg = zld(S, kZShSigma + 2 * k);
    const zc pi = zld(S, kZShPi + 2 * k), po = zld(S, kZShPiOld + 2 * k);
    const zc th = zld(S, kZShTheta + 2 * k);
    const zc pn = zadd(zmul(zadd(zmk(1.0), zmul(alpha, sg)), pi),
                       zmul(ab, zsub(po, pi)));                       // :418-419
    const zc q = zdiv(po, pi);
    const zc bk = zmul(zmul(q, q), beta);                             // :422-423
    const zc ak = zmul(zdiv(pi, pn), alpha);                          // :426
    zst(S, kZShPiNew + 2 * k, pn);
    zst(S, kZShAlpha + 2 * k, ak);
    zst(S, kZShCb + 2 * k, zneg(bk));                                 // :430
    zst(S, kZShCr + 2 * k, zinv(zmul(pi, th)));                       // :432
    zst(S, kZShCq + 2 * k, zinv(pi));                                 // :437
    zst(S, kZShCn + 2 * k, zneg(zinv(pn)));                           // :456
    zst(S, kZShCs + 2 * k, zinv(zmul(th, ak)));                       // :458
  }
}

// Shifted BiCGSTAB(l) MR part, src/shbicgstabl.c:489-557: the seed's omega
// (l - 1 convention) and omega'', then per shift the Horner polynomial,
// theta update and the all-shift kernel's mode-2 coefficients.
__device__ __forceinline__ void zsh_mr(double* S, int l) {
  auto om = [&](int i) { return zld(S, kZOmega + 2 * i); };
  auto tau = [&](int i) { return zld(S, kZTau + 2 * i); };
  zst(S, kZOmega + 2 * (l - 1), zld(S, kZOmegaD + 2 * (l - 1)));   // :489
  for (int j = l - 2; j >= 0; --j) {                                // :491-497
    zc t = zmk(0.0);
    for (int i = j + 1; i < l; ++i) t = zadd(t, zmul(tau(i * l + j), om(i)));
    zst(S, kZOmega + 2 * j, zsub(zld(S, kZOmegaD + 2 * j), t));
  }
  for (int j = 0; j < l - 1; ++j) {                                 // :499-505
    zc t = zmk(0.0);
    for (int i = j + 1; i < l - 1; ++i) t = zadd(t, zmul(tau(i * l + j), om(i + 1)));
    zst(S, kZOmegaDD + 2 * j, zadd(om(j + 1), t));
  }
  const int ns = (int)S[kNs];
  zc h[kBlMaxL + 1], osd[kBlMaxL];
  for (int k = 0; k < ns; ++k) {                                    // :518-557
    const zc sg = zld(S, kZShSigma + 2 * k);
    zhorner_shift(S, l, sg, h);
    const zc psi = h[0];
    const zc th = zld(S, kZShTheta + 2 * k);
    const zc e = zmul(th, zld(S, kZShPi + 2 * k));                  // :525
    zst(S, kZShTheta + 2 * k, zmul(th, psi));                       // :526
    for (int j = 0; j < l; ++j) {                                   // :528-534
      zc acc = zmk(0.0);
      for (int i = j; i < l; ++i)   // M[k][i l + j] = sigma^(i - j) C(i, j)
        acc = zadd(acc, zmul(zscal(binom_d(i, j), zpow_int(sg, i - j)), h[i + 1]));
      osd[j] = acc;
    }
    zst(S, kZShCx + 2 * (k * kBlMaxL), zdiv(osd[0], e));            // :545
    for (int j = 0; j < l - 1; ++j) {                               // :536-542
      zc acc = zmk(0.0);
      for (int i = j + 1; i < l - 1; ++i) acc = zadd(acc, zmul(tau(i * l + j), osd[i + 1]));
      zst(S, kZShCx + 2 * (k * kBlMaxL + j + 1), zdiv(zadd(osd[j + 1], acc), e));   // :552
    }
    zst(S, kZShCp + 2 * k, zinv(psi));                              // :555
  }
}

static __device__ __noinline__ void run_zepilogue(const Red& rd) {
  double* S = rd.S;
  const int D = rd.out;
  const int l = (int)S[kL];
  switch (rd.epi) {
    case EZ_SET_FNB:
      S[kFnb] = sqrt(S[D]);
      break;
    // ---------------- zbicg, src/bicg.c
    case EZ_BICG_INIT:       // :116-117
      S[kFnb] = sqrt(S[D]);
      zst(S, kZRdot, zld(S, D + 2));
      break;
    case EZ_BICG_ALPHA:      // :130-131
      zst(S, kZAlpha, zdiv(zld(S, kZRdot), zld(S, D)));
      break;
    case EZ_BICG_CHECK: {    // :145-148, :158-161
      const zc rdot = zld(S, D);
      zst(S, kZBeta, zdiv(rdot, zld(S, kZRdot)));
      zst(S, kZRdot, rdot);
      conv_check(rd, sqrt(S[D + 2]) / S[kFnb]);
      break;
    }
    // ---------------- zbicgstabl, src/bicgstabl.c
    case EZ_BL_BETA0:        // :187, then :190-192 for j = 0
      zst(S, kZG0, zmul(zneg(zld(S, kZOmega + 2 * l)), zld(S, kZG0)));
      zbl_beta(S, zld(S, D));
      break;
    case EZ_BL_ALPHA:        // :201-202
      zst(S, kZAlpha, zdiv(zld(S, kZG1), zld(S, D)));
      break;
    case EZ_BL_BETA:         // :190-192
      zbl_beta(S, zld(S, D));
      break;
    case EZ_BL_TAU:          // :218-219  tau[j l + i] = (r_i, r_j) / sigma_i
      zst(S, kZTau + 2 * (rd.a1 * l + rd.a0),
          zdiv(zld(S, D), zld(S, kZSigma + 2 * rd.a0)));
      break;
    case EZ_BL_SIG: {        // :223-225 (+ :228-244 after the last j)
      const int j = rd.a1;
      const zc sg = zld(S, D);
      zst(S, kZSigma + 2 * j, sg);
      zst(S, kZOmegaD + 2 * j, zdiv(zld(S, D + 2), sg));
      if (j == l) zbl_back_substitution(S, l);
      break;
    }
    case EZ_BL_CHECK:        // :260-263, then :187-192 of the next iteration
      conv_check(rd, sqrt(S[D]) / S[kFnb]);
      zst(S, kZG0, zmul(zneg(zld(S, kZOmega + 2 * l)), zld(S, kZG0)));
      zbl_beta(S, zld(S, D + 2));
      break;
    // ---------------- zshbicgstabl, src/shbicgstabl.c
    case EZ_SH_INIT:         // :329
      S[kFnb] = sqrt(S[D]);
      break;
    case EZ_SH_ALPHA: {      // :409-410, :416-442
      const zc alpha = zdiv(zld(S, kZRho), zld(S, D));
      zst(S, kZAlpha, alpha);
      zsh_shift_step(S, alpha, zld(S, kZBeta));
      break;
    }
    case EZ_SH_STEP: {       // :466-471 (+ :394-395 of the next j when a0)
      const int ns = (int)S[kNs];
      zst(S, kZAlphaOld, zld(S, kZAlpha));
      zst(S, kZRdot, zld(S, kZRho));       // rho_old
      for (int k = 0; k < ns; ++k) {
        zst(S, kZShPiOld + 2 * k, zld(S, kZShPi + 2 * k));
        zst(S, kZShPi + 2 * k, zld(S, kZShPiNew + 2 * k));
      }
      if (rd.a0) {
        const zc rho = zld(S, D);
        zst(S, kZRho, rho);
        zst(S, kZBeta, zdiv(zmul(zld(S, kZAlpha), rho), zld(S, kZRdot)));
      }
      break;
    }
    case EZ_SH_TAU:          // :479-480  tau[j l + i] = (r_{i+1}, r_{j+1}) / s_i
    case EZ_BB_TAU:          // src/blbicgstabl.c:414-415, same form on blocks
      zst(S, kZTau + 2 * (rd.a1 * l + rd.a0),
          zdiv(zld(S, D), zld(S, kZSigma + 2 * rd.a0)));
      break;
    case EZ_SH_SIG: {        // :484-486 (+ :489-557 after the last j)
      const int j = rd.a1;
      const zc sg = zld(S, D);
      zst(S, kZSigma + 2 * j, sg);
      zst(S, kZOmegaD + 2 * j, zdiv(zld(S, D + 2), sg));
      if (j == l - 1) zsh_mr(S, l);
      break;
    }
    case EZ_SH_CHECK: {      // :565-568, then :391-395 of the next iteration
      // (a0 = 1: the set-up's launch, which only starts the first iteration)
      if (!rd.a0) conv_check(rd, sqrt(S[D]) / S[kFnb]);
      const zc ro = zmul(zneg(zld(S, kZOmega + 2 * (l - 1))), zld(S, kZRdot));
      zst(S, kZRdot, ro);
      const zc rho = zld(S, D + 2);
      zst(S, kZRho, rho);
      zst(S, kZBeta, zdiv(zmul(zld(S, kZAlpha), rho), ro));
      break;
    }
    // ---------------- complex Cholesky-QR and zblbicgstabl
    case EZ_QR1:
      if (!zqr_pass(S, 1)) fail_divergence(rd);
      break;
    case EZ_QR2:
      if (!zqr_pass(S, 2)) fail_divergence(rd);
      break;
    case EZ_QR3:
      if (!zqr_pass(S, 3)) fail_divergence(rd);
      else zqr_post(S, rd.a0);
      break;
    case EZ_BB_INIT:         // src/blbicgstabl.c:333 ||B||_F, zqreco pass 1 (:326)
      S[kFnb] = sqrt(S[D]);
      if (!zqr_pass(S, 1)) fail_divergence(rd);
      break;
    case EZ_BB_BETA: {       // :343-349  gamma1 = Rs^T V_j, beta = alpha gamma0^-1 gamma1
      const int s = (int)S[kZBkS];
      zm_copy(S + kZBkG1, S + kZBkGam1, s);
      zm_copy(S + kZBkGam0, S + kZBkLU, s);
      if (!zm_lu(S + kZBkLU, S + kZBkPiv, s)) { fail_divergence(rd); break; }
      zm_copy(S + kZBkGam1, S + kZBkScr, s);
      zm_lu_solve(S + kZBkLU, S + kZBkPiv, S + kZBkScr, s);
      zm_mul(S + kZBkAlpha, S + kZBkScr, S + kZBkBeta, s);
      zm_copy(S + kZBkGam1, S + kZBkGam0, s);
      break;
    }
    case EZ_BB_ALPHA: {      // :362-365  alpha = (Rs^T P_{j+1})^-1 gamma1
      const int s = (int)S[kZBkS];
      zm_copy(S + kZBkG1, S + kZBkLU, s);
      if (!zm_lu(S + kZBkLU, S + kZBkPiv, s)) { fail_divergence(rd); break; }
      zm_copy(S + kZBkGam1, S + kZBkAlpha, s);
      zm_lu_solve(S + kZBkLU, S + kZBkPiv, S + kZBkAlpha, s);
      break;
    }
    case EZ_BB_SIG: {        // :419-421 (+ :423-431 after the last j)
      const int j = rd.a1;
      const zc sg = zld(S, D);
      zst(S, kZSigma + 2 * j, sg);
      zst(S, kZOmegaD + 2 * j, zdiv(zld(S, D + 2), sg));
      if (j == l - 1) {
        zst(S, kZOmega + 2 * (l - 1), zld(S, kZOmegaD + 2 * (l - 1)));
        for (int jj = l - 2; jj >= 0; --jj) {
          // t_local is a real double in the reference (:259): only the real
          // part of each product accumulates.
          double t = 0.0;
          for (int i = jj + 1; i < l; ++i)
            t = t + zmul(zld(S, kZTau + 2 * (i * l + jj)), zld(S, kZOmega + 2 * i)).re;
          zst(S, kZOmega + 2 * jj, zsub(zld(S, kZOmegaD + 2 * jj), zmk(t)));
        }
      }
      break;
    }
    case EZ_BB_CHECK: {      // :454-457, then :338-339 of the next iteration
      const int s = (int)S[kZBkS];
      conv_check(rd, zm_fro(S + kZBkXi, s) / S[kFnb]);
      const zc m = zneg(zld(S, kZOmega + 2 * (l - 1)));
      double* g0 = S + kZBkGam0;
      for (int q = 0; q < s * s; ++q) {
        const zc v = zmul(m, zc{g0[2 * q], g0[2 * q + 1]});
        g0[2 * q] = v.re;
        g0[2 * q + 1] = v.im;
      }
      break;
    }
    default:
      break;
  }
}

// The dispatcher finish_reduction calls (dev_common.cuh) in the complex
// kernels' translation unit.
static __device__ __noinline__ void run_epilogue(const Red& rd) {
  run_zepilogue(rd);
}

}  // namespace bk
