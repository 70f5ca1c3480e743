// Scalar-slot layout and scalar-epilogue codes shared by the device
// epilogues (epilogues.cuh) and the host solver drivers.
//
// Every solve owns kScalars FP64 slots S[].  Reduction kernels write their
// dot products to S[kD + d]; the epilogue named in the launch consumes them
// and advances the method's recurrence scalars, all on the device.
#pragma once

namespace bk {

// Common slots.
enum : short {
  kFnb = 0,      // ||b|| (||B||_F for block methods)
  kErr = 1,      // last convergence-test value
  kL = 2,        // degree l (BiCGSTAB(l) family), stored as a double
  kNs = 3,       // number of shifts
  kTrue = 4,     // scratch: true-residual norms etc.
  kBkU = 5,      // block methods: unit roundoff of the block elements
  kD = 8,        // dot outputs D0..D7
  kUser = 16,    // first method-specific slot
};

// CG / CR / BiCG / BiCGSTAB scalars.
enum : short {
  kAlpha = 16, kBeta = 17, kRdotOld = 18, kRho = 19, kOmega1 = 20, kRR = 21,
};

// BiCGSTAB(l) (and the seed system of shifted BiCGSTAB(l)) scalars.
enum : short {
  kBlAlpha = 16, kBlG0 = 17, kBlG1 = 18, kBlBeta = 19,
  kBlOmega = 32,      // omega[0..l]
  kBlOmegaD = 48,     // omega'[0..l]
  kBlOmegaDD = 64,    // omega''[0..l]
  kBlSigma = 80,      // sigma[0..l]
  kBlTau = 96,        // tau[i*l + j], (l+1)^2 <= 81 entries
  kBlMaxL = 8,
  kBlfCr = 180,       // one-pass MR: r0 update coefficients on r_1..r_l
  kBlfCx = 190,       // one-pass MR: x update coefficients on r_1..r_l
  kGramOut = 300,     // pairwise Gram <r_i, r_j>, i <= j (45 slots)
};

// Mixed-precision BiCGSTAB(l) (FP32 vectors, FP64 scalars, FP64 reliable
// residual replacement); shares the BiCGSTAB(l) slots above.
enum : short {
  kMxTarget = 200,    // FP64 true relative residual to reach
  kMxDelta = 201,     // replace when rec < delta * (residual at last replacement)
  kMxLastRep = 202,   // true residual at the last replacement
  kMxDoRep = 203,     // guard: replacement pending in this iteration
  kMxPeriod = 204,    // replace at least every `period` outer iterations
  kMxSinceRep = 205,  // outer iterations since the last replacement
  kMxTrue = 206,      // last FP64 true relative residual
  kMxReps = 207,      // replacements performed
};

// Shifted methods: per-shift arrays (kMaxShifts entries each).
enum : short {
  kMaxShifts = 256,
  kShSigma = 2048,    // sigma_k
  kShPi = 2304,       // pi_k
  kShPiOld = 2560,    // pi_old_k
  kShPiNew = 2816,    // pi_new_k
  kShAlpha = 3072,    // alpha_k
  kShBeta = 3328,     // beta_k
  kShTheta = 3584,    // theta_k (shifted BiCGSTAB(l))
  kShPsiInv = 3840,   // 1 / psi_k
  kShCx = 4096,       // x_k update coefficients, [k][i], 8 per shift
  kShAlphaOld = 24, kShRho = 25, kShRhoOld = 26,   // seed scalars
  kShBetaS = 27, kShAlphaS = 28, kShRhoNext = 29,
};

// Block methods: s-by-s matrices (row-major) in cells of 256 slots.
constexpr short bk_cell(int m) { return (short)(512 + 256 * m); }
enum : short {
  kBkS = 30,                  // block width s (as a double)
  kBkRows = 31,               // block rows n (as a double)
  kBkG1 = bk_cell(0),         // Gram outputs of block kernels
  kBkG2 = bk_cell(1),
  kBkAlpha = bk_cell(2),
  kBkBeta = bk_cell(3),
  kBkC = bk_cell(4),          // Block CG's C
  kBkTmp = bk_cell(5),
  kBkRinv = bk_cell(6),       // inverse of the last Cholesky-QR factor
  kBkR = bk_cell(7),          // accumulated R of the running QR
  kBkLU = bk_cell(8),         // LU of the current s-by-s system
  kBkPiv = bk_cell(9),        // its pivots
  kBkXi = bk_cell(10),        // Block BiCGSTAB(l)'s xi
  kBkGam0 = bk_cell(11),
  kBkGam1 = bk_cell(12),
  kBkT = bk_cell(13),
  kBkTinv = bk_cell(14),
  kBkXiOld = bk_cell(15),
  kBkATinv = bk_cell(16),     // alpha * t^-1
  kBkScr = bk_cell(17),       // scratch
  kBkScr2 = bk_cell(18),
};

// Actions run after the third Cholesky-QR pass (E_QR3's a0).
enum : short {
  QR_POST_NONE = 0,
  QR_POST_BCG = 1,        // beta = R, C = beta C, error = ||C||_F / ||B||_F
  QR_POST_BCG_INIT = 2,   // C = R, beta = I
  QR_POST_BBL_INIT = 3,   // xi = R
  QR_POST_BBL_T = 4,      // t = R: xi_old = xi, xi = t xi, t^-1, alpha t^-1
};

// Epilogue codes.
enum : short {
  E_NONE = 0,
  E_SET_FNB,        // S[kFnb] = sqrt(D0)
  // CG (src/cg.c)
  E_CG_INIT, E_CG_ALPHA, E_CG_CHECK,
  // CR (src/cr.c)
  E_CR_INIT1, E_CR_INIT2, E_CR_SAVE_RR, E_CR_BETA, E_CR_CHECK,
  // BiCG (src/bicg.c)
  E_BICG_INIT, E_BICG_ALPHA, E_BICG_CHECK,
  // BiCGSTAB (src/bicgstab.c)
  E_BS_INIT, E_BS_ALPHA, E_BS_OMEGA, E_BS_CHECK,
  // BiCGSTAB(l) (src/bicgstabl.c)
  E_BL_INIT0, E_BL_BETA0, E_BL_ALPHA, E_BL_BETA, E_BL_TAU, E_BL_SIG,
  E_BL_CHECK,
  E_BLF_MR,         // one-pass minimal-residual step from the Gram matrix
  // mixed-precision BiCGSTAB(l)
  E_MX_INIT, E_MX_INIT2, E_MX_CHECK, E_MX_TRUE, E_MX_REBETA,
  // mixed-precision preconditioned CG
  E_MCG_RHO0, E_MCG_ALPHA, E_MCG_RES, E_MCG_BETA,
  // shifted BiCG (src/shbicg.c)
  E_SHB_INIT, E_SHB_ALPHA, E_SHB_CHECK,
  // shifted BiCGSTAB(l) (src/shbicgstabl.c)
  E_SHL_INIT, E_SHL_BETA, E_SHL_ALPHA, E_SHL_ROTATE, E_SHL_TAU, E_SHL_SIG,
  E_SHL_CHECK,
  // Cholesky-QR passes of the block methods (a0: action after pass 3)
  E_QR1, E_QR2, E_QR3,
  // Block CG (src/blcg.c)
  E_BCG_INIT, E_BCG_ALPHA,
  // Block BiCGSTAB (src/blbicgstab.c)
  E_BBS_INIT, E_BBS_ALPHA, E_BBS_OMEGA, E_BBS_BETA,
  // Block BiCGSTAB(l) (src/blbicgstabl.c)
  E_BBL_INIT, E_BBL_BETA, E_BBL_ALPHA, E_BBL_CHECK,
  E_COUNT_BASE,
};

// ---------------------------------------------------------------- complex
// Complex solves (zsolvers.cpp): a complex scalar occupies the slot pair
// (k, k + 1) = (re, im); a complex dot d of a reduction lands in
// S[kD + 2d], S[kD + 2d + 1].  The common slots kFnb .. kBkU keep their
// meaning.
enum : short {
  kZBkS = 6,          // block width s (as a double)
  kZBkRows = 7,       // block rows (as a double)
  kZAlpha = 16, kZBeta = 18, kZRdot = 20, kZG0 = 22, kZG1 = 24,
  kZAlphaOld = 26, kZRho = 28,
  kZOmega = 32,       // omega[0..l]       (l + 1 <= 9 pairs)
  kZOmegaD = 50,      // omega'[0..l]
  kZOmegaDD = 68,     // omega''[0..l]
  kZSigma = 86,       // sigma[0..l]
  kZTau = 104,        // tau[i], (l + 1)^2 <= 81 pairs, to 265
  kZBkPiv = 280,      // pivots of the complex block LU (s doubles)
  // shifted BiCGSTAB(l): per-shift arrays of kZMaxShifts pairs
  kZMaxShifts = 128,
  kZShSigma = 1024, kZShPi = 1280, kZShPiOld = 1536, kZShPiNew = 1792,
  kZShAlpha = 2048, kZShTheta = 2304, kZShCb = 2560, kZShCr = 2816,
  kZShCq = 3072, kZShCn = 3328, kZShCs = 3584, kZShCp = 3840,
  kZShCx = 4096,      // [k][i], kBlMaxL pairs per shift, to 6143
};

// Complex s-by-s matrices (row-major pairs) of the complex block method in
// cells of 512 slots (kZBkG2 doubles as epilogue scratch).
constexpr short zbk_cell(int m) { return (short)(512 + 512 * m); }
enum : short {
  kZBkG1 = zbk_cell(0), kZBkG2 = zbk_cell(1), kZBkAlpha = zbk_cell(2),
  kZBkBeta = zbk_cell(3), kZBkGam0 = zbk_cell(4), kZBkGam1 = zbk_cell(5),
  kZBkXi = zbk_cell(6), kZBkT = zbk_cell(7), kZBkTinv = zbk_cell(8),
  kZBkLU = zbk_cell(9), kZBkXiOld = zbk_cell(10), kZBkR = zbk_cell(11),
  kZBkScr = zbk_cell(12), kZBkRinv = zbk_cell(13), kZBkATinv = zbk_cell(14),
};

// Complex epilogue codes (zepilogues.cuh), dispatched from run_epilogue.
enum : short {
  EZ_BASE = 200,
  EZ_SET_FNB = EZ_BASE,   // S[kFnb] = sqrt(re D0)
  // zbicg (src/bicg.c:91-177)
  EZ_BICG_INIT, EZ_BICG_ALPHA, EZ_BICG_CHECK,
  // zbicgstabl (src/bicgstabl.c:141-276)
  EZ_BL_BETA0, EZ_BL_ALPHA, EZ_BL_BETA, EZ_BL_TAU, EZ_BL_SIG, EZ_BL_CHECK,
  // zshbicgstabl (src/shbicgstabl.c:288-592)
  EZ_SH_INIT, EZ_SH_ALPHA, EZ_SH_STEP, EZ_SH_TAU, EZ_SH_SIG, EZ_SH_CHECK,
  // complex Cholesky-QR passes (a0: action after pass 3) and zblbicgstabl
  // (src/blbicgstabl.c:255-486)
  EZ_QR1, EZ_QR2, EZ_QR3,
  EZ_BB_INIT, EZ_BB_BETA, EZ_BB_ALPHA, EZ_BB_TAU, EZ_BB_SIG, EZ_BB_CHECK,
  EZ_END,
};

// Actions after the third complex Cholesky-QR pass (EZ_QR3's a0).
enum : short {
  ZQR_POST_NONE = 0,
  ZQR_POST_INIT = 1,   // xi = R
  ZQR_POST_T = 2,      // t = R: xi_old = xi, xi = t xi, t^-1, alpha t^-1
};

}  // namespace bk
