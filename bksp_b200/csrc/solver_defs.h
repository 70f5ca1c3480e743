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
  // mixed-precision BiCGSTAB(l)
  E_MX_INIT, E_MX_INIT2, E_MX_CHECK, E_MX_TRUE, E_MX_REBETA,
  // shifted BiCG (src/shbicg.c)
  E_SHB_INIT, E_SHB_ALPHA, E_SHB_CHECK,
  // shifted BiCGSTAB(l) (src/shbicgstabl.c)
  E_SHL_INIT, E_SHL_BETA, E_SHL_ALPHA, E_SHL_ROTATE, E_SHL_TAU, E_SHL_SIG,
  E_SHL_CHECK,
  E_COUNT_BASE,
};

}  // namespace bk
