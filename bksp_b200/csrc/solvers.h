// Device-resident Krylov solvers.  Each takes an uploaded operator, device
// vectors (padded to pad64(n), zero beyond n) and returns the bksp return
// code; the iteration runs entirely on the GPU (see dev_common.cuh).
#pragma once

#include "runtime.h"

namespace bk {

struct SolveOut {
  int ret = 0;           // bksp return code
  int iters = 0;         // convergence tests performed
  double err = 0.0;      // last convergence-test value
};

// Single right-hand side, FP64 (reference-parity methods).
SolveOut cg(const DevCsr& A, const double* b, double* x, double tol,
            int max_iter, SolveState& ss, cudaStream_t st);
SolveOut cr(const DevCsr& A, const double* b, double* x, double tol,
            int max_iter, SolveState& ss, cudaStream_t st);
SolveOut bicg(const DevCsr& A, const DevCsr& At, const double* b, double* x,
              double tol, int max_iter, SolveState& ss, cudaStream_t st);
SolveOut bicgstab(const DevCsr& A, const double* b, double* x, double tol,
                  int max_iter, SolveState& ss, cudaStream_t st);
// fast_mr: the minimal-residual step from one Gram pass (blf_mr) instead
// of the reference's modified Gram-Schmidt sweeps.
SolveOut bicgstabl(const DevCsr& A, const double* b, int l, double* x,
                   double tol, int max_iter, SolveState& ss, cudaStream_t st,
                   bool fast_mr = false);

// Shifted methods: x holds (ns + 1) padded vectors (seed first), the
// shifted parts zero on entry (the reference's assumption).
SolveOut shbicg(const DevCsr& A, const DevCsr& At, const double* b,
                const double* sigma_host, int ns, double* x, double tol,
                int max_iter, SolveState& ss, cudaStream_t st);
// fp32_ps: the per-shift direction vectors p_k (the bulk of the traffic)
// stored in FP32, every update still computed in FP64 (the first stage of
// the mixed-precision shifted solve).
SolveOut shbicgstabl(const DevCsr& A, const double* b, int l,
                     const double* sigma_host, int ns, double* x, double tol,
                     int max_iter, SolveState& ss, cudaStream_t st,
                     bool fp32_ps = false);

// Mixed-precision right-preconditioned BiCGSTAB(l): FP32 matrix values and
// Krylov vectors (A.v32 / M->v32), FP64 dot products, scalars and solution,
// FP64 reliable residual replacement; stops on the FP64 true relative
// residual.  M == nullptr: no preconditioner.
struct MixedOpts {
  double target = 1e-8;   // FP64 true relative residual to reach
  double delta = 1e-3;    // replacement when the recursive residual fell by delta
  int period = 6;         // ... or every `period` outer iterations
  bool fast_mr = true;    // one-pass minimal-residual step
  double shift = 0.0;     // solve (A + shift I) x = b (unpreconditioned)
};
struct MixedOut : SolveOut {
  int replacements = 0;
  double true_res = 0.0;
};
MixedOut bicgstabl_mixed(const DevCsr& A, const DevCsr* M, const double* b,
                         int l, double* x, int max_iter, const MixedOpts& o,
                         SolveState& ss, cudaStream_t st);
// Mixed-precision shifted BiCGSTAB(l): the shifted solve with FP32 shift
// vectors (FP64 seed, x_k and scalars) to the seed tolerance `target`, then
// every system (A + sigma_k I) x_k = b (and the seed) whose FP64 true
// relative residual is above target is polished from its x_k by the
// mixed-precision BiCGSTAB(l) on the shifted operator.  x: (ns + 1) padded
// vectors, seed first, shifted parts zero on entry.  ret: the seed's
// return code of the shifted solve, or NOT_CONVERGED when a polish does not
// reach the target; true_res: the worst FP64 true relative residual over
// the seed and every shift; iters: polishing outer iterations in total.
MixedOut shbicgstabl_mixed(const DevCsr& A, const double* b, int l,
                           const double* sigma_host, int ns, double* x,
                           double target, int max_iter, SolveState& ss,
                           cudaStream_t st);
// Mixed-precision preconditioned CG (A symmetric positive definite, M
// symmetric; nullptr: none) with the same precision split and reliable
// replacement; stops on the FP64 true relative residual.
MixedOut cg_mixed(const DevCsr& A, const DevCsr* M, const double* b, double* x,
                  int max_iter, const MixedOpts& o, SolveState& ss,
                  cudaStream_t st);

}  // namespace bk
