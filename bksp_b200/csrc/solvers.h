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
SolveOut bicgstabl(const DevCsr& A, const double* b, int l, double* x,
                   double tol, int max_iter, SolveState& ss, cudaStream_t st);

}  // namespace bk
