// Block methods (multiple right-hand sides) and the thin QR.
#pragma once

#include <cmath>
#include <vector>

#include "solvers.h"

namespace bk {

constexpr int kBlockMaxS = 16;   // widest block (right-hand sides)

// Per-solve context of a block method: sizes, reduction scratch sized for
// s-by-s Gram products, and the solve's device blocks.
struct BlockCtx {
  int n, s;
  long long np;
  SolveState& ss;
  cudaStream_t st;
  double* bpart = nullptr;
  std::vector<double*> owned;
  BlockCtx(int n, int s, SolveState& ss, cudaStream_t st);
  ~BlockCtx();
  RedH red(short out, short epi, short a0 = 0, short a1 = 0) const;
  double* block(int count);     // zeroed np x s blocks (freed by release)
  void release();
  void start(int max_iter, double tol);
  void qr_tail(double* V, short post, double* copy, cudaStream_t s);
};

// B, X: row-major np x s device blocks (X in/out).
SolveOut blcg(BlockCtx& bc, const DevCsr& A, const double* B, double* X,
              double tol, int max_iter);
SolveOut blbicgstab(BlockCtx& bc, const DevCsr& A, const double* B, double* X,
                    double tol, int max_iter);
SolveOut blbicgstabl(BlockCtx& bc, const DevCsr& A, const double* B,
                     double* X, int l, double tol, int max_iter,
                     double* true_res_out);
// Thin QR of the row-major np x s block V in place; R (row-major, upper,
// positive diagonal) is left in the scalar slots at kBkR.
void thin_qr(BlockCtx& bc, double* V);

}  // namespace bk
