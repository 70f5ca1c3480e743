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
  double unit = 1.1102230246251565e-16;   // unit roundoff of the blocks (QR shift)
  std::vector<void*> owned;
  BlockCtx(int n, int s, SolveState& ss, cudaStream_t st);
  ~BlockCtx();
  RedH red(short out, short epi, short a0 = 0, short a1 = 0) const;
  // `count` zeroed np x s blocks of T (freed by release).
  template <typename T>
  T* block(int count) { return static_cast<T*>(block_bytes(count, sizeof(T))); }
  void* block_bytes(int count, size_t esz);
  void release();
  void start(int max_iter, double tol);
  template <typename T>
  struct Same { using type = T; };
  template <typename T>
  void qr_tail(T* V, short post, typename Same<T>::type* copy, cudaStream_t s);
};

// B, X: row-major np x s device blocks (X in/out).  T = double: the
// reference-parity methods; T = float: FP32 blocks and operator values
// (A.v32), FP64 Gram products, dots and s-by-s algebra -- the inner solves
// of the mixed-precision block methods.
template <typename T>
SolveOut blcg(BlockCtx& bc, const DevCsr& A, const T* B, T* X, double tol,
              int max_iter);
template <typename T>
SolveOut blbicgstab(BlockCtx& bc, const DevCsr& A, const T* B, T* X, double tol,
                    int max_iter);
template <typename T>
SolveOut blbicgstabl(BlockCtx& bc, const DevCsr& A, const T* B, T* X, int l,
                     double tol, int max_iter, double* true_res_out);
// Mixed-precision block solve (method 0 Block CG, 2 Block BiCGSTAB(l)): FP64
// iterative refinement around FP32 inner solves of the method; B, X FP64
// row-major np x s (X in/out); A needs FP32 values.  ret: total inner
// iterations - 1 at convergence (every column at target), or NOT_CONVERGED
// / DIVERGENCE; true_res = the worst column's FP64 true relative residual.
struct BlockMixedOut {
  int ret = kNotConverged;
  int sweeps = 0;
  int fp64_sweeps = 0;   // sweeps whose FP32 inner solve broke down
  int inner_iters = 0;
  double true_res = 0.0;
};
BlockMixedOut block_mixed(int method, const DevCsr& A, const double* B,
                          double* X, int n, int s, int l, double target,
                          int max_iter, double inner_tol, SolveState& ss,
                          cudaStream_t st);
// Thin QR of the row-major np x s block V in place; R (row-major, upper,
// positive diagonal) is left in the scalar slots at kBkR.
void thin_qr(BlockCtx& bc, double* V);

}  // namespace bk
