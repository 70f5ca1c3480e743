// Pieces shared by the real (epilogues.cuh) and complex (zepilogues.cuh)
// scalar epilogues: the convergence test and the breakdown exit.
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

// A breakdown (zero pivot, non-positive Cholesky pivot): stop with
// DIVERGENCE.
__device__ __forceinline__ void fail_divergence(const Red& rd) {
  rd.ctl->done = 1;
  rd.ctl->ret = kDivergence;
}

}  // namespace bk
