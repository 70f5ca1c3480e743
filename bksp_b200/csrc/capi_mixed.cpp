// bksp_gpu.h mixed-precision entry points (device and host arrays) and the
// Jacobi preconditioner.  The learned preconditioner lives in spai.cpp.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "capi_internal.h"
#include "solvers.h"
#include "spai.h"

using namespace bk;

namespace bk {

// M = diag(A)^-1 (first stored diagonal entry of each row, from the
// operator's structure scan) as a one-entry-per-row CSR.
void build_jacobi(bksp_gpu_matrix* m, cudaStream_t st) {
  if (m->has_jacobi || !m->diag_ok) return;
  const int n = m->A.n;
  std::vector<int> rp(n + 1), col(n);
  std::vector<double> v(n);
  BK_CHECK(cudaMemcpyAsync(v.data(), m->A.ddiag, sizeof(double) * n,
                           cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i) {
    rp[i] = i;
    col[i] = i;
    v[i] = 1.0 / v[i];
  }
  rp[n] = n;
  upload_csr(n, rp.data(), col.data(), v.data(), true, m->jacobi, st);
  m->has_jacobi = true;
}

}  // namespace bk

namespace {

int fail(const std::exception& e) {
  if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
  cudaGetLastError();
  return INVALID_PARAMETERS;
}

enum MixedMethod { kMixedBicgstabl = 0, kMixedCg = 1 };

MixedOut run_mixed(bksp_gpu_matrix* m, int method, const double* db, double* dx,
                   const bksp_gpu_mixed_opts* o, int precond, SolveState& ss,
                   cudaStream_t st, float* mvals_scratch) {
  MixedOpts mo;
  mo.target = o->target > 0 ? o->target : 1e-8;
  if (o->delta > 0) mo.delta = o->delta;
  if (o->period > 0) mo.period = o->period;
  const DevCsr* M = nullptr;
  DevCsr view;
  if (precond == BKSP_GPU_PRECOND_JACOBI) {
    build_jacobi(m, st);
    if (!m->has_jacobi) throw CudaError("Jacobi: zero diagonal entry");
    M = &m->jacobi;
  } else if (precond == BKSP_GPU_PRECOND_LEARNED) {
    if (m->spai.ok) {
      // CG needs a symmetric preconditioner: (M + M^T) / 2.
      view = spai_apply(o->model, m, mvals_scratch, st, method == kMixedCg);
      M = &view;
    } else if (m->diag_ok) {   // not stencil-like: Jacobi instead
      build_jacobi(m, st);
      M = &m->jacobi;
    }
  }
  const int max_iter = o->max_iter > 0 ? o->max_iter : 10000;
  if (method == kMixedCg) return cg_mixed(m->A, M, db, dx, max_iter, mo, ss, st);
  return bicgstabl_mixed(m->A, M, db, o->l, dx, max_iter, mo, ss, st);
}

int solve_mixed_impl(bksp_gpu_matrix* m, int method, const double* b, double* x,
                     const bksp_gpu_mixed_opts* o, void* stream,
                     bksp_gpu_stats* stats);

}  // namespace

extern "C" {

int bksp_gpu_solve_mixed(bksp_gpu_matrix* m, const double* b, double* x,
                         const bksp_gpu_mixed_opts* o, void* stream,
                         bksp_gpu_stats* stats) {
  return solve_mixed_impl(m, kMixedBicgstabl, b, x, o, stream, stats);
}

int bksp_gpu_cg_mixed(bksp_gpu_matrix* m, const double* b, double* x,
                      const bksp_gpu_mixed_opts* o, void* stream,
                      bksp_gpu_stats* stats) {
  return solve_mixed_impl(m, kMixedCg, b, x, o, stream, stats);
}

}  // extern "C"

namespace {

int solve_mixed_impl(bksp_gpu_matrix* m, int method, const double* b, double* x,
                     const bksp_gpu_mixed_opts* o, void* stream,
                     bksp_gpu_stats* stats) {
  if (!m || !b || !x || !o) return INVALID_PARAMETERS;
  if (!m->A.v32) return INVALID_PARAMETERS;
  if (method == kMixedBicgstabl && (o->l < 1 || o->l > kBlMaxL)) return INVALID_PARAMETERS;
  if (o->precond < 0 || o->precond > 2) return INVALID_PARAMETERS;
  if (o->precond == BKSP_GPU_PRECOND_LEARNED && !o->model) return INVALID_PARAMETERS;
  bksp_gpu_stats* saved = g_stats;
  g_stats = stats;
  int ret = INVALID_PARAMETERS;
  try {
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : Ctx::get().st;
    Timer tm(st);
    const long long l0 = launch_count(), y0 = byte_count();
    const int n = m->A.n;
    const long long np = pad64(n);
    double* db = dalloc_n<double>(np, st);
    double* dx = dalloc_n<double>(np, st);
    double* x0 = dalloc_n<double>(np, st);
    float* mv = o->precond == BKSP_GPU_PRECOND_LEARNED
                    ? dalloc_n<float>(spai_scratch_floats(m, method == kMixedCg), st)
                    : nullptr;
    BK_CHECK(cudaMemsetAsync(db, 0, sizeof(double) * np, st));
    BK_CHECK(cudaMemsetAsync(dx, 0, sizeof(double) * np, st));
    tm.begin_solve();
    BK_CHECK(cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    BK_CHECK(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    BK_CHECK(cudaMemcpyAsync(x0, dx, sizeof(double) * np, cudaMemcpyDeviceToDevice, st));
    SolveState ss;
    ss.create(hist_cap_for(o->max_iter > 0 ? o->max_iter : 10000), st);
    MixedOut r = run_mixed(m, method, db, dx, o, o->precond, ss, st, mv);
    int sweeps = 1, inner = r.iters, reps = r.replacements;
    if (r.ret < 0 && o->fallback && o->precond == BKSP_GPU_PRECOND_LEARNED) {
      // Stagnation / breakdown of the learned preconditioner: plain Jacobi
      // from the original initial guess.
      BK_CHECK(cudaMemcpyAsync(dx, x0, sizeof(double) * np, cudaMemcpyDeviceToDevice, st));
      r = run_mixed(m, method, db, dx, o, m->diag_ok ? BKSP_GPU_PRECOND_JACOBI
                                                     : BKSP_GPU_PRECOND_NONE,
                    ss, st, mv);
      sweeps = 2;
      inner += r.iters;
      reps += r.replacements;
    }
    BK_CHECK(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    tm.end_solve();
    BK_CHECK(cudaStreamSynchronize(st));
    tm.report(r.ret, &ss, r.iters);
    if (stats) {
      stats->launches = launch_count() - l0;
      stats->alg_bytes = byte_count() - y0;
      stats->true_res = r.true_res;
      stats->inner_iters = inner;
      stats->sweeps = sweeps * 1000 + reps;   // sweeps*1000 + replacements
    }
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    dfree(x0, st);
    dfree(mv, st);
    BK_CHECK(cudaStreamSynchronize(st));
    ret = r.ret;
  } catch (const std::exception& e) {
    ret = fail(e);
  }
  g_stats = saved;
  return ret;
}

// Host arrays in the bksp.h style: upload A (flags), b, x; solve; download.
int host_mixed(dspmat* A, int flags, int method, double* b,
               const bksp_gpu_mixed_opts* o, double* x) {
  bksp_gpu_matrix* m = nullptr;
  int rc = bksp_gpu_matrix_create(A, flags, &m);
  if (rc != 0) return rc;
  int ret = INVALID_PARAMETERS;
  try {
    cudaStream_t st = Ctx::get().st;
    const int n = *A->row_size;
    double* db = dalloc_n<double>(n, st);
    double* dx = dalloc_n<double>(n, st);
    BK_CHECK(cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    BK_CHECK(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    ret = solve_mixed_impl(m, method, db, dx, o, st, g_stats);
    BK_CHECK(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    dfree(db, st);
    dfree(dx, st);
  } catch (const std::exception& e) {
    ret = fail(e);
  }
  bksp_gpu_matrix_destroy(m);
  return ret;
}

}  // namespace

extern "C" {

int bksp_dbicgstabl_mixed(dspmat* A, double* b, const bksp_gpu_mixed_opts* o,
                          double* x) {
  if (check_matrix(A) != 0 || !b || !x || !o) return INVALID_PARAMETERS;
  return host_mixed(A, BKSP_GPU_FP32, kMixedBicgstabl, b, o, x);
}

int bksp_dcg_mixed(dspmat* A, double* b, const bksp_gpu_mixed_opts* o, double* x) {
  if (check_matrix(A) != 0 || !b || !x || !o) return INVALID_PARAMETERS;
  // As bksp_dcg: a "symmetric" matrix holding one triangle (src/cg.c:9-11).
  if (!is_symmetric(A)) return INVALID_MATRIX_TYPE;
  return host_mixed(A, BKSP_GPU_FP32 | BKSP_GPU_MIRROR, kMixedCg, b, o, x);
}

}  // extern "C"
