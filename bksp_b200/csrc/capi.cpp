// extern "C" entry points of libbksp.so: the bksp.h API (host arrays in and
// out, one GPU solve per call) and the bksp_gpu.h extensions.
//
// Every bksp.h solver call: validates its arguments, uploads the CSR
// operator (mirroring a "symmetric" one-triangle matrix for the symmetric-
// only methods; building A^T for BiCG), uploads b and the initial guess,
// runs the device solve, downloads the solution and returns the
// reference's code.  CUDA failures are caught and returned as
// INVALID_PARAMETERS; nothing aborts the caller.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bksp.h"
#include "../../include/bksp_gpu.h"
#include "capi_internal.h"
#include "runtime.h"
#include "solvers.h"
#include "solvers_block.h"

using namespace bk;

namespace bk {

thread_local bksp_gpu_stats* g_stats = nullptr;

bool is_symmetric(const dspmat* A) {
  return A->type && std::strcmp(A->type, "symmetric") == 0;
}

int check_matrix(const dspmat* A) {
  if (!A || !A->row || !A->row_size || !A->nnz || !A->value) return -3;
  if (*A->row_size <= 0) return -3;
  if (*A->nnz > 0 && !A->col) return -3;
  if (A->row[*A->row_size] != *A->nnz) return -3;
  return 0;
}

// Device vector padded to pad64(n), zero beyond n.
double* upload_vec(const double* h, int n, long long extra_cols,
                   cudaStream_t st) {
  const long long np = pad64(n);
  const long long cols = extra_cols > 0 ? extra_cols : 1;
  double* d = dalloc_n<double>(np * cols, st);
  BK_CHECK(cudaMemsetAsync(d, 0, sizeof(double) * np * cols, st));
  if (h) {
    for (long long c = 0; c < cols; ++c)
      BK_CHECK(cudaMemcpyAsync(d + c * np, h + c * n, sizeof(double) * n,
                               cudaMemcpyHostToDevice, st));
  }
  return d;
}

void download_vec(double* h, const double* d, int n, long long cols,
                  cudaStream_t st) {
  const long long np = pad64(n);
  for (long long c = 0; c < cols; ++c)
    BK_CHECK(cudaMemcpyAsync(h + c * n, d + c * np, sizeof(double) * n,
                             cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
}

// Upload the operator a method sees: the mirrored full matrix when
// `expand` (symmetric-only methods on a "symmetric" matrix), otherwise the
// stored entries as they are (the reference's dcsrgemm0 ignores `type`).
void upload_operator(const dspmat* A, bool expand, bool want_fp32, DevCsr& out,
                     cudaStream_t st) {
  const int n = *A->row_size;
  if (expand) {
    HostCsr h = expand_symmetric(n, A->row, A->col, A->value);
    upload_csr(n, h.rowptr.data(), h.col.data(), h.val.data(), want_fp32, out,
               st);
  } else {
    // Column indices are checked by the structure scan on the GPU.
    upload_csr(n, A->row, A->col, A->value, want_fp32, out, st);
  }
}

Timer::Timer(cudaStream_t s) : st(s) {
  t0 = std::chrono::steady_clock::now();
  BK_CHECK(cudaEventCreate(&e0));
  BK_CHECK(cudaEventCreate(&e1));
}
Timer::~Timer() {
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}
void Timer::begin_solve() { BK_CHECK(cudaEventRecord(e0, st)); }
void Timer::end_solve() { BK_CHECK(cudaEventRecord(e1, st)); }
void Timer::report(int ret, const SolveState* ss, int hist_len) {
  if (!g_stats) return;
  bksp_gpu_stats* s = g_stats;
  s->ret = ret;
  cudaEventSynchronize(e1);
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) s->solve_ms = ms;
  s->total_ms = std::chrono::duration<double, std::milli>(
                    std::chrono::steady_clock::now() - t0).count();
  s->hist_len = hist_len;
  if (ss && ss->hist && s->hist && s->hist_cap > 0) {
    const int m = std::min(hist_len, std::min(s->hist_cap, ss->hist_cap));
    if (m > 0)
      cudaMemcpy(s->hist, ss->hist, sizeof(double) * m, cudaMemcpyDeviceToHost);
  }
}

int hist_cap_for(int max_iter) {
  if (!g_stats || g_stats->hist_cap <= 0) return 0;
  return std::min(g_stats->hist_cap, std::max(max_iter, 1) + 2);
}

}  // namespace bk

namespace {

enum class Method { CG, CR, BICG, BICGSTAB, BICGSTABL };

int solve_single(Method m, dspmat* A, double* b, int l, double tol,
                 int max_iter, double* x) {
  if (check_matrix(A) != 0 || !b || !x) return INVALID_PARAMETERS;
  const bool sym_only = (m == Method::CG || m == Method::CR);
  if (sym_only && !is_symmetric(A)) return INVALID_MATRIX_TYPE;
  if (m == Method::BICGSTABL && (l < 1 || l > kBlMaxL)) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    const int n = *A->row_size;
    DevCsr dA, dAt;
    upload_operator(A, sym_only, false, dA, st);
    if (m == Method::BICG) {
      HostCsr t = transpose(n, A->row, A->col, A->value);
      upload_csr(n, t.rowptr.data(), t.col.data(), t.val.data(), false, dAt, st);
    }
    double* db = upload_vec(b, n, 1, st);
    double* dx = upload_vec(x, n, 1, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    SolveOut o;
    switch (m) {
      case Method::CG: o = bk::cg(dA, db, dx, tol, max_iter, ss, st); break;
      case Method::CR: o = bk::cr(dA, db, dx, tol, max_iter, ss, st); break;
      case Method::BICG: o = bk::bicg(dA, dAt, db, dx, tol, max_iter, ss, st); break;
      case Method::BICGSTAB: o = bk::bicgstab(dA, db, dx, tol, max_iter, ss, st); break;
      case Method::BICGSTABL: o = bk::bicgstabl(dA, db, l, dx, tol, max_iter, ss, st); break;
    }
    tm.end_solve();
    download_vec(x, dx, n, 1, st);
    tm.report(o.ret, &ss, o.iters);
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    dA.release(st);
    dAt.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

}  // namespace

extern "C" {

void bksp_gpu_record(bksp_gpu_stats* s) { bk::g_stats = s; }

const char* bksp_gpu_version(void) { return "bksp-b200 0.1 (sm_100a)"; }

int bksp_dcg(dspmat* A, double* b, double tol, int max_iter, double* x) {
  return solve_single(Method::CG, A, b, 0, tol, max_iter, x);
}
int dcr(dspmat* A, double* b, double tol, int max_iter, double* x) {
  return solve_single(Method::CR, A, b, 0, tol, max_iter, x);
}
int dbicg(dspmat* A, double* b, double tol, int max_iter, double* x) {
  return solve_single(Method::BICG, A, b, 0, tol, max_iter, x);
}
int dbicgstab(dspmat* A, double* b, double tol, int max_iter, double* x) {
  return solve_single(Method::BICGSTAB, A, b, 0, tol, max_iter, x);
}
int dbicgstabl(dspmat* A, double* b, int l, double tol, int max_iter,
               double* x) {
  return solve_single(Method::BICGSTABL, A, b, l, tol, max_iter, x);
}

}  // extern "C"

// --------------------------------------------------------- block methods

namespace {

enum class BMethod { CG, BICGSTAB, BICGSTABL };

int solve_block(BMethod m, dspmat* A, dmat* B, int l, double tol, int max_iter,
                dmat* X) {
  if (check_matrix(A) != 0 || !B || !X || !B->value || !X->value)
    return INVALID_PARAMETERS;
  if (m == BMethod::CG && !is_symmetric(A)) return INVALID_MATRIX_TYPE;
  const int n = *A->row_size, s = B->col_size;
  if (B->row_size != n || X->row_size != n || X->col_size != s || s < 1 ||
      s > kBlockMaxS)
    return INVALID_PARAMETERS;
  if (m == BMethod::BICGSTABL && (l < 1 || l > kBlMaxL)) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    DevCsr dA;
    upload_operator(A, m == BMethod::CG, false, dA, st);
    const long long np = pad64(n);
    double* tmp = dalloc_n<double>((long long)n * s, st);
    double* dB = dalloc_n<double>(np * s, st);
    double* dX = dalloc_n<double>(np * s, st);
    BK_CHECK(cudaMemsetAsync(dB, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemsetAsync(dX, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemcpyAsync(tmp, B->value, sizeof(double) * n * s,
                             cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dB, n, s, st);
    BK_CHECK(cudaMemcpyAsync(tmp, X->value, sizeof(double) * n * s,
                             cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dX, n, s, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    SolveOut o;
    double true_res = 0.0;
    {
      BlockCtx bc(n, s, ss, st);
      tm.begin_solve();
      switch (m) {
        case BMethod::CG: o = bk::blcg<double>(bc, dA, dB, dX, tol, max_iter); break;
        case BMethod::BICGSTAB:
          o = bk::blbicgstab<double>(bc, dA, dB, dX, tol, max_iter);
          break;
        case BMethod::BICGSTABL:
          o = bk::blbicgstabl<double>(bc, dA, dB, dX, l, tol, max_iter, &true_res);
          break;
      }
      tm.end_solve();
      bc.release();
    }
    launch_rm2cm(dX, tmp, n, s, st);
    BK_CHECK(cudaMemcpyAsync(X->value, tmp, sizeof(double) * n * s,
                             cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    if (m == BMethod::BICGSTABL) {
      // The reference prints this summary on every exit
      // (src/blbicgstabl.c:220-224).
      const double err = ss.get_scalar(kErr, st);
      const int it = o.ret >= 0 ? o.ret : max_iter;
      std::printf("Block BiCGSTAB(%d) has converged at:\n"
                  "        The number of iteration ... %d\n"
                  "        Frobenius norm of the relative residual ... %e\n"
                  "        Frobenius norm of the true residual ... %e\n",
                  l, it, err, true_res);
      std::fflush(stdout);
    }
    tm.report(o.ret, &ss, o.iters);
    if (g_stats) g_stats->true_res = true_res;
    ss.release(st);
    dfree(tmp, st);
    dfree(dB, st);
    dfree(dX, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

// Host arrays in, the mixed-precision block solve, host arrays out.
int solve_block_mixed(BMethod m, dspmat* A, dmat* B, const bksp_gpu_mixed_opts* o,
                      dmat* X) {
  if (check_matrix(A) != 0 || !B || !X || !B->value || !X->value || !o)
    return INVALID_PARAMETERS;
  if (m == BMethod::CG && !is_symmetric(A)) return INVALID_MATRIX_TYPE;
  const int n = *A->row_size, s = B->col_size;
  if (B->row_size != n || X->row_size != n || X->col_size != s || s < 1 ||
      s > kBlockMaxS)
    return INVALID_PARAMETERS;
  const int l = o->l;
  if (m == BMethod::BICGSTABL && (l < 1 || l > kBlMaxL)) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    DevCsr dA;
    upload_operator(A, m == BMethod::CG, true, dA, st);
    const long long np = pad64(n);
    double* tmp = dalloc_n<double>((long long)n * s, st);
    double* dB = dalloc_n<double>(np * s, st);
    double* dX = dalloc_n<double>(np * s, st);
    BK_CHECK(cudaMemsetAsync(dB, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemsetAsync(dX, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemcpyAsync(tmp, B->value, sizeof(double) * n * s,
                             cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dB, n, s, st);
    BK_CHECK(cudaMemcpyAsync(tmp, X->value, sizeof(double) * n * s,
                             cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dX, n, s, st);
    const int max_iter = o->max_iter > 0 ? o->max_iter : 10000;
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    const BlockMixedOut r = block_mixed(m == BMethod::CG ? 0 : 2, dA, dB, dX, n, s, l,
                                        o->target > 0 ? o->target : 1e-8, max_iter,
                                        o->delta > 0 ? o->delta : 1e-4, ss, st);
    tm.end_solve();
    launch_rm2cm(dX, tmp, n, s, st);
    BK_CHECK(cudaMemcpyAsync(X->value, tmp, sizeof(double) * n * s,
                             cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    tm.report(r.ret, nullptr, r.inner_iters);
    if (g_stats) {
      g_stats->true_res = r.true_res;
      g_stats->inner_iters = r.inner_iters;
      g_stats->sweeps = r.sweeps;
    }
    ss.release(st);
    dfree(tmp, st);
    dfree(dB, st);
    dfree(dX, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return r.ret;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

}  // namespace

extern "C" {

int bksp_dblcg_mixed(dspmat* A, dmat* B, const bksp_gpu_mixed_opts* opts, dmat* X) {
  return solve_block_mixed(BMethod::CG, A, B, opts, X);
}

int bksp_dblbicgstabl_mixed(dspmat* A, dmat* B, const bksp_gpu_mixed_opts* opts,
                            dmat* X) {
  return solve_block_mixed(BMethod::BICGSTABL, A, B, opts, X);
}

int dblcg(dspmat* A, dmat* B, double tol, int max_iter, dmat* X) {
  return solve_block(BMethod::CG, A, B, 0, tol, max_iter, X);
}

int dblbicgstab(dspmat* A, dmat* B, double tol, int max_iter, dmat* X) {
  return solve_block(BMethod::BICGSTAB, A, B, 0, tol, max_iter, X);
}

int dblbicgstabl(dspmat* A, dmat* B, int l, double tol, int max_iter, dmat* X) {
  return solve_block(BMethod::BICGSTABL, A, B, l, tol, max_iter, X);
}

// Thin QR on the GPU (reference src/myqr.c:4-39): mat (m-by-n,
// column-major) becomes Q, r (n-by-n, column-major) receives the upper-
// triangular R with non-negative diagonal.  Returns 0, or
// INVALID_PARAMETERS (bad sizes, n > 16, rank-deficient input, CUDA error).
int myqr(int m, int n, double* mat, double* r) {
  if (m < 1 || n < 1 || n > kBlockMaxS || m < n || !mat || !r)
    return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    const long long np = pad64(m);
    double* tmp = dalloc_n<double>((long long)m * n, st);
    double* V = dalloc_n<double>(np * n, st);
    BK_CHECK(cudaMemsetAsync(V, 0, sizeof(double) * np * n, st));
    BK_CHECK(cudaMemcpyAsync(tmp, mat, sizeof(double) * m * n,
                             cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, V, m, n, st);
    SolveState ss;
    ss.create(0, st);
    int rc = 0;
    {
      BlockCtx bc(m, n, ss, st);
      bk::thin_qr(bc, V);
      const CtlH c = ss.read(st);
      if (c.done) rc = INVALID_PARAMETERS;   // Cholesky breakdown
    }
    launch_rm2cm(V, tmp, m, n, st);
    BK_CHECK(cudaMemcpyAsync(mat, tmp, sizeof(double) * m * n,
                             cudaMemcpyDeviceToHost, st));
    std::vector<double> R((size_t)n * n);
    BK_CHECK(cudaMemcpyAsync(R.data(), ss.S + kBkR, sizeof(double) * n * n,
                             cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i)        // column-major, zero below the diagonal
      for (int j = 0; j < n; ++j) r[i * n + j] = j <= i ? R[(size_t)j * n + i] : 0.0;
    ss.release(st);
    dfree(tmp, st);
    dfree(V, st);
    BK_CHECK(cudaStreamSynchronize(st));
    return rc;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

}  // extern "C"

// ------------------------------------------------------- shifted methods

namespace {

// mixed: the mixed-precision shifted BiCGSTAB(l) (tol = FP64 target).
int solve_shifted(bool stab, dspmat* A, double* b, int l, double* sigma,
                  int ns, double tol, int max_iter, double* x, bool mixed = false) {
  if (check_matrix(A) != 0 || !b || !x || ns < 0 || ns > kMaxShifts ||
      (ns > 0 && !sigma))
    return INVALID_PARAMETERS;
  if (stab && (l < 1 || l > kBlMaxL)) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    const int n = *A->row_size;
    DevCsr dA, dAt;
    upload_operator(A, false, mixed, dA, st);
    if (!stab) {
      HostCsr t = transpose(n, A->row, A->col, A->value);
      upload_csr(n, t.rowptr.data(), t.col.data(), t.val.data(), false, dAt, st);
    }
    double* db = upload_vec(b, n, 1, st);
    double* dx = upload_vec(x, n, (long long)ns + 1, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    SolveOut o;
    MixedOut mo;
    if (mixed) {
      mo = bk::shbicgstabl_mixed(dA, db, l, sigma, ns, dx, tol, max_iter, ss, st);
      o = mo;
    } else {
      o = stab ? bk::shbicgstabl(dA, db, l, sigma, ns, dx, tol, max_iter, ss, st)
               : bk::shbicg(dA, dAt, db, sigma, ns, dx, tol, max_iter, ss, st);
    }
    tm.end_solve();
    download_vec(x, dx, n, (long long)ns + 1, st);
    tm.report(o.ret, mixed ? nullptr : &ss, o.iters);
    if (mixed && g_stats) {
      g_stats->true_res = mo.true_res;
      g_stats->inner_iters = mo.iters;
      g_stats->sweeps = mo.replacements;
    }
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    dA.release(st);
    dAt.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

}  // namespace

extern "C" {

int dshbicg(dspmat* A, double* b, double* sigma, int sigma_size, double tol,
            int max_iter, double* x) {
  return solve_shifted(false, A, b, 0, sigma, sigma_size, tol, max_iter, x);
}

int dshbicgstabl(dspmat* A, double* b, int l, double* sigma, int sigma_size,
                 double tol, int max_iter, double* x) {
  return solve_shifted(true, A, b, l, sigma, sigma_size, tol, max_iter, x);
}

int bksp_dshbicgstabl_mixed(dspmat* A, double* b, double* sigma, int sigma_size,
                            const bksp_gpu_mixed_opts* o, double* x) {
  if (!o) return INVALID_PARAMETERS;
  return solve_shifted(true, A, b, o->l, sigma, sigma_size,
                       o->target > 0 ? o->target : 1e-8,
                       o->max_iter > 0 ? o->max_iter : 10000, x, true);
}

}  // extern "C"

extern "C" {

// ---------------------------------------------------------- dense helpers
// Host-side containers (reference src/util.c:5-67); no computation.

dmat* dmat_create(int m, int n) {
  if (m < 0 || n < 0) return nullptr;
  dmat* d = static_cast<dmat*>(std::malloc(sizeof(dmat)));
  if (!d) return nullptr;
  d->row_size = m;
  d->col_size = n;
  d->value = static_cast<double*>(std::calloc((size_t)m * n > 0 ? (size_t)m * n : 1,
                                              sizeof(double)));
  return d;
}

int darray2dmat(double* arr, int row_size, int col_size, dmat* mat) {
  mat->row_size = row_size;
  mat->col_size = col_size;
  mat->value = arr;
  return 0;
}

int dmat_free(dmat* mat) {
  if (!mat) return 0;
  std::free(mat->value);
  std::free(mat);
  return 0;
}

int dvec2mat(double* x, int m, dmat* mat) {
  const int l = mat->row_size, n = mat->col_size;
  for (int i = 0; i < l; ++i) mat->value[i * n + m] = x[i];
  return 0;
}

}  // extern "C"

// ------------------------------------------------------- device utilities

extern "C" int bksp_gpu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// y = A x (trans 'n') or y = A^T x (trans 't') with the stored entries of A
// (reference mkl_cspblas_dcsrgemv -> dcsrgemm0, include/bksp_internal.h:45-52,
// src/matvec.c:11-53), or the mirrored operator of a one-triangle matrix
// (trans 's', reference mkl_cspblas_dcsrsymv -> dcsrsymm0, :35-43,
// src/matvec.c:100-127).  Host arrays; one GPU product.
extern "C" int bksp_gpu_dcsrmv(dspmat* A, char trans, const double* x,
                               double* y) {
  if (check_matrix(A) != 0 || !x || !y) return INVALID_PARAMETERS;
  if (trans != 'n' && trans != 't' && trans != 's') return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    const int n = *A->row_size;
    DevCsr dA;
    if (trans == 't') {
      HostCsr t = transpose(n, A->row, A->col, A->value);
      upload_csr(n, t.rowptr.data(), t.col.data(), t.val.data(), false, dA, st);
    } else {
      upload_operator(A, trans == 's', false, dA, st);
    }
    double* dx = upload_vec(x, n, 1, st);
    double* dy = upload_vec(nullptr, n, 1, st);
    SolveState ss;
    ss.create(0, st);
    ss.start(0, 1, 0.0, st);
    spmv(dA, spmv_io<double>(dx, dy), ss.red(kD, E_NONE), st);
    BK_CHECK(cudaGetLastError());
    download_vec(y, dy, n, 1, st);
    ss.release(st);
    dfree(dx, st);
    dfree(dy, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}

// C = beta C + alpha A B on the GPU with host arrays (reference
// src/matvec.c:130-172 dcsrgemm1 / 219-247 dcsrsymm1, via mkl_dcsrmm),
// B and C column-major n x s: the product runs on row-major device blocks
// (the block methods' layout) with the SpMM kernel the block methods use --
// the diagonal-form kernel for stencil operators, the CSR kernel otherwise.
extern "C" int bksp_gpu_dcsrmm(dspmat* A, char trans, int s, double alpha,
                               const double* B, double beta, double* C) {
  if (check_matrix(A) != 0 || !B || !C) return INVALID_PARAMETERS;
  if ((trans != 'n' && trans != 's') || s < 1 || s > kBlockMaxS) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    const int n = *A->row_size;
    DevCsr dA;
    upload_operator(A, trans == 's', false, dA, st);
    const long long np = pad64(n);
    std::vector<double> cb((size_t)n * s);
    for (size_t q = 0; q < cb.size(); ++q) cb[q] = beta * C[q];
    double* tmp = dalloc_n<double>((long long)n * s, st);
    double* dB = dalloc_n<double>(np * s, st);
    double* dC = dalloc_n<double>(np * s, st);
    BK_CHECK(cudaMemsetAsync(dB, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemsetAsync(dC, 0, sizeof(double) * np * s, st));
    BK_CHECK(cudaMemcpyAsync(tmp, B, sizeof(double) * n * s, cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dB, n, s, st);
    BK_CHECK(cudaMemcpyAsync(tmp, cb.data(), sizeof(double) * n * s, cudaMemcpyHostToDevice, st));
    launch_cm2rm(tmp, dC, n, s, st);
    SolveState ss;
    ss.create(0, st);
    ss.start(0, 1, 0.0, st);
    SpmmH a;
    std::memset(&a, 0, sizeof(a));
    a.X = dB;
    a.Y = dC;
    a.C = dC;
    a.alpha = alpha;
    a.mode = 1;
    a.s = s;
    spmm_autotune(dA.h64(), s, 0, st);
    launch_spmm(dA.h64(), a, ss.red(kD, E_NONE), st);
    BK_CHECK(cudaGetLastError());
    launch_rm2cm(dC, tmp, n, s, st);
    BK_CHECK(cudaMemcpyAsync(C, tmp, sizeof(double) * n * s, cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    ss.release(st);
    dfree(tmp, st);
    dfree(dB, st);
    dfree(dC, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
}
