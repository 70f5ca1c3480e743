// bksp_gpu.h device-resident entry points: operator handles, solves on
// device vectors, single SpMV launches and FP64 true residuals.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>

#include "capi_internal.h"
#include "solvers.h"

using namespace bk;

namespace {

cudaStream_t pick(void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : Ctx::get().st;
}

int fail(const std::exception& e) {
  if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
  cudaGetLastError();
  return INVALID_PARAMETERS;
}

}  // namespace

namespace bk {

// FP64 true residual ||b - A x|| / ||b|| of padded device vectors.
double true_residual_dev(const DevCsr& A, const double* b, const double* x,
                         cudaStream_t st) {
  const long long np = pad64(A.n);
  double* r = dalloc_n<double>(np, st);
  BK_CHECK(cudaMemsetAsync(r, 0, sizeof(double) * np, st));
  SolveState ss;
  ss.create(0, st);
  ss.start(0, 1, 0.0, st);
  SpmvH<double> io = spmv_io<double>(x, r);
  io.b = b;
  io.mode = 1;
  io.nd = 2;
  io.dot[0][0] = 0; io.dot[0][1] = 0;   // (r, r)
  io.dot[1][0] = 1; io.dot[1][1] = 1;   // (b, b)
  spmv(A, io, ss.red(kD, E_NONE), st);
  const double rr = ss.get_scalar(kD, st), bb = ss.get_scalar(kD + 1, st);
  ss.release(st);
  dfree(r, st);
  return std::sqrt(rr) / std::sqrt(bb);
}

}  // namespace bk

extern "C" {

int bksp_gpu_matrix_create(dspmat* A, int flags, bksp_gpu_matrix** out) {
  if (!out || check_matrix(A) != 0) return INVALID_PARAMETERS;
  *out = nullptr;
  bksp_gpu_matrix* m = new (std::nothrow) bksp_gpu_matrix();
  if (!m) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    m->flags = flags;
    m->device = cx.device;
    const int n = *A->row_size;
    const bool f32 = (flags & BKSP_GPU_FP32) != 0;
    if (flags & BKSP_GPU_MIRROR) {
      HostCsr h = expand_symmetric(n, A->row, A->col, A->value);
      upload_csr(n, h.rowptr.data(), h.col.data(), h.val.data(), f32, m->A, st);
    } else {
      upload_operator(A, false, f32, m->A, st);
    }
    if (f32) spai_build_slots(m->A, m->spai, st);
    m->diag_ok = !(m->A.scan.flags & kScanNoDiag);
    if (flags & BKSP_GPU_TRANSPOSE) {
      HostCsr t = transpose(n, A->row, A->col, A->value);
      upload_csr(n, t.rowptr.data(), t.col.data(), t.val.data(),
                 (flags & BKSP_GPU_FP32) != 0, m->At, st);
      m->has_t = true;
    }
    BK_CHECK(cudaStreamSynchronize(st));
    *out = m;
    return 0;
  } catch (const std::exception& e) {
    cudaStream_t st = Ctx::get().st;
    cudaStreamSynchronize(st);
    m->A.release(st);
    m->At.release(st);
    m->spai.release(st);
    cudaStreamSynchronize(st);
    delete m;
    return fail(e);
  }
}

int bksp_gpu_matrix_destroy(bksp_gpu_matrix* m) {
  if (!m) return 0;
  cudaStream_t st = Ctx::get().st;
  m->A.release(st);
  m->At.release(st);
  m->jacobi.release(st);
  m->spai.release(st);
  cudaStreamSynchronize(st);
  delete m;
  return 0;
}

int bksp_gpu_matrix_variant(bksp_gpu_matrix* m, int variant) {
  if (!m) return INVALID_PARAMETERS;
  if (variant > 8) return INVALID_PARAMETERS;
  if (variant >= 0) {
    m->A.variant = variant;
    m->At.variant = variant;
  }
  return m->A.variant;
}

int bksp_gpu_matrix_diagonals(const bksp_gpu_matrix* m, int* offsets) {
  if (!m) return INVALID_PARAMETERS;
  if (offsets)
    for (int d = 0; d < m->A.ndia; ++d) offsets[d] = m->A.doff[d];
  return m->A.ndia;
}

int bksp_gpu_matrix_info(const bksp_gpu_matrix* m, int* n, int* nnz) {
  if (!m) return INVALID_PARAMETERS;
  if (n) *n = m->A.n;
  if (nnz) *nnz = m->A.nnz;
  return 0;
}

int bksp_gpu_solve(bksp_gpu_matrix* m, int method, int l, const double* b,
                   double* x, double tol, int max_iter, void* stream,
                   bksp_gpu_stats* stats) {
  if (!m || !b || !x) return INVALID_PARAMETERS;
  if (method == BKSP_GPU_BICG && !m->has_t) return INVALID_PARAMETERS;
  if ((method == BKSP_GPU_BICGSTABL || method == BKSP_GPU_BICGSTABL_FAST) &&
      (l < 1 || l > kBlMaxL))
    return INVALID_PARAMETERS;
  bksp_gpu_stats* saved = g_stats;
  g_stats = stats;
  int ret = INVALID_PARAMETERS;
  try {
    cudaStream_t st = pick(stream);
    Timer tm(st);
    const long long l0 = launch_count(), y0 = byte_count();
    const int n = m->A.n;
    const long long np = pad64(n);
    double* db = dalloc_n<double>(np, st);
    double* dx = dalloc_n<double>(np, st);
    BK_CHECK(cudaMemsetAsync(db, 0, sizeof(double) * np, st));
    BK_CHECK(cudaMemsetAsync(dx, 0, sizeof(double) * np, st));
    tm.begin_solve();
    BK_CHECK(cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    BK_CHECK(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    SolveOut o;
    switch (method) {
      case BKSP_GPU_CG: o = bk::cg(m->A, db, dx, tol, max_iter, ss, st); break;
      case BKSP_GPU_CR: o = bk::cr(m->A, db, dx, tol, max_iter, ss, st); break;
      case BKSP_GPU_BICG: o = bk::bicg(m->A, m->At, db, dx, tol, max_iter, ss, st); break;
      case BKSP_GPU_BICGSTAB: o = bk::bicgstab(m->A, db, dx, tol, max_iter, ss, st); break;
      case BKSP_GPU_BICGSTABL: o = bk::bicgstabl(m->A, db, l, dx, tol, max_iter, ss, st); break;
      case BKSP_GPU_BICGSTABL_FAST:
        o = bk::bicgstabl(m->A, db, l, dx, tol, max_iter, ss, st, true);
        break;
      default: throw CudaError("unknown method");
    }
    BK_CHECK(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    tm.end_solve();
    BK_CHECK(cudaStreamSynchronize(st));
    tm.report(o.ret, &ss, o.iters);
    if (stats) {
      stats->launches = launch_count() - l0;
      stats->alg_bytes = byte_count() - y0;
      stats->true_res = true_residual_dev(m->A, db, dx, st);
    }
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    BK_CHECK(cudaStreamSynchronize(st));
    ret = o.ret;
  } catch (const std::exception& e) {
    ret = fail(e);
  }
  g_stats = saved;
  return ret;
}

int bksp_gpu_spmv(bksp_gpu_matrix* m, int fp32, const void* x, void* y,
                  void* stream) {
  if (!m || !x || !y) return INVALID_PARAMETERS;
  if (fp32 && !m->A.v32) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = pick(stream);
    thread_local SolveState ss;
    thread_local bool ready = false;
    if (!ready) {
      ss.create(0, st);
      ss.start(0, 1, 0.0, st);
      ready = true;
    }
    if (fp32)
      spmv(m->A, spmv_io<float>(static_cast<const float*>(x), static_cast<float*>(y)),
           ss.red(kD, E_NONE), st);
    else
      spmv(m->A, spmv_io<double>(static_cast<const double*>(x), static_cast<double*>(y)),
           ss.red(kD, E_NONE), st);
    BK_CHECK(cudaGetLastError());
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int bksp_gpu_spmm(bksp_gpu_matrix* m, int fp32, int s, int kernel,
                  const void* X, void* Y, void* stream) {
  if (!m || !X || !Y || s < 1 || s > 16 || kernel < -1 || kernel > 1)
    return INVALID_PARAMETERS;
  if (fp32 && !m->A.v32) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = pick(stream);
    thread_local SolveState ss;
    thread_local bool ready = false;
    if (!ready) {
      ss.create(0, st);
      ss.start(0, 1, 0.0, st);
      ready = true;
    }
    CsrH h = fp32 ? m->A.h32() : m->A.h64();
    if (kernel == 1) h.dia.nd = 0;   // the CSR kernel
    SpmmH a{};
    a.X = static_cast<const double*>(X);
    a.Y = static_cast<double*>(Y);
    a.alpha = 1.0;
    a.s = s;
    a.prec = fp32 ? 1 : 0;
    if (kernel == -1) spmm_autotune(h, s, a.prec, st);
    spmm_force(kernel);
    launch_spmm(h, a, ss.red(kD, E_NONE), st);
    spmm_force(-1);
    BK_CHECK(cudaGetLastError());
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

double bksp_gpu_true_residual(bksp_gpu_matrix* m, const double* b,
                              const double* x, void* stream) {
  if (!m || !b || !x) return NAN;
  try {
    cudaStream_t st = pick(stream);
    const int n = m->A.n;
    const long long np = pad64(n);
    double* db = dalloc_n<double>(np, st);
    double* dx = dalloc_n<double>(np, st);
    BK_CHECK(cudaMemsetAsync(db, 0, sizeof(double) * np, st));
    BK_CHECK(cudaMemsetAsync(dx, 0, sizeof(double) * np, st));
    BK_CHECK(cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    BK_CHECK(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    const double r = true_residual_dev(m->A, db, dx, st);
    dfree(db, st);
    dfree(dx, st);
    BK_CHECK(cudaStreamSynchronize(st));
    return r;
  } catch (const std::exception& e) {
    fail(e);
    return NAN;
  }
}

}  // extern "C"
