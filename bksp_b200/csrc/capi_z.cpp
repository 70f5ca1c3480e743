// extern "C" entry points of the complex API of bksp.h (reference
// include/bksp.h:111-182): zbicg, zbicgstabl, zblbicgstabl, zshbicgstabl,
// zqreco, zmat_create / zmat_free and zread_matrix_market.  Each solver call
// validates its arguments, uploads the complex CSR operator (and A^H for
// zbicg), the right-hand side and the initial guess, runs the device solve
// (zsolvers.cpp), downloads the solution and returns the reference's code;
// CUDA failures come back as INVALID_PARAMETERS.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bksp.h"
#include "../../include/bksp_gpu.h"
#include "capi_internal.h"
#include "mmio.h"
#include "runtime.h"
#include "zsolvers.h"

using namespace bk;

namespace {

int check_zmatrix(const zspmat* A) {
  if (!A || !A->row || !A->row_size || !A->nnz || !A->value) return -3;
  if (*A->row_size <= 0) return -3;
  if (*A->nnz > 0 && !A->col) return -3;
  if (A->row[*A->row_size] != *A->nnz) return -3;
  return 0;
}

// Host complex (interleaved re, im) vectors <-> padded device double2.
double2* zupload(const double* h, int n, int cols, cudaStream_t st) {
  const long long np = pad64(n);
  double2* d = dalloc_n<double2>(np * cols, st);
  BK_CHECK(cudaMemsetAsync(d, 0, sizeof(double2) * np * cols, st));
  if (h)
    for (int c = 0; c < cols; ++c)
      BK_CHECK(cudaMemcpyAsync(d + c * np, h + 2 * (size_t)c * n,
                               sizeof(double2) * n, cudaMemcpyHostToDevice, st));
  return d;
}

void zdownload(double* h, const double2* d, int n, int cols, cudaStream_t st) {
  const long long np = pad64(n);
  for (int c = 0; c < cols; ++c)
    BK_CHECK(cudaMemcpyAsync(h + 2 * (size_t)c * n, d + c * np,
                             sizeof(double2) * n, cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
}

// Column-major n-by-s zmat values <-> row-major padded device block.
double2* zupload_block(const double* h, int n, int s, cudaStream_t st) {
  const long long np = pad64(n);
  std::vector<double> rm(2 * (size_t)np * s, 0.0);
  for (int j = 0; j < s; ++j)
    for (int i = 0; i < n; ++i) {
      rm[2 * ((size_t)i * s + j)] = h[2 * ((size_t)j * n + i)];
      rm[2 * ((size_t)i * s + j) + 1] = h[2 * ((size_t)j * n + i) + 1];
    }
  double2* d = dalloc_n<double2>(np * s, st);
  BK_CHECK(cudaMemcpyAsync(d, rm.data(), sizeof(double2) * np * s,
                           cudaMemcpyHostToDevice, st));
  BK_CHECK(cudaStreamSynchronize(st));
  return d;
}

void zdownload_block(double* h, const double2* d, int n, int s, cudaStream_t st) {
  std::vector<double> rm(2 * (size_t)n * s);
  BK_CHECK(cudaMemcpyAsync(rm.data(), d, sizeof(double2) * (size_t)n * s,
                           cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
  for (int j = 0; j < s; ++j)
    for (int i = 0; i < n; ++i) {
      h[2 * ((size_t)j * n + i)] = rm[2 * ((size_t)i * s + j)];
      h[2 * ((size_t)j * n + i) + 1] = rm[2 * ((size_t)i * s + j) + 1];
    }
}

const double* dv(const double _Complex* p) { return reinterpret_cast<const double*>(p); }
double* dv(double _Complex* p) { return reinterpret_cast<double*>(p); }

int fail(const std::exception& e) {
  if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
  cudaGetLastError();
  return INVALID_PARAMETERS;
}

// Launches and algorithmic bytes of the call, into the recorded stats.
struct Counts {
  long long l0 = launch_count(), y0 = byte_count();
  void report() const {
    if (!g_stats) return;
    g_stats->launches = launch_count() - l0;
    g_stats->alg_bytes = byte_count() - y0;
  }
};

enum class ZMethod { BICG, BICGSTABL };

int zsolve_single(ZMethod m, zspmat* A, double _Complex* b, int l, double tol,
                  int max_iter, double _Complex* x) {
  if (check_zmatrix(A) != 0 || !b || !x) return INVALID_PARAMETERS;
  if (m == ZMethod::BICGSTABL && (l < 1 || l > kBlMaxL)) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    const Counts cnt;
    const int n = *A->row_size;
    ZDevCsr dA, dAH;
    upload_zcsr(n, A->row, A->col, dv(A->value), false, dA, st);
    if (m == ZMethod::BICG) upload_zcsr(n, A->row, A->col, dv(A->value), true, dAH, st);
    double2* db = zupload(dv(b), n, 1, st);
    double2* dx = zupload(dv(x), n, 1, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    SolveOut o = m == ZMethod::BICG
                     ? zbicg(dA, dAH, db, dx, tol, max_iter, ss, st)
                     : zbicgstabl(dA, db, l, dx, tol, max_iter, ss, st);
    tm.end_solve();
    zdownload(dv(x), dx, n, 1, st);
    tm.report(o.ret, &ss, o.iters);
    cnt.report();
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    dA.release(st);
    if (m == ZMethod::BICG) dAH.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

}  // namespace

extern "C" {

int zbicg(zspmat* A, double _Complex* b, double tol, int max_iter,
          double _Complex* x) {
  return zsolve_single(ZMethod::BICG, A, b, 0, tol, max_iter, x);
}

int zbicgstabl(zspmat* A, double _Complex* b, int ell, double tol,
               int max_iter, double _Complex* x) {
  return zsolve_single(ZMethod::BICGSTABL, A, b, ell, tol, max_iter, x);
}

int zshbicgstabl(zspmat* A, double _Complex* b, int l, double _Complex* sigma,
                 int sigma_size, double tol, int max_iter, double _Complex* x) {
  if (check_zmatrix(A) != 0 || !b || !x || (sigma_size > 0 && !sigma))
    return INVALID_PARAMETERS;
  if (l < 1 || l > kBlMaxL || sigma_size < 0 || sigma_size > kZMaxShifts)
    return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    const Counts cnt;
    const int n = *A->row_size;
    ZDevCsr dA;
    upload_zcsr(n, A->row, A->col, dv(A->value), false, dA, st);
    double2* db = zupload(dv(b), n, 1, st);
    double2* dx = zupload(dv(x), n, sigma_size + 1, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    SolveOut o = zshbicgstabl(dA, db, l, dv(sigma), sigma_size, dx, tol,
                              max_iter, ss, st);
    tm.end_solve();
    zdownload(dv(x), dx, n, sigma_size + 1, st);
    tm.report(o.ret, &ss, o.iters);
    cnt.report();
    ss.release(st);
    dfree(db, st);
    dfree(dx, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int zblbicgstabl(zspmat* A, zmat* B, int ell, double tol, int max_iter,
                 zmat* X) {
  if (check_zmatrix(A) != 0 || !B || !X || !B->value || !X->value)
    return INVALID_PARAMETERS;
  const int n = *A->row_size, s = B->col_size;
  if (B->row_size != n || X->row_size != n || X->col_size != s || s < 1 ||
      s > 16 || ell < 1 || ell > kBlMaxL)
    return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    Timer tm(st);
    const Counts cnt;
    ZDevCsr dA;
    upload_zcsr(n, A->row, A->col, dv(A->value), false, dA, st);
    double2* dB = zupload_block(dv(B->value), n, s, st);
    double2* dX = zupload_block(dv(X->value), n, s, st);
    SolveState ss;
    ss.create(hist_cap_for(max_iter), st);
    tm.begin_solve();
    double true_res = 0.0;
    SolveOut o = zblbicgstabl(dA, dB, s, ell, dX, tol, max_iter, ss, st, &true_res);
    tm.end_solve();
    zdownload_block(dv(X->value), dX, n, s, st);
    // The reference prints this summary on every exit
    // (src/blbicgstabl.c:465-469).
    const double err = ss.get_scalar(kErr, st);
    const int it = o.ret >= 0 ? o.ret : max_iter;
    std::printf("Block BiCGSTAB(%d) has converged at:\n"
                "        The number of iteration ... %d\n"
                "        Frobenius norm of the relative residual ... %e\n"
                "        Frobenius norm of the true residual ... %e\n",
                ell, it, err, true_res);
    std::fflush(stdout);
    tm.report(o.ret, &ss, o.iters);
    cnt.report();
    if (g_stats) g_stats->true_res = true_res;
    ss.release(st);
    dfree(dB, st);
    dfree(dX, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return o.ret;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int zqreco(int m, int n, double _Complex* mat, double _Complex* r) {
  if (m < 1 || n < 1 || n > 16 || n > m || !mat || !r) return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    double2* dV = zupload_block(dv(mat), m, n, st);
    SolveState ss;
    ss.create(0, st);
    std::vector<double> R(2 * (size_t)n * n);
    const bool ok = zthin_qr(m, n, dV, R.data(), ss, st);
    zdownload_block(dv(mat), dV, m, n, st);
    // R row-major pairs -> column-major r, zero below the diagonal.
    double* rr = dv(r);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        rr[2 * ((size_t)j * n + i)] = i <= j ? R[2 * ((size_t)i * n + j)] : 0.0;
        rr[2 * ((size_t)j * n + i) + 1] = i <= j ? R[2 * ((size_t)i * n + j) + 1] : 0.0;
      }
    ss.release(st);
    dfree(dV, st);
    BK_CHECK(cudaStreamSynchronize(st));
    return ok ? 0 : 1;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int bksp_gpu_zcsrmv(zspmat* A, char trans, const double _Complex* x,
                    double _Complex* y) {
  if (check_zmatrix(A) != 0 || !x || !y || (trans != 'n' && trans != 't'))
    return INVALID_PARAMETERS;
  try {
    Ctx& cx = Ctx::get();
    cudaStream_t st = cx.st;
    const int n = *A->row_size;
    ZDevCsr dA;
    upload_zcsr(n, A->row, A->col, dv(A->value), trans == 't', dA, st);
    double2* dx = zupload(dv(x), n, 1, st);
    double2* dy = zupload(nullptr, n, 1, st);
    SolveState ss;
    ss.create(0, st);
    ZSpmvH io;
    std::memset(&io, 0, sizeof(io));
    io.x = dx;
    io.y = dy;
    launch_zspmv(dA.h(), io, ss.red_after(kD, E_NONE), st);
    zdownload(dv(y), dy, n, 1, st);
    ss.release(st);
    dfree(dx, st);
    dfree(dy, st);
    dA.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

zmat* zmat_create(int m, int n) {
  zmat* mat = (zmat*)std::malloc(sizeof(zmat));
  if (!mat) return nullptr;
  const size_t cnt = (size_t)(m > 0 ? m : 0) * (size_t)(n > 0 ? n : 0);
  mat->value = (double _Complex*)std::calloc(cnt > 0 ? cnt : 1, sizeof(double _Complex));
  if (!mat->value) {
    std::free(mat);
    return nullptr;
  }
  mat->row_size = m;
  mat->col_size = n;
  return mat;
}

int zmat_free(zmat* mat) {
  if (!mat) return 0;
  std::free(mat->value);
  std::free(mat);
  return 0;
}

// src/read_matrix.c:176-246 + zcoo2csr (:248-301): entries in file order
// within each row.  Unlike the reference (which exits the process), an
// unreadable or non-complex file returns NULL.
zspmat* zread_matrix_market(char* filename) {
  if (!filename) return nullptr;
  MmData d;
  if (!mm_parse(filename, d, true)) return nullptr;
  const int n = (int)d.rows;
  const long long nz = (long long)d.ri.size();
  zspmat* mat = (zspmat*)std::malloc(sizeof(zspmat));
  int* row_size = (int*)std::malloc(sizeof(int));
  int* col_size = (int*)std::malloc(sizeof(int));
  int* nnzp = (int*)std::malloc(sizeof(int));
  int* row = (int*)std::calloc((size_t)n + 1, sizeof(int));
  int* col = (int*)std::malloc(sizeof(int) * (nz > 0 ? nz : 1));
  double* val = (double*)std::malloc(2 * sizeof(double) * (nz > 0 ? nz : 1));
  if (!mat || !row_size || !col_size || !nnzp || !row || !col || !val) {
    std::free(mat); std::free(row_size); std::free(col_size); std::free(nnzp);
    std::free(row); std::free(col); std::free(val);
    return nullptr;
  }
  for (long long k = 0; k < nz; ++k) row[d.ri[k] + 1]++;
  for (int i = 0; i < n; ++i) row[i + 1] += row[i];
  std::vector<int> pos(row, row + n);
  for (long long k = 0; k < nz; ++k) {
    const int p = pos[d.ri[k]]++;
    col[p] = d.ci[k];
    val[2 * (size_t)p] = d.vv[k];
    val[2 * (size_t)p + 1] = d.vi[k];
  }
  *row_size = n;
  *col_size = (int)d.cols;
  *nnzp = (int)nz;
  mat->row = row;
  mat->col = col;
  mat->nnz = nnzp;
  mat->row_size = row_size;
  mat->col_size = col_size;
  mat->value = (double _Complex*)val;
  mat->format = (char*)"csr";
  mat->type = (char*)(d.symmetric ? "symmetric" : "unsymmetric");
  return mat;
}

}  // extern "C"
