// bksp_gpu.h: Matrix Market file straight into a device-resident operator.
// The host parses the text (mmio.cpp, several threads); the row sort, the
// mirroring of a stored triangle and the CSR assembly run on the GPU, so no
// O(nnz) host pass follows the parse.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

#include "capi_internal.h"
#include "mmio.h"

using namespace bk;

namespace {

int fail(const std::exception& e) {
  if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
  cudaGetLastError();
  return INVALID_PARAMETERS;
}

}  // namespace

extern "C" int bksp_gpu_read_matrix_market(const char* path, int flags,
                                           bksp_gpu_matrix** out) {
  if (!path || !out || (flags & BKSP_GPU_TRANSPOSE)) return INVALID_PARAMETERS;
  *out = nullptr;
  MmData d;
  if (!mm_parse(path, d) || d.rows != d.cols) return INVALID_PARAMETERS;
  bksp_gpu_matrix* m = new (std::nothrow) bksp_gpu_matrix();
  if (!m) return INVALID_PARAMETERS;
  Ctx& cx = Ctx::get();
  cudaStream_t st = cx.st;
  int *dri = nullptr, *dci = nullptr, *cnt = nullptr, *drp = nullptr, *col = nullptr;
  double *dvv = nullptr, *val = nullptr;
  long long* key = nullptr;
  auto free_tmp = [&]() {
    dfree(dri, st); dfree(dci, st); dfree(dvv, st); dfree(cnt, st);
    dfree(drp, st); dfree(col, st); dfree(val, st); dfree(key, st);
    dri = dci = cnt = drp = col = nullptr;
    dvv = val = nullptr;
    key = nullptr;
  };
  try {
    m->flags = flags;
    m->device = cx.device;
    const int n = (int)d.rows;
    const long long nz = (long long)d.ri.size();
    const int mirror = (flags & BKSP_GPU_MIRROR) && d.symmetric ? 1 : 0;
    dri = dalloc_n<int>(nz, st);
    dci = dalloc_n<int>(nz, st);
    dvv = dalloc_n<double>(nz, st);
    cnt = dalloc_n<int>(n, st);
    if (nz > 0) {
      BK_CHECK(cudaMemcpyAsync(dri, d.ri.data(), sizeof(int) * nz, cudaMemcpyHostToDevice, st));
      BK_CHECK(cudaMemcpyAsync(dci, d.ci.data(), sizeof(int) * nz, cudaMemcpyHostToDevice, st));
      BK_CHECK(cudaMemcpyAsync(dvv, d.vv.data(), sizeof(double) * nz, cudaMemcpyHostToDevice, st));
    }
    BK_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * n, st));
    if (nz > 0) launch_coo_count(dri, dci, nz, mirror, cnt, st);
    BK_CHECK(cudaGetLastError());
    // Row pointers: the counts' prefix sum (O(n), on the host).
    std::vector<int> rp(n + 1, 0);
    BK_CHECK(cudaMemcpyAsync(rp.data() + 1, cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    long long total = 0;
    for (int i = 0; i < n; ++i) {
      total += rp[i + 1];
      if (total > 0x7fffffff) throw CudaError("matrix: too many entries");
      rp[i + 1] = (int)total;
    }
    drp = dalloc_n<int>(n + 1, st);
    col = dalloc_n<int>(total, st);
    val = dalloc_n<double>(total, st);
    key = dalloc_n<long long>(total, st);
    BK_CHECK(cudaMemcpyAsync(drp, rp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    BK_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * n, st));   // reused as fill
    if (nz > 0) {
      launch_coo_scatter(dri, dci, dvv, nz, mirror, drp, cnt, col, val, key, st);
      launch_row_sort(drp, n, mirror, col, val, key, st);
      BK_CHECK(cudaGetLastError());
    }
    const bool f32 = (flags & BKSP_GPU_FP32) != 0;
    upload_csr(n, rp.data(), col, val, f32, m->A, st, /*cv_on_device=*/true);
    if (f32) spai_build_slots(m->A, m->spai, st);
    m->diag_ok = !(m->A.scan.flags & kScanNoDiag);
    free_tmp();
    BK_CHECK(cudaStreamSynchronize(st));
    *out = m;
    return 0;
  } catch (const std::exception& e) {
    cudaStreamSynchronize(st);
    free_tmp();
    m->A.release(st);
    m->spai.release(st);
    cudaStreamSynchronize(st);
    delete m;
    return fail(e);
  }
}

extern "C" int bksp_gpu_matrix_csr(const bksp_gpu_matrix* m, int* rowptr, int* col,
                                   double* val) {
  if (!m) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = Ctx::get().st;
    const int n = m->A.n, nnz = m->A.nnz;
    if (rowptr)
      BK_CHECK(cudaMemcpyAsync(rowptr, m->A.rowptr, sizeof(int) * (n + 1),
                               cudaMemcpyDeviceToHost, st));
    if (col && nnz > 0)
      BK_CHECK(cudaMemcpyAsync(col, m->A.col, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
    if (val && nnz > 0)
      BK_CHECK(cudaMemcpyAsync(val, m->A.v64, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
