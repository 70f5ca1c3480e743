// Matrix Market -> CSR on the GPU: a counting sort by row of the parsed
// coordinates (atomic row counts, host prefix sum, atomic placement), then a
// per-row sort that restores the host reader's order -- file order within
// a row (the reference's coo2csr, src/read_matrix.c, is a stable counting
// sort by row), or, for a mirrored symmetric file, ascending column with
// ties in insertion order (as the host expansion of a one-triangle operator
// orders its rows).
#include <cuda_runtime.h>

#include "kernel_api.h"

namespace bk {

namespace {

__global__ void k_coo_count(const int* __restrict__ ri, const int* __restrict__ ci,
                            long long nz, int mirror, int* __restrict__ cnt) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nz;
       k += (long long)gridDim.x * blockDim.x) {
    const int r = ri[k], c = ci[k];
    atomicAdd(cnt + r, 1);
    if (mirror && c != r) atomicAdd(cnt + c, 1);
  }
}

__global__ void k_coo_scatter(const int* __restrict__ ri, const int* __restrict__ ci,
                              const double* __restrict__ vv, long long nz, int mirror,
                              const int* __restrict__ rowptr, int* __restrict__ fill,
                              int* __restrict__ col, double* __restrict__ val,
                              long long* __restrict__ key) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nz;
       k += (long long)gridDim.x * blockDim.x) {
    const int r = ri[k], c = ci[k];
    const double v = vv[k];
    const long long kk = ((long long)r << 32) | (long long)(unsigned)k;
    int p = rowptr[r] + atomicAdd(fill + r, 1);
    col[p] = c;
    val[p] = v;
    key[p] = kk;
    if (mirror && c != r) {
      p = rowptr[c] + atomicAdd(fill + c, 1);
      col[p] = r;
      val[p] = v;
      key[p] = kk;
    }
  }
}

// Heap sort of one row (O(L log L), in place), by key or by (column, key).
__device__ __forceinline__ bool row_less(const int* col, const long long* key,
                                         int a, int b, int by_col) {
  if (by_col && col[a] != col[b]) return col[a] < col[b];
  return key[a] < key[b];
}

__device__ void row_swap(int* col, double* val, long long* key, int a, int b) {
  const int c = col[a]; col[a] = col[b]; col[b] = c;
  const double v = val[a]; val[a] = val[b]; val[b] = v;
  const long long k = key[a]; key[a] = key[b]; key[b] = k;
}

__device__ void sift_down(int* col, double* val, long long* key, int base, int root,
                          int len, int by_col) {
  for (;;) {
    int child = 2 * root + 1;
    if (child >= len) return;
    if (child + 1 < len && row_less(col, key, base + child, base + child + 1, by_col))
      ++child;
    if (!row_less(col, key, base + root, base + child, by_col)) return;
    row_swap(col, val, key, base + root, base + child);
    root = child;
  }
}

__global__ void k_row_sort(const int* __restrict__ rowptr, int n, int by_col,
                           int* col, double* val, long long* key) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int base = rowptr[r], len = rowptr[r + 1] - base;
  if (len < 2) return;
  for (int i = len / 2 - 1; i >= 0; --i) sift_down(col, val, key, base, i, len, by_col);
  for (int end = len - 1; end > 0; --end) {
    row_swap(col, val, key, base, base + end);
    sift_down(col, val, key, base, 0, end, by_col);
  }
}

int grid_of(long long items) {
  long long g = (items + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

}  // namespace

void launch_coo_count(const int* ri, const int* ci, long long nz, int mirror,
                      int* cnt, cudaStream_t st) {
  ++launch_count();
  k_coo_count<<<grid_of(nz), 256, 0, st>>>(ri, ci, nz, mirror, cnt);
}

void launch_coo_scatter(const int* ri, const int* ci, const double* vv,
                        long long nz, int mirror, const int* rowptr, int* fill,
                        int* col, double* val, long long* key, cudaStream_t st) {
  ++launch_count();
  k_coo_scatter<<<grid_of(nz), 256, 0, st>>>(ri, ci, vv, nz, mirror, rowptr, fill,
                                             col, val, key);
}

void launch_row_sort(const int* rowptr, int n, int by_col, int* col, double* val,
                     long long* key, cudaStream_t st) {
  ++launch_count();
  k_row_sort<<<(n + 255) / 256, 256, 0, st>>>(rowptr, n, by_col, col, val, key);
}

}  // namespace bk
