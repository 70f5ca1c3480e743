// Kernels and launch wrappers (kernel_api.h) of the precision conversions,
// the mixed-precision steps and the scalar / control nodes of a solve, plus
// the shared launch bookkeeping.  The other kernels live in kernels_spmv.cu,
// kernels_vec.cu and kernels_block.cu; every translation unit compiles its
// own copy of the scalar epilogues (epilogues.cuh).
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "kernel_api.h"
#include "launch_util.h"

namespace bk {

long long& launch_count() {
  thread_local long long n = 0;
  return n;
}

long long& byte_count() {
  thread_local long long n = 0;
  return n;
}

// Blocks of `kernel` (kThreads threads, no dynamic shared memory) that are
// resident on the whole GPU at once, cached per kernel.
int resident_grid(const void* kernel) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  const auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int dev = 0, sms = kSMs, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  long long g = (long long)per_sm * sms;
  if (g > kMaxBlocks) g = kMaxBlocks;
  cache[kernel] = (int)g;
  return (int)g;
}

// ----------------------------------------------------------- conversions

__global__ void k_convert_d2f(const double* __restrict__ a, float* __restrict__ b,
                              long long n) {
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads)
    b[i] = (float)a[i];
}
__global__ void k_convert_f2d(const float* __restrict__ a, double* __restrict__ b,
                              long long n) {
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads)
    b[i] = (double)a[i];
}
void launch_convert_d2f(const double* a, float* b, long long n, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("precision conversion");
  ++launch_count();
  byte_count() += n * 12;
  k_convert_d2f<<<grid_for(n), kThreads, 0, st>>>(a, b, n);
}
void launch_convert_f2d(const float* a, double* b, long long n, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("precision conversion");
  ++launch_count();
  byte_count() += n * 12;
  k_convert_f2d<<<grid_for(n), kThreads, 0, st>>>(a, b, n);
}

// ---------------------------------------------------- operator analysis

constexpr int kEmptyOff = INT_MIN;   // never a column offset (|j - i| < n)

// Insert offset o into a table of kScanOffs slots filled front to back
// (shared or global memory); false when the table is full of other offsets.
__device__ __forceinline__ bool offset_insert(int* tab, int o) {
  for (int s = 0; s < kScanOffs; ++s) {
    const int v = *(volatile int*)(tab + s);
    if (v == o) return true;
    if (v == kEmptyOff) {
      const int prev = atomicCAS(tab + s, kEmptyOff, o);
      if (prev == kEmptyOff || prev == o) return true;
    }
  }
  return false;
}

__global__ void __launch_bounds__(kThreads)
k_csr_scan(const int* __restrict__ rowptr, const int* __restrict__ col,
           const double* __restrict__ val, int n, double* __restrict__ diag,
           CsrScanH* scan) {
  __shared__ int tab[kScanOffs];
  __shared__ int sflags;
  if (threadIdx.x < kScanOffs) tab[threadIdx.x] = kEmptyOff;
  if (threadIdx.x == 0) sflags = 0;
  __syncthreads();
  const int i = blockIdx.x * kThreads + threadIdx.x;
  int fl = 0;
  if (i < n) {
    const int k0 = rowptr[i], k1 = rowptr[i + 1];
    int prev = -1;
    double d = 0.0;
    bool has_d = false;
    for (int k = k0; k < k1; ++k) {
      const int c = col[k];
      if (c < 0 || c >= n) {
        fl |= kScanBadCol;
        continue;
      }
      if (c <= prev) fl |= kScanUnsorted;
      prev = c;
      if (c == i && !has_d) {
        d = val[k];
        has_d = true;
      }
      if (!offset_insert(tab, c - i)) fl |= kScanManyOffs;
    }
    if (!has_d || d == 0.0) fl |= kScanNoDiag;
    diag[i] = d;
  }
  if (fl) atomicOr(&sflags, fl);
  __syncthreads();
  if (threadIdx.x == 0 && sflags) atomicOr(&scan->flags, sflags);
  if (threadIdx.x < kScanOffs) {
    const int o = tab[threadIdx.x];
    if (o != kEmptyOff && !offset_insert(scan->off, o))
      atomicOr(&scan->flags, (int)kScanManyOffs);
  }
}

__global__ void k_scan_init(CsrScanH* scan) {
  scan->flags = 0;
  scan->noff = 0;
  for (int s = 0; s < kScanOffs; ++s) scan->off[s] = kEmptyOff;
}

__global__ void k_scan_count(CsrScanH* scan) {
  int c = 0;
  for (int s = 0; s < kScanOffs; ++s) c += scan->off[s] != kEmptyOff;
  scan->noff = c;
}

void launch_csr_scan(const int* rowptr, const int* col, const double* val, int n,
                     double* diag, CsrScanH* scan, cudaStream_t st) {
  launch_count() += 3;
  k_scan_init<<<1, 1, 0, st>>>(scan);
  k_csr_scan<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(rowptr, col, val, n,
                                                                  diag, scan);
  k_scan_count<<<1, 1, 0, st>>>(scan);
}

// ------------------------------------------------- mixed-precision steps

// o0 = o1 = o2 = fl32(in) (null outputs skipped); optional dot (w, o0),
// where w == nullptr with ND = 1 means (o0, o0).
template <int ND>
__global__ void __launch_bounds__(kThreads)
k_mx_d2f(const double* __restrict__ in, float* o0, float* o1, float* o2,
         const float* w, long long n, Red rd) {
  if (skip(rd)) return;
  double acc[ND > 0 ? ND : 1];
  if (ND > 0) acc[0] = 0.0;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    const float v = (float)in[i];
    const float wv = (ND > 0 && w) ? w[i] : v;   // read before any store
    o0[i] = v;
    if (o1) o1[i] = v;
    if (o2) o2[i] = v;
    if (ND > 0) acc[0] += (double)wv * (double)v;
  }
  if (ND > 0 || rd.epi) finish_reduction<ND>(acc, rd);
}

void launch_mx_d2f(const double* in, float* o0, float* o1, float* o2,
                   const float* w, int nd, long long n, const RedH& rd,
                   cudaStream_t st) {
  byte_count() += n * (8 + 4 * ((o1 != nullptr) + (o2 != nullptr) + 1 + (w != nullptr)));
  if (g_prog_rec) {
    if (n % 4) prog_unsupported("unpadded vector");
    for (const void* p : {(const void*)in, (const void*)o0, (const void*)o1,
                          (const void*)o2, (const void*)w})
      if (p) prog_require_aligned(p);
    ProgOpH op;
    std::memset(&op, 0, sizeof(op));
    op.kind = kOpMxD2f;
    op.u.d2f = MxD2fH{in, o0, o1, o2, w, n, nd ? 1 : 0};
    op.units = prog_units(n);
    op.rd = rd;
    prog_push(op);
    return;
  }
  ++launch_count();
  if (nd)
    launch_k(k_mx_d2f<1>, grid_wave(k_mx_d2f<1>, n), kThreads, 0, st, in, o0, o1, o2, w, n, rd);
  else
    launch_k(k_mx_d2f<0>, grid_wave(k_mx_d2f<0>, n), kThreads, 0, st, in, o0, o1, o2, w, n, rd);
}

// x64 += t32 (the preconditioned correction M y), then y32 = 0.
__global__ void __launch_bounds__(kThreads)
k_mx_accum(double* __restrict__ x, const float* __restrict__ t,
           float* __restrict__ y, long long n, Red rd) {
  if (skip(rd)) return;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    x[i] += (double)t[i];
    y[i] = 0.0f;
  }
}

void launch_mx_accum(double* x, const float* t, float* y, long long n,
                     const RedH& rd, cudaStream_t st) {
  byte_count() += n * 24;   // x read and written, t read, y written
  if (g_prog_rec) {
    if (n % 4) prog_unsupported("unpadded vector");
    prog_require_aligned(x);
    prog_require_aligned(t);
    prog_require_aligned(y);
    ProgOpH op;
    std::memset(&op, 0, sizeof(op));
    op.kind = kOpMxAccum;
    op.u.acc = MxAccH{x, t, y, n};
    op.units = prog_units(n);
    op.rd = rd;
    prog_push(op);
    return;
  }
  ++launch_count();
  launch_k(k_mx_accum, grid_wave(k_mx_accum, n), kThreads, 0, st, x, t, y, n, rd);
}

// ------------------------------------------------------- scalar / control

// Start of a solve: control block and arrival ticket reset on the device
// (no host synchronisation), optional scalar preset.
__global__ void k_ctl_init(Ctl* c, unsigned* ticket, double* S, int iter0,
                           int max_iter, double tol, double* hist, int hist_cap,
                           short slot, double value) {
  c->done = 0;
  c->iter = iter0;
  c->ret = kNotConverged;
  c->max_iter = max_iter;
  c->hist_cap = hist_cap;
  c->trips = 0;
  c->trip_cap = max_iter - iter0 + 2 > 1 ? max_iter - iter0 + 2 : 1;
  c->hist_len = 0;
  c->tol = tol;
  c->hist = hist;
  c->cond = 0ull;
  c->cond_alt = 0ull;
  c->use_cond = 0;
  ticket[0] = 0u;
  if (slot >= 0) S[slot] = value;
}

void launch_ctl_init(CtlH* c, unsigned* ticket, double* S, int iter0,
                     int max_iter, double tol, double* hist, int hist_cap,
                     short slot, double value, cudaStream_t st) {
  ++launch_count();
  k_ctl_init<<<1, 1, 0, st>>>(c, ticket, S, iter0, max_iter, tol, hist,
                              hist_cap, slot, value);
}

__global__ void k_set_scalar(double* S, short slot, double v) {
  pdl_enter();
  S[slot] = v;
}

void launch_set_scalar(double* S, short slot, double v, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("scalar preset");
  ++launch_count();
  launch_k(k_set_scalar, 1, 1, 0, st, S, slot, v);
}

__global__ void k_epilogue(Red rd) {
  if (skip(rd)) return;
  run_epilogue(rd);
}

void launch_epilogue(const RedH& rd, cudaStream_t st) {
  if (g_prog_rec) {
    ProgOpH op;
    std::memset(&op, 0, sizeof(op));
    op.kind = kOpEpi;
    op.units = 1;
    op.rd = rd;
    prog_push(op);
    return;
  }
  ++launch_count();
  launch_k(k_epilogue, 1, 1, 0, st, rd);
}

// Body-final node of a solve's CUDA-graph while loop.  The loop ends when a
// convergence test has finished the solve, and in any case after trip_cap
// trips: the cap is checked here, independently of the method's epilogues,
// so a device-side loop can never outlive its iteration budget.
__global__ void k_loop_control(Ctl* c, cudaGraphConditionalHandle h,
                               int use_handle) {
  pdl_enter();
  const int trips = ++c->trips;
  bool keep = !c->done;
  if (keep && trips >= c->trip_cap) {
    c->done = 1;
    c->ret = kNotConverged;
    keep = false;
  }
  if (use_handle) cudaGraphSetConditional(h, keep ? 1u : 0u);
}

void launch_loop_control(CtlH* ctl, unsigned long long handle, int use_handle,
                         cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("loop control");
  ++launch_count();
  launch_k(k_loop_control, 1, 1, 0, st, ctl, (cudaGraphConditionalHandle)handle,
                                  use_handle);
}

}  // namespace bk
