// Single translation unit holding every device kernel of the library (the
// scalar epilogues are one device function shared by all reductions) and
// the host-callable launch wrappers declared in kernel_api.h.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_spmv.cuh"
#include "k_spmv_tma.cuh"
#include "k_spmv_vec.cuh"
#include "k_spmv_wtile.cuh"
#include "k_vec.cuh"
#include "k_shift.cuh"
#include "k_block.cuh"
#include "kernel_api.h"

namespace bk {

long long& launch_count() {
  thread_local long long n = 0;
  return n;
}

static inline int grid_for(long long work_items) {
  long long g = (work_items + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > kMaxBlocks) g = kMaxBlocks;
  return (int)g;
}

// ------------------------------------------------------------------ SpMV

// SpMV kernel variants (every one sums a row in the reference's order):
//   0 tile (register-staged products), 1 tile with TMA bulk copies,
//   2..5 vector CSR with 4, 8, 16, 32 lanes per row, 6 warp tile.
// CsrH.variant carries the choice made for the operator (autotuner);
// BKSP_GPU_SPMV=tile|tma|vec4|vec8|vec16|vec32 overrides it.
static int spmv_override() {
  static int v = -2;
  if (v == -2) {
    const char* e = std::getenv("BKSP_GPU_SPMV");
    v = -1;
    if (e) {
      const std::string s(e);
      if (s == "tile") v = 0;
      else if (s == "tma") v = 1;
      else if (s == "vec4") v = 2;
      else if (s == "vec8") v = 3;
      else if (s == "vec16") v = 4;
      else if (s == "vec32") v = 5;
      else if (s == "wtile") v = 6;
    }
  }
  return v;
}

template <typename VT, typename XT, int L>
static void spmv_vec_launch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                            cudaStream_t st) {
  long long g = ((long long)A.n * L + kThreads - 1) / kThreads;
  if (g > kMaxBlocks) g = kMaxBlocks;
  if (g < 1) g = 1;
  switch (io.nd) {
    case 0: k_spmv_vec<VT, XT, 0, L><<<(int)g, kThreads, 0, st>>>(A, io, rd); break;
    case 1: k_spmv_vec<VT, XT, 1, L><<<(int)g, kThreads, 0, st>>>(A, io, rd); break;
    case 2: k_spmv_vec<VT, XT, 2, L><<<(int)g, kThreads, 0, st>>>(A, io, rd); break;
    default: k_spmv_vec<VT, XT, 3, L><<<(int)g, kThreads, 0, st>>>(A, io, rd); break;
  }
}

template <typename VT, typename XT, int ND>
static void spmv_tma_launch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                            cudaStream_t st) {
  const size_t sm = 2 * (size_t)kStageEnt * (sizeof(int) + sizeof(VT));
  static int attr_dev = -1, per_sm = 1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_spmv_tma<VT, XT, ND>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_tma<VT, XT, ND>,
                                                  kThreads, sm);
    if (per_sm < 1) per_sm = 1;
    attr_dev = dev;
  }
  int g = kSMs * per_sm;
  if (g > kMaxBlocks) g = kMaxBlocks;
  if (g > A.nrb) g = A.nrb > 0 ? A.nrb : 1;
  k_spmv_tma<VT, XT, ND><<<g, kThreads, sm, st>>>(A, io, rd);
}

template <typename VT, typename XT>
static void spmv_dispatch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                          cudaStream_t st) {
  int var = spmv_override();
  if (var < 0) var = A.variant;
  switch (var) {
    case 1:
      switch (io.nd) {
        case 0: spmv_tma_launch<VT, XT, 0>(A, io, rd, st); return;
        case 1: spmv_tma_launch<VT, XT, 1>(A, io, rd, st); return;
        case 2: spmv_tma_launch<VT, XT, 2>(A, io, rd, st); return;
        default: spmv_tma_launch<VT, XT, 3>(A, io, rd, st); return;
      }
    case 2: spmv_vec_launch<VT, XT, 4>(A, io, rd, st); return;
    case 3: spmv_vec_launch<VT, XT, 8>(A, io, rd, st); return;
    case 4: spmv_vec_launch<VT, XT, 16>(A, io, rd, st); return;
    case 5: spmv_vec_launch<VT, XT, 32>(A, io, rd, st); return;
    case 6: {
      const int g = A.nrb < kMaxBlocks ? (A.nrb > 0 ? A.nrb : 1) : kMaxBlocks;
      switch (io.nd) {
        case 0: k_spmv_wtile<VT, XT, 0><<<g, kThreads, 0, st>>>(A, io, rd); return;
        case 1: k_spmv_wtile<VT, XT, 1><<<g, kThreads, 0, st>>>(A, io, rd); return;
        case 2: k_spmv_wtile<VT, XT, 2><<<g, kThreads, 0, st>>>(A, io, rd); return;
        default: k_spmv_wtile<VT, XT, 3><<<g, kThreads, 0, st>>>(A, io, rd); return;
      }
    }
    default: break;
  }
  const int g = A.nrb < kMaxBlocks ? (A.nrb > 0 ? A.nrb : 1) : kMaxBlocks;
  switch (io.nd) {
    case 0: k_spmv<VT, XT, 0><<<g, kThreads, 0, st>>>(A, io, rd); break;
    case 1: k_spmv<VT, XT, 1><<<g, kThreads, 0, st>>>(A, io, rd); break;
    case 2: k_spmv<VT, XT, 2><<<g, kThreads, 0, st>>>(A, io, rd); break;
    default: k_spmv<VT, XT, 3><<<g, kThreads, 0, st>>>(A, io, rd); break;
  }
}

void launch_spmv_d(const CsrH& A, const SpmvH<double>& io, const RedH& rd,
                   cudaStream_t st) {
  ++launch_count();
  spmv_dispatch<double, double>(A, io, rd, st);
}
void launch_spmv_f(const CsrH& A, const SpmvH<float>& io, const RedH& rd,
                   cudaStream_t st) {
  ++launch_count();
  spmv_dispatch<float, float>(A, io, rd, st);
}

// ------------------------------------------------------ linear combination

template <typename T, int MI, int MO>
static void lc_nd(const LcH<T>& d, const RedH& rd, cudaStream_t st) {
  const int g = grid_for(d.n / Pack<T>::N);
  switch (d.nd) {
    case 0: k_lincomb<T, MI, MO, 0><<<g, kThreads, 0, st>>>(d, rd); break;
    case 1: k_lincomb<T, MI, MO, 1><<<g, kThreads, 0, st>>>(d, rd); break;
    case 2: k_lincomb<T, MI, MO, 2><<<g, kThreads, 0, st>>>(d, rd); break;
    default: k_lincomb<T, MI, MO, 3><<<g, kThreads, 0, st>>>(d, rd); break;
  }
}

template <typename T>
static void lc_dispatch(const LcH<T>& d, const RedH& rd, cudaStream_t st) {
  if (d.nin <= 4 && d.nout <= 2) lc_nd<T, 4, 2>(d, rd, st);
  else if (d.nin <= 8 && d.nout <= 4) lc_nd<T, 8, 4>(d, rd, st);
  else if (d.nout <= 4) lc_nd<T, 24, 4>(d, rd, st);
  else if (d.nin <= 16) lc_nd<T, 16, 6>(d, rd, st);
  else lc_nd<T, 24, 6>(d, rd, st);
}

void launch_lincomb_d(const LcH<double>& d, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  lc_dispatch<double>(d, rd, st);
}
void launch_lincomb_f(const LcH<float>& d, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  lc_dispatch<float>(d, rd, st);
}

// ------------------------------------------------------ pairwise Gram

template <typename T>
static void gram_dispatch(const GramH<T>& g, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  const int gr = grid_for(g.n / Pack<T>::N);
  switch (g.m) {
    case 2: k_gram_vec<T, 2><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 3: k_gram_vec<T, 3><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 4: k_gram_vec<T, 4><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 5: k_gram_vec<T, 5><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 6: k_gram_vec<T, 6><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 7: k_gram_vec<T, 7><<<gr, kThreads, 0, st>>>(g, rd); break;
    case 8: k_gram_vec<T, 8><<<gr, kThreads, 0, st>>>(g, rd); break;
    default: k_gram_vec<T, 9><<<gr, kThreads, 0, st>>>(g, rd); break;
  }
}
void launch_gram_d(const GramH<double>& g, const RedH& rd, cudaStream_t st) {
  gram_dispatch<double>(g, rd, st);
}
void launch_gram_f(const GramH<float>& g, const RedH& rd, cudaStream_t st) {
  gram_dispatch<float>(g, rd, st);
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
  ++launch_count();
  k_convert_d2f<<<grid_for(n), kThreads, 0, st>>>(a, b, n);
}
void launch_convert_f2d(const float* a, double* b, long long n, cudaStream_t st) {
  ++launch_count();
  k_convert_f2d<<<grid_for(n), kThreads, 0, st>>>(a, b, n);
}

// ------------------------------------------------------- shifted methods

void launch_shift(const ShiftArgsH& a, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  ShiftArgs s{a.r, a.p, a.x, a.xs, a.ps, a.np, a.ns, a.l, a.j, a.mode};
  const int g = grid_for(a.np);
  switch (a.mode) {
    case 0: k_shift<0><<<g, kThreads, 0, st>>>(s, rd); break;
    case 1: k_shift<1><<<g, kThreads, 0, st>>>(s, rd); break;
    case 2: k_shift<2><<<g, kThreads, 0, st>>>(s, rd); break;
    default: k_shift<3><<<g, kThreads, 0, st>>>(s, rd); break;
  }
}

// --------------------------------------------------------- block methods

void launch_spmm(const CsrH& A, const SpmmH& a, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  SpmmArgs s{a.X, a.Y, a.C, a.W, a.alpha, a.mode, a.s, a.nd};
  const int g = grid_for((long long)A.n * kBlkS);
  switch (a.nd) {
    case 0: k_spmm<0><<<g, kThreads, 0, st>>>(A, s, rd); break;
    case 1: k_spmm<1><<<g, kThreads, 0, st>>>(A, s, rd); break;
    default: k_spmm<2><<<g, kThreads, 0, st>>>(A, s, rd); break;
  }
}

void launch_block(const BlkH& a, const RedH& rd, cudaStream_t st) {
  ++launch_count();
  BlkArgs b;
  static_assert(sizeof(BlkArgs) == sizeof(BlkH), "BlkArgs layout");
  memcpy(&b, &a, sizeof(b));
  const long long tiles = (a.n + kBlkTileRows - 1) / kBlkTileRows;
  int g = (int)(tiles < kMaxBlocks ? tiles : kMaxBlocks);
  if (g < 1) g = 1;
  k_block<<<g, kThreads, 0, st>>>(b, rd);
}

// Column-major n x s (leading dimension n) <-> row-major np x s.
__global__ void k_cm2rm(const double* __restrict__ cm, double* __restrict__ rm,
                        int n, int s) {
  const long long tot = (long long)n * s;
  for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < tot;
       q += (long long)gridDim.x * kThreads) {
    const long long i = q / s, c = q % s;
    rm[q] = cm[c * n + i];
  }
}
__global__ void k_rm2cm(const double* __restrict__ rm, double* __restrict__ cm,
                        int n, int s) {
  const long long tot = (long long)n * s;
  for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < tot;
       q += (long long)gridDim.x * kThreads) {
    const long long c = q / n, i = q % n;
    cm[q] = rm[i * s + c];
  }
}
void launch_cm2rm(const double* cm, double* rm, int n, int s, cudaStream_t st) {
  ++launch_count();
  k_cm2rm<<<grid_for((long long)n * s), kThreads, 0, st>>>(cm, rm, n, s);
}
void launch_rm2cm(const double* rm, double* cm, int n, int s, cudaStream_t st) {
  ++launch_count();
  k_rm2cm<<<grid_for((long long)n * s), kThreads, 0, st>>>(rm, cm, n, s);
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
  ++launch_count();
  const int g = grid_for(n);
  if (nd)
    k_mx_d2f<1><<<g, kThreads, 0, st>>>(in, o0, o1, o2, w, n, rd);
  else
    k_mx_d2f<0><<<g, kThreads, 0, st>>>(in, o0, o1, o2, w, n, rd);
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
  ++launch_count();
  k_mx_accum<<<grid_for(n), kThreads, 0, st>>>(x, t, y, n, rd);
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

__global__ void k_set_scalar(double* S, short slot, double v) { S[slot] = v; }

void launch_set_scalar(double* S, short slot, double v, cudaStream_t st) {
  ++launch_count();
  k_set_scalar<<<1, 1, 0, st>>>(S, slot, v);
}

__global__ void k_epilogue(Red rd) {
  if (skip(rd)) return;
  run_epilogue(rd);
}

void launch_epilogue(const RedH& rd, cudaStream_t st) {
  ++launch_count();
  k_epilogue<<<1, 1, 0, st>>>(rd);
}

// Body-final node of a solve's CUDA-graph while loop.  The loop ends when a
// convergence test has finished the solve, and in any case after trip_cap
// trips: the cap is checked here, independently of the method's epilogues,
// so a device-side loop can never outlive its iteration budget.
__global__ void k_loop_control(Ctl* c, cudaGraphConditionalHandle h,
                               int use_handle) {
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
  ++launch_count();
  k_loop_control<<<1, 1, 0, st>>>(ctl, (cudaGraphConditionalHandle)handle,
                                  use_handle);
}

}  // namespace bk
