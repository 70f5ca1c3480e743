// Shifted-method and block-method kernels and their launch wrappers
// (kernel_api.h).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_shift.cuh"
#include "k_block.cuh"
#include "kernel_api.h"
#include "launch_util.h"

namespace bk {

// ------------------------------------------------------- shifted methods

void launch_shift(const ShiftArgsH& a, const RedH& rd, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("block / shifted kernel");
  ++launch_count();
  if (a.ps32) {
    ShiftArgs<float> s{a.r, a.p, a.x, a.xs, a.ps32, a.np, a.ns, a.l, a.j, a.mode};
    switch (a.mode) {
      case 0: launch_k(k_shift<0, float>, grid_wave(k_shift<0, float>, a.np), kThreads, 0, st, s, rd); break;
      case 1: launch_k(k_shift<1, float>, grid_wave(k_shift<1, float>, a.np), kThreads, 0, st, s, rd); break;
      case 2: launch_k(k_shift<2, float>, grid_wave(k_shift<2, float>, a.np), kThreads, 0, st, s, rd); break;
      default: launch_k(k_shift<3, float>, grid_wave(k_shift<3, float>, a.np), kThreads, 0, st, s, rd); break;
    }
    return;
  }
  ShiftArgs<double> s{a.r, a.p, a.x, a.xs, a.ps, a.np, a.ns, a.l, a.j, a.mode};
  switch (a.mode) {
    case 0: launch_k(k_shift<0, double>, grid_wave(k_shift<0, double>, a.np), kThreads, 0, st, s, rd); break;
    case 1: launch_k(k_shift<1, double>, grid_wave(k_shift<1, double>, a.np), kThreads, 0, st, s, rd); break;
    case 2: launch_k(k_shift<2, double>, grid_wave(k_shift<2, double>, a.np), kThreads, 0, st, s, rd); break;
    default: launch_k(k_shift<3, double>, grid_wave(k_shift<3, double>, a.np), kThreads, 0, st, s, rd); break;
  }
}

// --------------------------------------------------------- block methods

// BKSP_GPU_SPMM=csr forces the CSR kernel (for comparisons).
static bool spmm_dia_off() {
  static const bool off = [] {
    const char* e = std::getenv("BKSP_GPU_SPMM");
    return e && std::strcmp(e, "csr") == 0;
  }();
  return off;
}

// SpMM autotuner: for an operator with a diagonal form, the faster of the
// diagonal-form and CSR kernels per (rows, entries, s, precision, device),
// timed once outside any stream capture (spmm_autotune) and cached; the two
// give bit-identical results.  Until a choice exists, the diagonal form.
namespace {
struct SpmmKey {
  int n, nnz, s, prec, dev;
  bool operator==(const SpmmKey& o) const {
    return n == o.n && nnz == o.nnz && s == o.s && prec == o.prec && dev == o.dev;
  }
};
std::mutex g_spmm_mu;
std::vector<std::pair<SpmmKey, int>> g_spmm_choice;   // 0 diagonal form, 1 CSR
thread_local int g_spmm_force = -1;                     // set while timing

int spmm_cached(const CsrH& A, int s, int prec) {
  int dev = 0;
  cudaGetDevice(&dev);
  const SpmmKey key{A.n, A.nnz, s, prec, dev};
  std::lock_guard<std::mutex> lk(g_spmm_mu);
  for (const auto& kv : g_spmm_choice)
    if (kv.first == key) return kv.second;
  return -1;
}
}  // namespace

void spmm_force(int kernel) { g_spmm_force = kernel; }

void spmm_autotune(const CsrH& A, int s, int prec, cudaStream_t st) {
  if (A.dia.nd == 0 || spmm_dia_off() || A.n < (1 << 14)) return;
  const char* e = std::getenv("BKSP_GPU_AUTOTUNE");
  if (e && std::strcmp(e, "0") == 0) return;
  if (spmm_cached(A, s, prec) >= 0) return;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t w = prec == 1 ? sizeof(float) : sizeof(double);
  const size_t bytes = (size_t)A.n * (size_t)s * w;
  void *X = nullptr, *Y = nullptr;
  CtlH* ctl = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float best[2] = {1e30f, 1e30f};
  bool ok = cudaMallocAsync(&X, bytes, st) == cudaSuccess &&
            cudaMallocAsync(&Y, bytes, st) == cudaSuccess &&
            cudaMallocAsync(reinterpret_cast<void**>(&ctl), sizeof(CtlH), st) == cudaSuccess &&
            cudaMemsetAsync(X, 0, bytes, st) == cudaSuccess &&
            cudaMemsetAsync(ctl, 0, sizeof(CtlH), st) == cudaSuccess &&
            cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  if (ok) {
    SpmmH a{};
    a.X = static_cast<const double*>(X);
    a.Y = static_cast<double*>(Y);
    a.alpha = 1.0;
    a.s = s;
    a.prec = prec;
    const RedH rd{nullptr, nullptr, nullptr, ctl, 0, 0, 0, 0, 0};
    const long long l0 = launch_count();
    for (int round = 0; round < 2 && ok; ++round)
      for (int v = 0; v < 2 && ok; ++v) {
        g_spmm_force = v;
        launch_spmm(A, a, rd, st);
        ok = cudaEventRecord(e0, st) == cudaSuccess;
        for (int r = 0; r < 5; ++r) launch_spmm(A, a, rd, st);
        ok = ok && cudaEventRecord(e1, st) == cudaSuccess &&
             cudaEventSynchronize(e1) == cudaSuccess;
        float ms = 0.f;
        if (ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
          best[v] = std::min(best[v], ms);
      }
    g_spmm_force = -1;
    launch_count() = l0;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (X) cudaFreeAsync(X, st);
  if (Y) cudaFreeAsync(Y, st);
  if (ctl) cudaFreeAsync(ctl, st);
  cudaGetLastError();
  if (!ok) return;
  const int choice = best[1] < 0.98f * best[0] ? 1 : 0;   // CSR only if clearly faster
  std::lock_guard<std::mutex> lk(g_spmm_mu);
  g_spmm_choice.push_back({SpmmKey{A.n, A.nnz, s, prec, dev}, choice});
}

void launch_spmm(const CsrH& A, const SpmmH& a, const RedH& rd, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("block / shifted kernel");
  ++launch_count();
  // Diagonal form: 16-byte row segments (s a multiple of the vector width,
  // aligned blocks) unless the autotuner found the CSR kernel faster; else
  // the CSR kernel.
  auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  const int vn = a.prec == 1 ? 4 : 2;
  const int pick = g_spmm_force >= 0 ? g_spmm_force
                                     : (A.dia.nd > 0 ? spmm_cached(A, a.s, a.prec) : 1);
  if (A.dia.nd > 0 && a.s % vn == 0 && al(a.X) && al(a.Y) && al(a.C) && al(a.W) &&
      !spmm_dia_off() && pick != 1) {
    const long long rows = A.n;
    const long long per = kThreads / (a.s / vn);
    const long long items = rows * (a.s / vn);
    if (a.prec == 1) {
      SpmmArgs<float> s{reinterpret_cast<const float*>(a.X), reinterpret_cast<float*>(a.Y),
                        reinterpret_cast<const float*>(a.C), reinterpret_cast<const float*>(a.W),
                        a.alpha, a.mode, a.s, a.nd, a.prec};
      switch (a.nd) {
        case 0: launch_k(k_spmm_dia<float, 0>, grid_wave(k_spmm_dia<float, 0>, items), kThreads, 0, st, A, s, rd); break;
        case 1: launch_k(k_spmm_dia<float, 1>, grid_wave(k_spmm_dia<float, 1>, items), kThreads, 0, st, A, s, rd); break;
        default: launch_k(k_spmm_dia<float, 2>, grid_wave(k_spmm_dia<float, 2>, items), kThreads, 0, st, A, s, rd); break;
      }
    } else {
      SpmmArgs<double> s{a.X, a.Y, a.C, a.W, a.alpha, a.mode, a.s, a.nd, a.prec};
      switch (a.nd) {
        case 0: launch_k(k_spmm_dia<double, 0>, grid_wave(k_spmm_dia<double, 0>, items), kThreads, 0, st, A, s, rd); break;
        case 1: launch_k(k_spmm_dia<double, 1>, grid_wave(k_spmm_dia<double, 1>, items), kThreads, 0, st, A, s, rd); break;
        default: launch_k(k_spmm_dia<double, 2>, grid_wave(k_spmm_dia<double, 2>, items), kThreads, 0, st, A, s, rd); break;
      }
    }
    (void)per;
    return;
  }
  const int g = grid_for((long long)A.n * kBlkS);
  if (a.prec == 1) {
    SpmmArgs<float> s{reinterpret_cast<const float*>(a.X), reinterpret_cast<float*>(a.Y),
                      reinterpret_cast<const float*>(a.C), reinterpret_cast<const float*>(a.W),
                      a.alpha, a.mode, a.s, a.nd, a.prec};
    switch (a.nd) {
      case 0: launch_k(k_spmm<float, 0>, g, kThreads, 0, st, A, s, rd); break;
      case 1: launch_k(k_spmm<float, 1>, g, kThreads, 0, st, A, s, rd); break;
      default: launch_k(k_spmm<float, 2>, g, kThreads, 0, st, A, s, rd); break;
    }
    return;
  }
  SpmmArgs<double> s{a.X, a.Y, a.C, a.W, a.alpha, a.mode, a.s, a.nd, a.prec};
  switch (a.nd) {
    case 0: launch_k(k_spmm<double, 0>, g, kThreads, 0, st, A, s, rd); break;
    case 1: launch_k(k_spmm<double, 1>, g, kThreads, 0, st, A, s, rd); break;
    default: launch_k(k_spmm<double, 2>, g, kThreads, 0, st, A, s, rd); break;
  }
}

void launch_block(const BlkH& a, const RedH& rd, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("block / shifted kernel");
  ++launch_count();
  static_assert(sizeof(BlkArgs<double>) == sizeof(BlkH), "BlkArgs layout");
  static_assert(sizeof(BlkArgs<float>) == sizeof(BlkH), "BlkArgs layout");
  const long long tiles = (a.n + kBlkTileRows - 1) / kBlkTileRows;
  if (a.prec == 1) {
    BlkArgs<float> b;
    memcpy(&b, &a, sizeof(b));
    const int cap = resident_grid(reinterpret_cast<const void*>(k_block<float>));
    int g = (int)(tiles < cap ? tiles : cap);
    launch_k(k_block<float>, g < 1 ? 1 : g, kThreads, 0, st, b, rd);
    return;
  }
  BlkArgs<double> b;
  memcpy(&b, &a, sizeof(b));
  const int cap = resident_grid(reinterpret_cast<const void*>(k_block<double>));   // one wave
  int g = (int)(tiles < cap ? tiles : cap);
  launch_k(k_block<double>, g < 1 ? 1 : g, kThreads, 0, st, b, rd);
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

}  // namespace bk
