// Shifted-method and block-method kernels and their launch wrappers
// (kernel_api.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

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

void launch_spmm(const CsrH& A, const SpmmH& a, const RedH& rd, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("block / shifted kernel");
  ++launch_count();
  // Diagonal form: 16-byte row segments (s a multiple of the vector width,
  // aligned blocks); else the CSR kernel.
  auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  const int vn = a.prec == 1 ? 4 : 2;
  if (A.dia.nd > 0 && a.s % vn == 0 && al(a.X) && al(a.Y) && al(a.C) && al(a.W) &&
      !spmm_dia_off()) {
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
