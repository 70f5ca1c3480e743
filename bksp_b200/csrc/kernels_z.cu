// Launch wrappers of the complex kernels (k_zvec.cuh; interface in
// zkernel_api.h).  Complex launches have no persistent-loop form: a
// recording solve falls back to its graph loop.
#include <cstdlib>
#include <cstring>

#include "dev_common.cuh"
#include "k_spmv_sell.cuh"
#include "k_zvec.cuh"
#include "kernel_api.h"
#include "launch_util.h"
#include "runtime.h"
#include "zepilogues.cuh"
#include "zkernel_api.h"

namespace bk {

namespace {

void no_record(const char* what) {
  if (g_prog_rec) prog_unsupported(what);
}

// BKSP_GPU_SPMV=tile keeps the complex product on the tile kernel even
// when the operator has a sliced-ELL copy.
bool zspmv_tile_forced() {
  static const bool v = [] {
    const char* e = std::getenv("BKSP_GPU_SPMV");
    return e && std::strcmp(e, "tile") == 0;
  }();
  return v;
}

}  // namespace

void launch_zlc(const ZLcH& d, const RedH& rd, cudaStream_t st) {
  no_record("complex linear combination");
  if (d.nin > kZLcIn || d.nout > kZLcOut || d.nd > kZDots)
    throw CudaError("complex lincomb: too many operands");
  long long vecs = 0;
  for (int i = 0; i < d.nin; ++i) vecs += (d.in_rep_mask >> i) & 1u ? d.reps : 1;
  for (int o = 0; o < d.nout; ++o) vecs += (d.out_rep_mask >> o) & 1u ? d.reps : 1;
  byte_count() += vecs * d.n * 16;
  ++launch_count();
  if (d.nin <= 4 && d.nout <= 2)
    launch_k(k_zlc<4, 2>, grid_wave(k_zlc<4, 2>, d.n), kThreads, 0, st, d, rd);
  else if (d.nin <= 8 && d.nout <= 4)
    launch_k(k_zlc<8, 4>, grid_wave(k_zlc<8, 4>, d.n), kThreads, 0, st, d, rd);
  else
    launch_k(k_zlc<kZLcIn, kZLcOut>, grid_wave(k_zlc<kZLcIn, kZLcOut>, d.n), kThreads,
             0, st, d, rd);
}

void launch_zspmv(const CsrH& A, const ZSpmvH& io, const RedH& rd,
                  cudaStream_t st) {
  no_record("complex SpMV");
  byte_count() += (long long)A.nnz * 20 + 4LL * (A.n + 1) + 32LL * A.n;
  ++launch_count();
  if (A.sell.nslice > 0 && !zspmv_tile_forced()) {
    const long long threads = (long long)A.sell.nslice * 32;
    switch (io.nd) {
      case 0: launch_k(k_zspmv_sell<0>, grid_wave(k_zspmv_sell<0>, threads), kThreads, 0, st, A, io, rd); return;
      case 1: launch_k(k_zspmv_sell<1>, grid_wave(k_zspmv_sell<1>, threads), kThreads, 0, st, A, io, rd); return;
      case 2: launch_k(k_zspmv_sell<2>, grid_wave(k_zspmv_sell<2>, threads), kThreads, 0, st, A, io, rd); return;
      default: launch_k(k_zspmv_sell<3>, grid_wave(k_zspmv_sell<3>, threads), kThreads, 0, st, A, io, rd); return;
    }
  }
  const int g = A.nrb < kMaxBlocks ? (A.nrb > 0 ? A.nrb : 1) : kMaxBlocks;
  switch (io.nd) {
    case 0: launch_k(k_zspmv<0>, g, kThreads, 0, st, A, io, rd); break;
    case 1: launch_k(k_zspmv<1>, g, kThreads, 0, st, A, io, rd); break;
    case 2: launch_k(k_zspmv<2>, g, kThreads, 0, st, A, io, rd); break;
    default: launch_k(k_zspmv<3>, g, kThreads, 0, st, A, io, rd); break;
  }
}

void launch_zspmm(const CsrH& A, const ZSpmmH& a, const RedH& rd,
                  cudaStream_t st) {
  no_record("complex SpMM");
  if (a.s < 1 || a.s > 16) throw CudaError("complex SpMM: block width out of range");
  byte_count() += (long long)A.nnz * 20 + 32LL * A.n * a.s;
  ++launch_count();
  const long long groups = (long long)A.n * 16;
  launch_k(k_zspmm, grid_wave(k_zspmm, groups), kThreads, 0, st, A, a, rd);
}

void launch_zblock(const ZBlkH& a, const RedH& rd, cudaStream_t st) {
  no_record("complex block kernel");
  if (a.s < 1 || a.s > 16 || a.nin > 4 || a.nout > 2 || a.ng > 2 || a.nd > 2)
    throw CudaError("complex block kernel: bad arguments");
  int nm = 0;
  for (int o = 0; o < a.nout; ++o)
    for (int i = 0; i < a.nin; ++i)
      if (a.c[o][i].op && a.mslot[o][i] >= 0) ++nm;
  if (nm > 2) throw CudaError("complex block kernel: more than two matrix terms");
  byte_count() += 16LL * a.n * a.s * (a.nin + a.nout);
  ++launch_count();
  const long long tiles = (a.n + kZBlkRows - 1) / kZBlkRows;
  launch_k(k_zblock, grid_wave(k_zblock, tiles * kThreads), kThreads, 0, st, a, rd);
}

void launch_csr2sell_z(const int* rowptr, const int* col, const double2* val,
                       int n, int nslice, const int* sptr, int* scol,
                       double2* sval, cudaStream_t st) {
  const long long rows = (long long)nslice * 32;
  k_csr2sell<double2><<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(
      rowptr, col, val, n, nslice, sptr, scol, sval);
}

void launch_zshift(const ZShiftH& a, const RedH& rd, cudaStream_t st) {
  no_record("complex shifted update");
  if (a.ns < 0 || a.ns > kZMaxShifts || a.l < 1 || a.l > kBlMaxL)
    throw CudaError("complex shifted update: bad arguments");
  if (a.ns == 0 && !rd.epi) return;
  byte_count() += 16LL * a.np * (long long)a.ns * (a.mode == 0 ? 2 * (a.j + 2) + 2
                                                   : a.mode == 1 ? 3 : a.l + 3);
  ++launch_count();
  launch_k(k_zshift, grid_wave(k_zshift, a.np), kThreads, 0, st, a, rd);
}

}  // namespace bk
