// SpMV kernels (every variant) and their launch wrappers (kernel_api.h),
// plus the CSR -> diagonal-form scatter.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_spmv.cuh"
#include "k_spmv_tma.cuh"
#include "k_spmv_vec.cuh"
#include "k_spmv_wtile.cuh"
#include "k_spmv_dia.cuh"
#include "k_spmv_sell.cuh"
#include "kernel_api.h"
#include "launch_util.h"

namespace bk {

// ------------------------------------------------------------------ SpMV

// SpMV kernel variants (every one sums a row in the reference's order):
//   0 tile (register-staged products), 1 tile with TMA bulk copies,
//   2..5 vector CSR with 4, 8, 16, 32 lanes per row, 6 warp tile,
//   7 diagonal form (operators that have one; else the tile kernel),
//   8 sliced ELL (operators that have the copy; else the tile kernel).
// CsrH.variant carries the choice made for the operator (autotuner);
// BKSP_GPU_SPMV=tile|tma|vec4|vec8|vec16|vec32|wtile|dia|sell overrides it.
static int parse_spmv_override() {
  const char* e = std::getenv("BKSP_GPU_SPMV");
  if (!e) return -1;
  const std::string s(e);
  if (s == "tile") return 0;
  if (s == "tma") return 1;
  if (s == "vec4") return 2;
  if (s == "vec8") return 3;
  if (s == "vec16") return 4;
  if (s == "vec32") return 5;
  if (s == "wtile") return 6;
  if (s == "dia") return 7;
  if (s == "sell") return 8;
  return -1;
}
static int spmv_override() {
  static const int v = parse_spmv_override();   // thread-safe initialisation
  return v;
}

template <typename VT, typename XT, int L>
static void spmv_vec_launch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                            cudaStream_t st) {
  long long g = ((long long)A.n * L + kThreads - 1) / kThreads;
  if (g > kMaxBlocks) g = kMaxBlocks;
  if (g < 1) g = 1;
  switch (io.nd) {
    case 0: launch_k(k_spmv_vec<VT, XT, 0, L>, (int)g, kThreads, 0, st, A, io, rd); break;
    case 1: launch_k(k_spmv_vec<VT, XT, 1, L>, (int)g, kThreads, 0, st, A, io, rd); break;
    case 2: launch_k(k_spmv_vec<VT, XT, 2, L>, (int)g, kThreads, 0, st, A, io, rd); break;
    default: launch_k(k_spmv_vec<VT, XT, 3, L>, (int)g, kThreads, 0, st, A, io, rd); break;
  }
}

template <typename VT, typename XT, int ND>
static void spmv_tma_launch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                            cudaStream_t st) {
  const size_t sm = 2 * (size_t)kStageEnt * (sizeof(int) + sizeof(VT));
  // The shared-memory attribute is per device: set it once on each.
  static std::mutex mu;
  static unsigned long long devs_set = 0;
  static int per_sm = 1;
  int dev = 0;
  cudaGetDevice(&dev);
  int blocks_per_sm = 1;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && !((devs_set >> dev) & 1ull)) {
      cudaFuncSetAttribute(k_spmv_tma<VT, XT, ND>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      int b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_spmv_tma<VT, XT, ND>,
                                                    kThreads, sm);
      per_sm = b < 1 ? 1 : b;
      devs_set |= 1ull << dev;
    }
    blocks_per_sm = per_sm;
  }
  int g = kSMs * blocks_per_sm;
  if (g > kMaxBlocks) g = kMaxBlocks;
  if (g > A.nrb) g = A.nrb > 0 ? A.nrb : 1;
  launch_k(k_spmv_tma<VT, XT, ND>, g, kThreads, sm, st, A, io, rd);
}

static inline bool aligned16(const void* p) {
  return ((uintptr_t)p & 15u) == 0;
}

// The diagonal kernel stores y and loads x, b, w0, w1 as 16-byte packets.
template <typename XT>
static bool dia_usable(const CsrH& A, const SpmvH<XT>& io) {
  return A.dia.nd > 0 && aligned16(io.x) && aligned16(io.y) &&
         aligned16(io.y2) && aligned16(io.b) && aligned16(io.w0) &&
         aligned16(io.w1);
}

template <typename VT, typename XT>
static void spmv_dia_launch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                            cudaStream_t st) {
  const long long groups = ((long long)A.n + 3) / 4;   // 4 rows per thread
  switch (io.nd) {
    case 0: launch_k(k_spmv_dia<VT, XT, 0>, grid_wave(k_spmv_dia<VT, XT, 0>, groups), kThreads, 0, st, A, io, rd); break;
    case 1: launch_k(k_spmv_dia<VT, XT, 1>, grid_wave(k_spmv_dia<VT, XT, 1>, groups), kThreads, 0, st, A, io, rd); break;
    case 2: launch_k(k_spmv_dia<VT, XT, 2>, grid_wave(k_spmv_dia<VT, XT, 2>, groups), kThreads, 0, st, A, io, rd); break;
    default: launch_k(k_spmv_dia<VT, XT, 3>, grid_wave(k_spmv_dia<VT, XT, 3>, groups), kThreads, 0, st, A, io, rd); break;
  }
}

// Algorithmic bytes of one product: the matrix as the chosen format stores
// it (diagonal form: nd values and a mask byte per row; CSR: values, column
// indices and row pointers) and each vector operand once.
template <typename VT, typename XT>
static long long spmv_bytes(const CsrH& A, const SpmvH<XT>& io, bool dia) {
  const long long n = A.n;
  const long long mat = dia ? n * ((long long)A.dia.nd * (long long)sizeof(VT) + 1)
                            : (long long)A.nnz * (long long)(sizeof(VT) + 4) + 4 * (n + 1);
  const int vecs = 2 + (io.y2 != nullptr) + (io.mode == 1 && io.b != nullptr) +
                   (io.w0 != nullptr) + (io.w1 != nullptr);
  return mat + vecs * n * (long long)sizeof(XT);
}

// Persistent-loop form of one product: the diagonal form where the
// stand-alone launch would use it, else the one-thread-per-row CSR unit.
template <typename VT, typename XT>
static void spmv_record(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                        int var) {
  if (io.nd > 3) prog_unsupported("spmv with more than three dots");
  ProgOpH op;
  std::memset(&op, 0, sizeof(op));
  const bool dia = var == 7 && dia_usable(A, io);
  byte_count() += spmv_bytes<VT, XT>(A, io, dia);
  if constexpr (sizeof(XT) == 8) {
    op.kind = dia ? kOpSpmvDiaD : kOpSpmvCsrD;
    op.u.sd.A = A;
    op.u.sd.io = io;
  } else {
    op.kind = dia ? kOpSpmvDiaF : kOpSpmvCsrF;
    op.u.sf.A = A;
    op.u.sf.io = io;
  }
  op.units = prog_units(A.n);
  op.rd = rd;
  prog_push(op);
}

template <typename VT, typename XT>
static void spmv_dispatch(const CsrH& A, const SpmvH<XT>& io, const RedH& rd,
                          cudaStream_t st) {
  int var = spmv_override();
  if (var < 0) var = A.variant;
  if (g_prog_rec) {
    if (io.shift != 0.0) prog_unsupported("shifted product");
    spmv_record<VT, XT>(A, io, rd, var);
    return;
  }
  // A shifted product runs on the diagonal-form or tile kernel only.
  if (io.shift != 0.0 && var != 7) var = 0;
  if (var == 7) {
    if (dia_usable(A, io)) {
      byte_count() += spmv_bytes<VT, XT>(A, io, true);
      spmv_dia_launch<VT, XT>(A, io, rd, st);
      return;
    }
    var = 0;
  }
  byte_count() += spmv_bytes<VT, XT>(A, io, false);
  if (var == 8 && A.sell.nslice > 0) {
    const long long threads = (long long)A.sell.nslice * 32;
    switch (io.nd) {
      case 0: launch_k(k_spmv_sell<VT, XT, 0>, grid_wave(k_spmv_sell<VT, XT, 0>, threads), kThreads, 0, st, A, io, rd); return;
      case 1: launch_k(k_spmv_sell<VT, XT, 1>, grid_wave(k_spmv_sell<VT, XT, 1>, threads), kThreads, 0, st, A, io, rd); return;
      case 2: launch_k(k_spmv_sell<VT, XT, 2>, grid_wave(k_spmv_sell<VT, XT, 2>, threads), kThreads, 0, st, A, io, rd); return;
      default: launch_k(k_spmv_sell<VT, XT, 3>, grid_wave(k_spmv_sell<VT, XT, 3>, threads), kThreads, 0, st, A, io, rd); return;
    }
  }
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
        case 0: launch_k(k_spmv_wtile<VT, XT, 0>, g, kThreads, 0, st, A, io, rd); return;
        case 1: launch_k(k_spmv_wtile<VT, XT, 1>, g, kThreads, 0, st, A, io, rd); return;
        case 2: launch_k(k_spmv_wtile<VT, XT, 2>, g, kThreads, 0, st, A, io, rd); return;
        default: launch_k(k_spmv_wtile<VT, XT, 3>, g, kThreads, 0, st, A, io, rd); return;
      }
    }
    default: break;
  }
  const int g = A.nrb < kMaxBlocks ? (A.nrb > 0 ? A.nrb : 1) : kMaxBlocks;
  switch (io.nd) {
    case 0: launch_k(k_spmv<VT, XT, 0>, g, kThreads, 0, st, A, io, rd); break;
    case 1: launch_k(k_spmv<VT, XT, 1>, g, kThreads, 0, st, A, io, rd); break;
    case 2: launch_k(k_spmv<VT, XT, 2>, g, kThreads, 0, st, A, io, rd); break;
    default: launch_k(k_spmv<VT, XT, 3>, g, kThreads, 0, st, A, io, rd); break;
  }
}

void launch_spmv_d(const CsrH& A, const SpmvH<double>& io, const RedH& rd,
                   cudaStream_t st) {
  if (!g_prog_rec) ++launch_count();
  spmv_dispatch<double, double>(A, io, rd, st);
}
void launch_spmv_f(const CsrH& A, const SpmvH<float>& io, const RedH& rd,
                   cudaStream_t st) {
  if (!g_prog_rec) ++launch_count();
  spmv_dispatch<float, float>(A, io, rd, st);
}

// ------------------------------------------------- fused diagonal product

template <typename T>
static bool fused_usable(const CsrH& A, const SpmvFuseH<T>& f) {
  return A.dia.nd > 0 && f.nd <= 3 && aligned16(f.xa) && aligned16(f.xb) &&
         aligned16(f.xe) && aligned16(f.y) && aligned16(f.f0) &&
         aligned16(f.f1) && aligned16(f.fo) && f.xa && f.y;
}
bool spmv_fused_usable_d(const CsrH& A, const SpmvFuseH<double>& f) {
  return fused_usable(A, f);
}
bool spmv_fused_usable_f(const CsrH& A, const SpmvFuseH<float>& f) {
  return fused_usable(A, f);
}

template <typename T>
static void spmv_fused_launch(const CsrH& A, const SpmvFuseH<T>& f, const RedH& rd,
                              cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("fused product");
  ++launch_count();
  const long long n = A.n;
  // Diagonal values and masks, the input vectors, the product, the stored
  // own x and the second update's operands, each once.
  const int vecs = 2 + (f.xb != nullptr) + (f.xe != nullptr) +
                   (f.fo != nullptr) * (1 + (f.f0 != nullptr) + (f.f1 != nullptr));
  byte_count() += n * ((long long)A.dia.nd * (long long)sizeof(T) + 1) +
                  vecs * n * (long long)sizeof(T);
  const long long groups = (n + 3) / 4;
  switch (f.nd) {
    case 0: launch_k(k_spmv_dia_fused<T, 0>, grid_wave(k_spmv_dia_fused<T, 0>, groups), kThreads, 0, st, A, f, rd); break;
    case 1: launch_k(k_spmv_dia_fused<T, 1>, grid_wave(k_spmv_dia_fused<T, 1>, groups), kThreads, 0, st, A, f, rd); break;
    case 2: launch_k(k_spmv_dia_fused<T, 2>, grid_wave(k_spmv_dia_fused<T, 2>, groups), kThreads, 0, st, A, f, rd); break;
    default: launch_k(k_spmv_dia_fused<T, 3>, grid_wave(k_spmv_dia_fused<T, 3>, groups), kThreads, 0, st, A, f, rd); break;
  }
}

void launch_spmv_fused_d(const CsrH& A, const SpmvFuseH<double>& f,
                         const RedH& rd, cudaStream_t st) {
  spmv_fused_launch<double>(A, f, rd, st);
}
void launch_spmv_fused_f(const CsrH& A, const SpmvFuseH<float>& f,
                         const RedH& rd, cudaStream_t st) {
  spmv_fused_launch<float>(A, f, rd, st);
}

// CSR values, columns and row pointers read; nd diagonals (and masks) written.
template <typename T>
static long long csr2dia_bytes(const CsrH& A, bool mask) {
  const long long n = A.n;
  return (long long)A.nnz * (long long)(sizeof(T) + 4) + 4 * (n + 1) +
         n * (long long)A.dia.nd * (long long)sizeof(T) + (mask ? n : 0);
}

void launch_csr2dia_d(const CsrH& A, const double* val, double* dval,
                      unsigned char* mask, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("csr2dia");
  ++launch_count();
  byte_count() += csr2dia_bytes<double>(A, mask != nullptr);
  launch_k(k_csr2dia<double>, (A.n + 255) / 256, 256, 0, st, A, val, dval, mask);
}
void launch_csr2dia_f(const CsrH& A, const float* val, float* dval,
                      unsigned char* mask, cudaStream_t st) {
  if (g_prog_rec) prog_unsupported("csr2dia");
  ++launch_count();
  byte_count() += csr2dia_bytes<float>(A, mask != nullptr);
  launch_k(k_csr2dia<float>, (A.n + 255) / 256, 256, 0, st, A, val, dval, mask);
}

void launch_csr2sell_d(const int* rowptr, const int* col, const double* val,
                       int n, int nslice, const int* sptr, int* scol,
                       double* sval, cudaStream_t st) {
  const long long rows = (long long)nslice * 32;
  k_csr2sell<double><<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(
      rowptr, col, val, n, nslice, sptr, scol, sval);
}
void launch_csr2sell_f(const int* rowptr, const int* col, const float* val,
                       int n, int nslice, const int* sptr, int* scol,
                       float* sval, cudaStream_t st) {
  const long long rows = (long long)nslice * 32;
  k_csr2sell<float><<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(
      rowptr, col, val, n, nslice, sptr, scol, sval);
}

}  // namespace bk
