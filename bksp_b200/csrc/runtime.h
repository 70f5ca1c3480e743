// Host runtime of the solver library: per-thread device context, stream-
// ordered device allocation, CSR upload, per-solve scalar/control state,
// linear-combination builder and the CUDA-graph iteration loop.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernel_api.h"
#include "solver_defs.h"

namespace bk {

// Any CUDA failure inside the library becomes this exception; the C entry
// points catch it and return INVALID_PARAMETERS.
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what);
#define BK_CHECK(call) ::bk::check((call), #call)

inline long long pad64(long long n) { return (n + 63) / 64 * 64; }

// Per-host-thread library context: device, stream, pinned staging.
struct Ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  bool use_cond_graph = true;   // CUDA-graph while loop (else host polling)
  bool persistent = false;      // iteration loops as persistent launches
  static Ctx& get();
};

// Stream-ordered device allocation from the device's memory pool (freed
// blocks stay cached in the pool for the next solve).
void* dalloc(size_t bytes, cudaStream_t st);
void dfree(void* p, cudaStream_t st);
template <typename T>
T* dalloc_n(long long n, cudaStream_t st) {
  return static_cast<T*>(dalloc(sizeof(T) * (size_t)(n > 0 ? n : 1), st));
}

// Device CSR operator.  Values are kept in FP64 (parity solves, true
// residuals) and, on request, FP32 (mixed-precision inner solves), sharing
// one index structure.
struct DevCsr {
  int n = 0, nnz = 0, nrb = 0;
  int* rowptr = nullptr;
  int* col = nullptr;
  double* v64 = nullptr;
  float* v32 = nullptr;
  int* rb = nullptr;
  int variant = 3;   // SpMV kernel variant chosen for this operator
  // Diagonal form (ndia = 0: none): values per precision, shared row masks.
  int ndia = 0;
  int doff[kDiaMax] = {};
  unsigned char* dmask = nullptr;
  double* d64 = nullptr;
  float* d32 = nullptr;
  bool owns_dmask = true;   // false for views sharing another operator's masks
  // Structure scan at upload (kernel_api.h: CsrScanH), offsets ascending,
  // and the first stored diagonal entry of every row (device, n doubles).
  CsrScanH scan{};
  double* ddiag = nullptr;
  // Sliced-ELL copy (kernel_api.h: SellH) for operators without a diagonal
  // form; nslice = 0: none.
  int nslice = 0;
  int* sptr = nullptr;
  int* scol = nullptr;
  double* s64 = nullptr;
  float* s32 = nullptr;
  CsrH h64() const { return hview(v64, d64); }
  CsrH h32() const { return hview(v32, d32); }
  CsrH hview(const void* v, const void* dv) const {
    CsrH h{rowptr, col, v, rb, n, nrb, variant, DiaH{}, nnz, SellH{}};
    if (nslice > 0 && v && (v == v64 || v == v32)) {
      h.sell.ptr = sptr;
      h.sell.col = scol;
      h.sell.val = v == v64 ? static_cast<const void*>(s64) : static_cast<const void*>(s32);
      h.sell.nslice = h.sell.val ? nslice : 0;
    }
    if (ndia > 0 && dv) {
      h.dia.val = dv;
      h.dia.mask = dmask;
      h.dia.stride = pad64(n);
      h.dia.nd = ndia;
      for (int d = 0; d < kDiaMax; ++d) h.dia.off[d] = doff[d];
    }
    return h;
  }
  void release(cudaStream_t st);
};

// Host-side CSR (0-based, int32).
struct HostCsr {
  int n = 0;
  std::vector<int> rowptr, col;
  std::vector<double> val;
};

// Mirror every stored off-diagonal entry (a "symmetric" bksp matrix stores
// one triangle; reference src/matvec.c:100-127).  Rows come out sorted by
// column.
HostCsr expand_symmetric(int n, const int* rowptr, const int* col,
                         const double* val);
// A^T in CSR; entries of each row ordered by the original row index, which
// reproduces the summation order of the reference's scatter A^T x
// (src/matvec.c:29-45).
HostCsr transpose(int n, const int* rowptr, const int* col, const double* val);

// Upload a host CSR (rows in the caller's order), scan its structure on the
// GPU (columns in range -- else CudaError --, diagonal offsets, diagonal),
// build its row blocks and, when it has one, its diagonal form.
void upload_csr(int n, const int* rowptr, const int* col, const double* val,
                bool want_fp32, DevCsr& out, cudaStream_t st,
                bool cv_on_device = false);   // col, val already in GPU memory

// Pick the fastest SpMV kernel variant for A by timing them (cached per
// operator signature); called by upload_csr for large operators.
void autotune_spmv(DevCsr& A, cudaStream_t st);

// Row-block partition used by the SpMV tile kernels.
std::vector<int> make_row_blocks(int n, const int* rowptr);

// Per-solve device state: scalar slots, control block, reduction scratch,
// optional residual history.
struct SolveState {
  double* S = nullptr;
  CtlH* ctl = nullptr;
  double* part = nullptr;
  unsigned* ticket = nullptr;
  double* hist = nullptr;
  int hist_cap = 0;
  CtlH* ctl_free = nullptr;   // a control block that is never finished
  // Conditional block of the captured iteration (cond_block): its handle
  // and the kernels it holds, valid for the solve being captured.
  bool has_cond = false;
  int n_cond = 0;                       // conditional nodes in the body
  unsigned long long cond_handle[2] = {0, 0};
  long long cond_kernels = 0;           // kernels of all of them
  long long cond_bytes = 0;   // their algorithmic bytes (byte_count)
  cudaStream_t side = nullptr;   // capture stream of the conditional body
  void create(int hist_cap, cudaStream_t st);
  void release(cudaStream_t st);
  // Reset control: iteration index starts at iter0, budget max_iter.
  void start(int iter0, int max_iter, double tol, cudaStream_t st);
  RedH red(short out, short epi, short a0 = 0, short a1 = 0) const {
    return RedH{part, ticket, S, ctl, out, epi, a0, a1, 0};
  }
  // For launches after the iteration loop (not skipped by `done`).
  RedH red_after(short out, short epi) const {
    return RedH{part, ticket, S, ctl_free, out, epi, 0, 0, 0};
  }
  // Same, for a launch that runs only while S[guard] != 0.
  RedH red_if(short guard, short out, short epi, short a0 = 0,
              short a1 = 0) const {
    return RedH{part, ticket, S, ctl, out, epi, a0, a1, guard};
  }
  CtlH read(cudaStream_t st) const;
  void set_scalar(short slot, double v, cudaStream_t st);
  void set_scalars(short slot, const double* host, int count, cudaStream_t st);
  double get_scalar(short slot, cudaStream_t st) const;
};

// Inside the body that run_loop captures: launch `inner`'s kernels in a
// conditional IF node, so they run only in the iterations in which an
// epilogue upstream sets the node's condition (through ctl->cond for the
// body's first node, ctl->cond_alt for a second); in the others no kernel
// is launched at all.  Outside a capture (host-polled loop) inner runs
// directly and its kernels' own guards decide.
void cond_block(SolveState& ss, cudaStream_t st,
                const std::function<void(cudaStream_t)>& inner);

// Builder for one fused linear-combination launch (LcH).
template <typename T>
struct Lc {
  LcH<T> d;
  explicit Lc(long long n) {
    std::memset(&d, 0, sizeof(d));
    d.n = n;
    d.reps = 1;
  }
  static constexpr int OUT = 100;   // dot operand code base for outputs
  int in(const T* p, bool rep = false) {
    if (d.nin >= kLcMaxIn) throw CudaError("lincomb: too many inputs");
    const int i = d.nin++;
    d.in[i] = p;
    if (rep) d.in_rep_mask |= 1u << i;
    return i;
  }
  int out(T* p, bool rep = false) {
    if (d.nout >= kLcMaxOut) throw CudaError("lincomb: too many outputs");
    const int o = d.nout++;
    d.out[o] = p;
    if (rep) d.out_rep_mask |= 1u << o;
    return o;
  }
  Lc& term(int o, int i, CfH c) {
    d.c[o][i] = c;
    return *this;
  }
  // Operands: input index, or OUT + output index.
  Lc& dot(int a, int b) {
    if (d.nd >= 3) throw CudaError("lincomb: too many dots");
    dots_.push_back({a, b});
    d.nd++;
    return *this;
  }
  Lc& batch(int reps, long long stride) {
    d.reps = reps;
    d.stride = stride;
    return *this;
  }
  void launch(const RedH& rd, cudaStream_t st);
 private:
  std::vector<std::pair<int, int>> dots_;
};

// Runs `body` (one iteration's launches) until the solve is done, as a
// CUDA-graph while loop (one graph launch per solve) or, as fallback, by
// host polling.  Returns the final control block.  When the calling thread
// has joined a persistent group (persist_group()), the body is recorded
// instead and runs, with the group's other systems, inside one persistent
// launch; a body that cannot be recorded runs as a graph loop.
CtlH run_loop(SolveState& ss, const std::function<void(cudaStream_t)>& body,
              cudaStream_t st);

// A set of solves whose iteration loops run together in one persistent
// cooperative launch (kernels_persist.cu).  Each member thread runs its
// solve as usual up to run_loop, which records the iteration, hands it to
// the group and waits; the last of `expected` members to arrive (or to
// withdraw) launches the kernel for all of them, after every member's
// set-up work on its own stream.  Every member then continues on its own
// stream with its converged state.
struct PersistGroup {
  explicit PersistGroup(int expected);
  ~PersistGroup();
  PersistGroup(const PersistGroup&) = delete;
  PersistGroup& operator=(const PersistGroup&) = delete;
  // Hand in this member's recorded iteration; returns its control block
  // after the launch (throws CudaError when the launch failed).
  CtlH join(SolveState& ss, std::vector<ProgOpH>& ops, cudaStream_t st);
  // This member will not join (its solve ended before the loop, or its
  // body has no persistent form).
  void withdraw(cudaStream_t st);
  // Launch parameters (set before any member arrives).
  long long spin_limit = 0;   // 0: default
  int absent_cta = -1;        // test hook (PersistH::absent_cta)
  int max_grid = 0;           // 0: every CTA that fits
  // Results.
  int status = 0;             // 0 ok, 1 a barrier wait ran out, 2 launch error
  int grid = 0;               // CTAs launched
  int err_phase = -1;
 private:
  struct Impl;
  Impl* p_;
  void launch_locked(cudaStream_t st);
};
// The group the calling thread's next run_loop joins (null: none); run_loop
// clears it, so one solve joins at most once.
PersistGroup*& persist_group();

// Convenience for SpMV launches.
template <typename T>
SpmvH<T> spmv_io(const T* x, T* y) {
  SpmvH<T> io;
  std::memset(&io, 0, sizeof(io));
  io.x = x;
  io.y = y;
  return io;
}

void spmv(const DevCsr& A, const SpmvH<double>& io, const RedH& rd,
          cudaStream_t st);
void spmv(const DevCsr& A, const SpmvH<float>& io, const RedH& rd,
          cudaStream_t st);

}  // namespace bk
