#include "runtime.h"

#include <algorithm>
#include <cstddef>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <unordered_map>

namespace bk {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    throw CudaError(m);
  }
}

Ctx& Ctx::get() {
  thread_local Ctx cx;
  thread_local bool ready = false;
  if (!ready) {
    BK_CHECK(cudaGetDevice(&cx.device));
    BK_CHECK(cudaStreamCreateWithFlags(&cx.st, cudaStreamNonBlocking));
    const char* loop = std::getenv("BKSP_GPU_LOOP");
    cx.use_cond_graph = !(loop && std::string(loop) == "poll");
    cx.persistent = loop && std::string(loop) == "persist";
    // Keep freed solve buffers cached in the device pool between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, cx.device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    ready = true;
  }
  return cx;
}

void* dalloc(size_t bytes, cudaStream_t st) {
  void* p = nullptr;
  BK_CHECK(cudaMallocAsync(&p, bytes, st));
  return p;
}

void dfree(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

void DevCsr::release(cudaStream_t st) {
  dfree(rowptr, st);
  dfree(col, st);
  dfree(v64, st);
  dfree(v32, st);
  dfree(rb, st);
  dfree(d64, st);
  dfree(d32, st);
  dfree(ddiag, st);
  ddiag = nullptr;
  dfree(sptr, st);
  dfree(scol, st);
  dfree(s64, st);
  dfree(s32, st);
  sptr = scol = nullptr;
  s64 = nullptr;
  s32 = nullptr;
  nslice = 0;
  if (owns_dmask) dfree(dmask, st);
  rowptr = col = rb = nullptr;
  v64 = nullptr;
  v32 = nullptr;
  d64 = nullptr;
  d32 = nullptr;
  dmask = nullptr;
  ndia = 0;
}

HostCsr expand_symmetric(int n, const int* rowptr, const int* col,
                         const double* val) {
  HostCsr h;
  h.n = n;
  std::vector<int> cnt(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      const int j = col[k];
      if (j < 0 || j >= n) throw CudaError("matrix: column index out of range");
      cnt[i]++;
      if (j != i) cnt[j]++;
    }
  h.rowptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) h.rowptr[i + 1] = h.rowptr[i] + cnt[i];
  const int nnz = h.rowptr[n];
  h.col.resize(nnz);
  h.val.resize(nnz);
  std::vector<int> pos(h.rowptr.begin(), h.rowptr.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      const int j = col[k];
      h.col[pos[i]] = j;
      h.val[pos[i]++] = val[k];
      if (j != i) {
        h.col[pos[j]] = i;
        h.val[pos[j]++] = val[k];
      }
    }
  // Sort each row by column.
  std::vector<std::pair<int, double>> tmp;
  for (int i = 0; i < n; ++i) {
    const int a = h.rowptr[i], b = h.rowptr[i + 1];
    bool sorted = true;
    for (int k = a + 1; k < b; ++k)
      if (h.col[k] < h.col[k - 1]) { sorted = false; break; }
    if (sorted) continue;
    tmp.clear();
    for (int k = a; k < b; ++k) tmp.push_back({h.col[k], h.val[k]});
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<int, double>& x,
                        const std::pair<int, double>& y) { return x.first < y.first; });
    for (int k = a; k < b; ++k) {
      h.col[k] = tmp[k - a].first;
      h.val[k] = tmp[k - a].second;
    }
  }
  return h;
}

HostCsr transpose(int n, const int* rowptr, const int* col, const double* val) {
  HostCsr h;
  h.n = n;
  h.rowptr.assign(n + 1, 0);
  const int nnz = rowptr[n];
  for (int k = 0; k < nnz; ++k) {
    if (col[k] < 0 || col[k] >= n) throw CudaError("matrix: column index out of range");
    h.rowptr[col[k] + 1]++;
  }
  for (int i = 0; i < n; ++i) h.rowptr[i + 1] += h.rowptr[i];
  h.col.resize(nnz);
  h.val.resize(nnz);
  std::vector<int> pos(h.rowptr.begin(), h.rowptr.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      const int p = pos[col[k]]++;
      h.col[p] = i;
      h.val[p] = val[k];
    }
  return h;
}

std::vector<int> make_row_blocks(int n, const int* rowptr) {
  std::vector<int> rb;
  rb.reserve(n / 64 + 2);
  rb.push_back(0);
  int rows = 0;
  long long nz = 0;
  for (int i = 0; i < n; ++i) {
    const long long len = rowptr[i + 1] - rowptr[i];
    if (rows > 0 && (rows == kTileRows || nz + len > kTileNnz)) {
      rb.push_back(i);
      rows = 0;
      nz = 0;
    }
    rows++;
    nz += len;
    if (len > kTileNnz) {   // a long row is a block by itself
      rb.push_back(i + 1);
      rows = 0;
      nz = 0;
    }
  }
  if (rows > 0) rb.push_back(n);
  return rb;
}

// The diagonal form is worth keeping when the rows' columns strictly ascend
// (the diagonal order is then each row's CSR summation order), the entries
// lie on at most kDiaMax diagonals and the form moves fewer bytes than CSR
// in FP64 (nd * 8 n + n < 12 nnz + 4 n).
static bool dia_wanted(const CsrScanH& sc, int n, int nnz) {
  if (sc.flags & (kScanUnsorted | kScanManyOffs | kScanBadCol)) return false;
  const int nd = sc.noff;
  return nd > 0 && nd <= kDiaMax &&
         (double)nd * 8.0 * n + n < 12.0 * nnz + 4.0 * n;
}

// Build the diagonal form of an uploaded, scanned operator (values of both
// precisions present, row masks).
static void build_dia(DevCsr& A, cudaStream_t st) {
  const int nd = A.scan.noff;
  const long long stride = pad64(A.n);
  A.ndia = nd;
  for (int d = 0; d < kDiaMax; ++d) A.doff[d] = d < nd ? A.scan.off[d] : 0;
  A.dmask = dalloc_n<unsigned char>(stride, st);
  A.owns_dmask = true;
  A.d64 = dalloc_n<double>(nd * stride, st);
  BK_CHECK(cudaMemsetAsync(A.dmask, 0, stride, st));
  BK_CHECK(cudaMemsetAsync(A.d64, 0, sizeof(double) * nd * stride, st));
  CsrH h = A.hview(A.v64, A.d64);
  launch_csr2dia_d(h, A.v64, A.d64, A.dmask, st);
  BK_CHECK(cudaGetLastError());
  if (A.v32) {
    A.d32 = dalloc_n<float>(nd * stride, st);
    launch_convert_d2f(A.d64, A.d32, nd * stride, st);
    BK_CHECK(cudaGetLastError());
  }
}

// SpMV variant without timing: the diagonal form when there is one, else
// vector CSR with the smallest lane count that covers a typical row.
// Sliced-ELL copy of an uploaded operator without a diagonal form (host
// rowptr: slice widths and offsets; the entries are placed on the GPU).
// Skipped when the padding would exceed half the stored entries or the
// offsets would overflow 32 bits.
static void build_sell(DevCsr& A, const int* rowptr, cudaStream_t st) {
  const int n = A.n;
  const int nslice = (n + 31) / 32;
  std::vector<int> ptr((size_t)nslice + 1, 0);
  long long total = 0;
  for (int s = 0; s < nslice; ++s) {
    int w = 0;
    const int r1 = std::min(n, (s + 1) * 32);
    for (int r = s * 32; r < r1; ++r) w = std::max(w, rowptr[r + 1] - rowptr[r]);
    total += 32LL * w;
    if (total > 0x7fffff00LL) return;
    ptr[s + 1] = (int)total;
  }
  if (total > (long long)A.nnz * 3 / 2 + 64) return;
  A.sptr = dalloc_n<int>(nslice + 1, st);
  A.scol = dalloc_n<int>(total, st);
  A.s64 = dalloc_n<double>(total, st);
  BK_CHECK(cudaMemcpyAsync(A.sptr, ptr.data(), sizeof(int) * (nslice + 1),
                           cudaMemcpyHostToDevice, st));
  launch_csr2sell_d(A.rowptr, A.col, A.v64, n, nslice, A.sptr, A.scol, A.s64, st);
  BK_CHECK(cudaGetLastError());
  if (A.v32) {
    A.s32 = dalloc_n<float>(total, st);
    launch_csr2sell_f(A.rowptr, A.col, A.v32, n, nslice, A.sptr, A.scol, A.s32, st);
    BK_CHECK(cudaGetLastError());
  }
  A.nslice = nslice;
  // ptr (a host vector) must outlive its copy.
  BK_CHECK(cudaStreamSynchronize(st));
}

static int heuristic_variant(int n, int nnz, bool dia) {
  if (dia) return 7;
  const double avg = n > 0 ? (double)nnz / n : 0.0;
  if (avg <= 4.5) return 2;
  if (avg <= 9.0) return 3;
  if (avg <= 18.0) return 4;
  return 5;
}

namespace {
struct TuneKey {
  int n, nnz, dev;
  bool fp32, dia, sell;
  bool operator==(const TuneKey& o) const {
    return n == o.n && nnz == o.nnz && dev == o.dev && fp32 == o.fp32 &&
           dia == o.dia && sell == o.sell;
  }
};
struct TuneHash {
  size_t operator()(const TuneKey& k) const {
    return ((size_t)k.n * 1000003u) ^ ((size_t)k.nnz * 7919u) ^
           ((size_t)k.dev << 2) ^ (size_t)k.fp32 ^ ((size_t)k.dia << 1);
  }
};
std::mutex g_tune_mu;
std::unordered_map<TuneKey, int, TuneHash> g_tune_cache;
}  // namespace

// Autotuner: time every SpMV variant on this operator (FP32 values when
// present, else FP64), keep the fastest; cached per (n, nnz, device,
// precision, diagonal form present).  BKSP_GPU_AUTOTUNE=0 keeps the
// heuristic choice.
void autotune_spmv(DevCsr& A, cudaStream_t st) {
  const char* e = std::getenv("BKSP_GPU_AUTOTUNE");
  if (e && std::string(e) == "0") return;
  int dev = 0;
  cudaGetDevice(&dev);
  const bool f32 = A.v32 != nullptr;
  const TuneKey key{A.n, A.nnz, dev, f32, A.ndia > 0, A.nslice > 0};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      A.variant = it->second;
      return;
    }
  }
  const long long np = pad64(A.n);
  const size_t w = f32 ? sizeof(float) : sizeof(double);
  void* x = dalloc(np * w, st);
  void* y = dalloc(np * w, st);
  BK_CHECK(cudaMemsetAsync(x, 0, np * w, st));
  SolveState ss;
  ss.create(0, st);
  ss.start(0, 1, 0.0, st);
  cudaEvent_t e0, e1;
  BK_CHECK(cudaEventCreate(&e0));
  BK_CHECK(cudaEventCreate(&e1));
  // Three interleaved rounds of 8 launches per candidate; a candidate's
  // time is its best round, so one noisy round cannot decide the choice.
  int cands[8] = {0, 6, 1, 2, 3, 4};
  int kC = 6;
  if (A.ndia > 0) cands[kC++] = 7;
  if (A.nslice > 0) cands[kC++] = 8;
  float best_of[8];
  for (int c = 0; c < kC; ++c) best_of[c] = 1e30f;
  for (int round = 0; round < 3; ++round) {
    for (int c = 0; c < kC; ++c) {
      A.variant = cands[c];
      auto run = [&]() {
        if (f32)
          spmv(A, spmv_io<float>(static_cast<const float*>(x), static_cast<float*>(y)),
               ss.red(kD, E_NONE), st);
        else
          spmv(A, spmv_io<double>(static_cast<const double*>(x), static_cast<double*>(y)),
               ss.red(kD, E_NONE), st);
      };
      run();
      BK_CHECK(cudaEventRecord(e0, st));
      for (int r = 0; r < 8; ++r) run();
      BK_CHECK(cudaEventRecord(e1, st));
      BK_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      BK_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      best_of[c] = std::min(best_of[c], ms);
    }
  }
  // The first candidate (the tile kernel) keeps the job unless another is
  // more than 2% faster.
  int best = cands[0];
  float best_ms = best_of[0];
  for (int c = 1; c < kC; ++c)
    if (best_of[c] < 0.98f * best_ms) {
      best_ms = best_of[c];
      best = cands[c];
    }
  A.variant = best;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ss.release(st);
  dfree(x, st);
  dfree(y, st);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best;
}

void upload_csr(int n, const int* rowptr, const int* col, const double* val,
                bool want_fp32, DevCsr& out, cudaStream_t st, bool cv_on_device) {
  if (n <= 0) throw CudaError("matrix: empty");
  const int nnz = rowptr[n];
  if (rowptr[0] != 0 || nnz < 0) throw CudaError("matrix: bad row pointer");
  const long long padn = (long long)(nnz + 3) / 4 * 4 + 4;
  out.n = n;
  out.nnz = nnz;
  out.rowptr = dalloc_n<int>(n + 1, st);
  out.col = dalloc_n<int>(padn, st);
  out.v64 = dalloc_n<double>(padn, st);
  BK_CHECK(cudaMemsetAsync(out.col, 0, sizeof(int) * padn, st));
  BK_CHECK(cudaMemsetAsync(out.v64, 0, sizeof(double) * padn, st));
  // The copies run (asynchronously from pinned memory) while the host checks
  // the row pointers and builds the row blocks below; nothing on the GPU
  // reads the operator before the check has passed.
  BK_CHECK(cudaMemcpyAsync(out.rowptr, rowptr, sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, st));
  if (nnz > 0) {
    const cudaMemcpyKind kind =
        cv_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    BK_CHECK(cudaMemcpyAsync(out.col, col, sizeof(int) * nnz, kind, st));
    BK_CHECK(cudaMemcpyAsync(out.v64, val, sizeof(double) * nnz, kind, st));
  }
  bool monotone = true;
  for (int i = 0; i < n && monotone; ++i) monotone = rowptr[i + 1] >= rowptr[i];
  if (!monotone) {
    cudaStreamSynchronize(st);   // the copies still read the caller's arrays
    out.release(st);
    throw CudaError("matrix: bad row pointer");
  }
  std::vector<int> rb = make_row_blocks(n, rowptr);
  out.nrb = (int)rb.size() - 1;
  out.rb = dalloc_n<int>((long long)rb.size(), st);
  BK_CHECK(cudaMemcpyAsync(out.rb, rb.data(), sizeof(int) * rb.size(),
                           cudaMemcpyHostToDevice, st));
  if (want_fp32) {
    out.v32 = dalloc_n<float>(padn, st);
    launch_convert_d2f(out.v64, out.v32, padn, st);
    BK_CHECK(cudaGetLastError());
  }
  // Structure scan on the GPU (one small read-back).
  out.ddiag = dalloc_n<double>(pad64(n), st);
  CsrScanH* dscan = dalloc_n<CsrScanH>(1, st);
  launch_csr_scan(out.rowptr, out.col, out.v64, n, out.ddiag, dscan, st);
  BK_CHECK(cudaGetLastError());
  BK_CHECK(cudaMemcpyAsync(&out.scan, dscan, sizeof(CsrScanH), cudaMemcpyDeviceToHost, st));
  dfree(dscan, st);
  BK_CHECK(cudaStreamSynchronize(st));
  if (out.scan.flags & kScanBadCol) {
    out.release(st);
    throw CudaError("matrix: column index out of range");
  }
  std::sort(out.scan.off, out.scan.off + std::min(out.scan.noff, kScanOffs));
  if (dia_wanted(out.scan, n, nnz)) build_dia(out, st);
  if (out.ndia == 0 && n >= (1 << 16)) build_sell(out, rowptr, st);
  out.variant = heuristic_variant(n, nnz, out.ndia > 0);
  if (n >= (1 << 16)) autotune_spmv(out, st);
}

void SolveState::create(int cap, cudaStream_t st) {
  S = dalloc_n<double>(kScalars, st);
  ctl = dalloc_n<CtlH>(2, st);
  ctl_free = ctl + 1;
  part = dalloc_n<double>((long long)kPartRows * kGridCap, st);
  ticket = dalloc_n<unsigned>(4, st);
  hist_cap = cap;
  hist = cap > 0 ? dalloc_n<double>(cap, st) : nullptr;
  BK_CHECK(cudaMemsetAsync(S, 0, sizeof(double) * kScalars, st));
  BK_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * 4, st));
  BK_CHECK(cudaMemsetAsync(ctl, 0, 2 * sizeof(CtlH), st));
}

void cond_block(SolveState& ss, cudaStream_t st,
                const std::function<void(cudaStream_t)>& inner) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess ||
      cs != cudaStreamCaptureStatusActive) {
    cudaGetLastError();
    inner(st);
    return;
  }
  // The capture's graph and its current dependencies (their edge types are
  // dropped: the conditional node follows them with plain edges).
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  const cudaGraphEdgeData* edges = nullptr;
  size_t nd = 0;
  BK_CHECK(cudaStreamGetCaptureInfo_v3(st, &cs, nullptr, &g, &deps, &edges, &nd));
  std::vector<cudaGraphNode_t> dv(deps, deps + nd);
  cudaGraphConditionalHandle h;
  BK_CHECK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  std::memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  BK_CHECK(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &cp));
  if (!ss.side) BK_CHECK(cudaStreamCreateWithFlags(&ss.side, cudaStreamNonBlocking));
  BK_CHECK(cudaStreamBeginCaptureToGraph(ss.side, cp.conditional.phGraph_out[0], nullptr,
                                         nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const long long c0 = launch_count(), y0 = byte_count();
  g_plain_scope = true;
  try {
    inner(ss.side);
  } catch (...) {
    g_plain_scope = false;
    cudaGraph_t dropped = nullptr;
    cudaStreamEndCapture(ss.side, &dropped);
    if (dropped) cudaGraphDestroy(dropped);
    throw;
  }
  g_plain_scope = false;
  g_plain_launches = 1;   // the kernel after the node follows it plainly
  ss.cond_kernels += launch_count() - c0;
  ss.cond_bytes += byte_count() - y0;
  cudaGraph_t captured = nullptr;
  BK_CHECK(cudaStreamEndCapture(ss.side, &captured));
  BK_CHECK(cudaStreamUpdateCaptureDependencies(st, &node, 1,
                                               cudaStreamSetCaptureDependencies));
  if (ss.n_cond >= 2) throw CudaError("more than two conditional nodes in a body");
  ss.cond_handle[ss.n_cond++] = (unsigned long long)h;
  ss.has_cond = true;
}

void SolveState::release(cudaStream_t st) {
  dfree(S, st);
  dfree(ctl, st);
  dfree(part, st);
  dfree(ticket, st);
  dfree(hist, st);
  if (side) {
    cudaStreamSynchronize(side);
    cudaStreamDestroy(side);
    side = nullptr;
  }
  has_cond = false;
  S = nullptr;
  ctl = nullptr;
  ctl_free = nullptr;
  part = nullptr;
  ticket = nullptr;
  hist = nullptr;
}

void SolveState::start(int iter0, int max_iter, double tol, cudaStream_t st) {
  launch_ctl_init(ctl, ticket, S, iter0, max_iter, tol, hist, hist_cap, -1,
                  0.0, st);
  BK_CHECK(cudaGetLastError());
}

CtlH SolveState::read(cudaStream_t st) const {
  CtlH c;
  BK_CHECK(cudaMemcpyAsync(&c, ctl, sizeof(c), cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
  return c;
}

void SolveState::set_scalar(short slot, double v, cudaStream_t st) {
  launch_set_scalar(S, slot, v, st);
  BK_CHECK(cudaGetLastError());
}

void SolveState::set_scalars(short slot, const double* host, int count,
                             cudaStream_t st) {
  if (count <= 0) return;
  BK_CHECK(cudaMemcpyAsync(S + slot, host, sizeof(double) * count,
                           cudaMemcpyHostToDevice, st));
  BK_CHECK(cudaStreamSynchronize(st));
}

double SolveState::get_scalar(short slot, cudaStream_t st) const {
  double v = 0.0;
  BK_CHECK(cudaMemcpyAsync(&v, S + slot, sizeof(double),
                           cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
  return v;
}

template <typename T>
void Lc<T>::launch(const RedH& rd, cudaStream_t st) {
  for (size_t k = 0; k < dots_.size(); ++k) {
    int a = dots_[k].first, b = dots_[k].second;
    if (a >= OUT) a = d.nin + (a - OUT);
    if (b >= OUT) b = d.nin + (b - OUT);
    d.dot[k][0] = (unsigned char)a;
    d.dot[k][1] = (unsigned char)b;
  }
  if constexpr (sizeof(T) == 8)
    launch_lincomb_d(d, rd, st);
  else
    launch_lincomb_f(d, rd, st);
}
template struct Lc<double>;
template struct Lc<float>;

void spmv(const DevCsr& A, const SpmvH<double>& io, const RedH& rd,
          cudaStream_t st) {
  launch_spmv_d(A.h64(), io, rd, st);
}
void spmv(const DevCsr& A, const SpmvH<float>& io, const RedH& rd,
          cudaStream_t st) {
  launch_spmv_f(A.h32(), io, rd, st);
}

static bool run_graph_while(SolveState& ss,
                            const std::function<void(cudaStream_t)>& body,
                            cudaStream_t st, long long& body_kernels,
                            long long& body_bytes) {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
  bool ok = false;
  do {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) !=
        cudaSuccess)
      break;
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) break;
    cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(st, bodyg, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
      break;
    const long long c0 = launch_count(), y0 = byte_count();
    ss.has_cond = false;
    ss.n_cond = 0;
    ss.cond_kernels = 0;
    ss.cond_bytes = 0;
    bool body_ok = true;
    try {
      body(st);
      launch_loop_control(ss.ctl, (unsigned long long)h, 1, st);
    } catch (const std::exception&) {
      body_ok = false;   // capture is ended below; the host-polled loop runs
    }
    g_plain_scope = false;
    g_plain_launches = 0;
    body_kernels = launch_count() - c0;
    launch_count() = c0;   // captured, not launched
    body_bytes = byte_count() - y0;
    byte_count() = y0;
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &captured);
    if (ce != cudaSuccess || !body_ok) {
      cudaGetLastError();
      ss.has_cond = false;
      break;
    }
    if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
      cudaGetLastError();
      ex = nullptr;
      break;
    }
    ok = true;
  } while (false);
  if (ok) {
    if (ss.has_cond) {
      // Hand the conditional node's handle to the device epilogues.
      struct { unsigned long long cond; int use; int pad; unsigned long long alt; } cc{
          ss.cond_handle[0], 1, 0, ss.cond_handle[1]};
      static_assert(sizeof(cc) == sizeof(CtlH) - offsetof(CtlH, cond), "control block tail");
      BK_CHECK(cudaMemcpyAsync(&ss.ctl->cond, &cc, sizeof(cc), cudaMemcpyHostToDevice, st));
    }
    BK_CHECK(cudaGraphLaunch(ex, st));
    BK_CHECK(cudaStreamSynchronize(st));
  }
  if (ex) cudaGraphExecDestroy(ex);
  cudaGraphDestroy(g);
  return ok;
}

// Records `body` and runs it in the group's persistent launch; false when
// the body has an operation without a persistent form (the caller then
// runs the graph loop).
static bool run_persist_member(PersistGroup& grp, SolveState& ss,
                               const std::function<void(cudaStream_t)>& body,
                               cudaStream_t st, CtlH& out) {
  std::vector<ProgOpH> ops;
  const long long c0 = launch_count(), y0 = byte_count();
  bool ok = true;
  g_prog_rec = &ops;
  ss.has_cond = false;
  try {
    body(st);
  } catch (const CudaError&) {
    ok = false;
  }
  g_prog_rec = nullptr;
  const long long body_bytes = byte_count() - y0;
  launch_count() = c0;
  byte_count() = y0;
  if (!ok || ops.empty()) {
    grp.withdraw(st);
    return false;
  }
  out = grp.join(ss, ops, st);
  launch_count() += 1;
  byte_count() += body_bytes * out.trips;
  return true;
}

CtlH run_loop(SolveState& ss, const std::function<void(cudaStream_t)>& body,
              cudaStream_t st) {
  if (PersistGroup* grp = persist_group()) {
    persist_group() = nullptr;
    CtlH c;
    if (run_persist_member(*grp, ss, body, st, c)) return c;
  } else if (Ctx::get().persistent) {
    PersistGroup one(1);   // this solve alone in a persistent launch
    CtlH c;
    if (run_persist_member(one, ss, body, st, c)) return c;
  }
  Ctx& cx = Ctx::get();
  if (cx.use_cond_graph) {
    long long bk_n = 0, bk_bytes = 0;
    if (run_graph_while(ss, body, st, bk_n, bk_bytes)) {
      CtlH c = ss.read(st);
      launch_count() += bk_n * c.trips;
      byte_count() += bk_bytes * c.trips;
      return c;
    }
    cx.use_cond_graph = false;   // not supported here: poll from now on
  }
  CtlH c = ss.read(st);
  if (c.done) return c;
  int chunk = 1;
  for (;;) {
    for (int k = 0; k < chunk; ++k) {
      body(st);
      launch_loop_control(ss.ctl, 0ull, 0, st);
    }
    BK_CHECK(cudaGetLastError());
    c = ss.read(st);
    if (c.done) return c;
    chunk = std::min(chunk * 2, 32);
  }
}

}  // namespace bk
