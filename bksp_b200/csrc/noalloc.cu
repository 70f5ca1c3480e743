// bksp_gpu_true_residual_noalloc: the FP64 relative true residual
// ||b - A x|| / ||b|| of device vectors, computed without allocating any
// memory.  It exists for callers that cannot allocate device memory at the
// point where they need the residual: a host application whose own memory
// pool already owns all of the GPU's memory (a cudaMalloc there would fail,
// or fragment that pool), and latency-critical monitoring loops that cannot
// accept the device-wide synchronisation cudaMalloc / cudaFree imply.
//
// The work is the same SpMV-with-dot-products kernel the allocating entry
// point bksp_gpu_true_residual launches; only its scratch differs: the
// residual vector, the per-block partial sums, the scalar slots and the
// control block all live in the file-scope array below.  That array is
// static device memory: every GPU that loads the library holds its
// kScratchBytes until the process exits, which is why it is capped at
// kNoAllocMaxRows rows (8 MiB of residual).  All calls on a device share it
// and it keeps the last call's contents, so the arrival ticket and the
// control block are cleared at the start of each call; two calls whose
// work overlaps on the GPU (different streams, or different host threads)
// race on it and must be serialised by the caller.  The device address of
// the array is looked up once per device and cached; a cudaDeviceReset
// invalidates it, so a process that resets a device must not call this
// entry point on that device again.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <exception>
#include <mutex>

#include "capi_internal.h"
#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_spmv.cuh"

namespace {

using namespace bk;

constexpr long long kNoAllocMaxRows = 1LL << 20;
constexpr long long kPartOff = kNoAllocMaxRows;                 // doubles
constexpr long long kSOff = kPartOff + 2LL * kMaxBlocks;
constexpr long long kCtlOff = kSOff + kScalars;                 // 256 B slot
constexpr long long kTicketOff = kCtlOff + 32;
constexpr long long kScratchDoubles = kTicketOff + 32;
constexpr size_t kScratchBytes = sizeof(double) * kScratchDoubles;
static_assert(sizeof(Ctl) <= 32 * sizeof(double), "control block slot");

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device.  The array's
// name is only a host-side stand-in; the address is looked up once per
// device, with that device current, on the first call made on it.
double* scratch_for_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    double* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (rc != cudaSuccess) {
      std::fprintf(stderr,
                   "bksp_gpu_true_residual_noalloc: cudaGetSymbolAddress "
                   "failed on device %d: %s\n", dev, cudaGetErrorString(rc));
      cudaGetLastError();
      return nullptr;
    }
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

}  // namespace

extern "C" int bksp_gpu_true_residual_noalloc(bksp_gpu_matrix* m,
                                              const double* b,
                                              const double* x, void* stream,
                                              double* res) {
  if (!m || !b || !x || !res) return INVALID_PARAMETERS;
  const int n = m->A.n;
  if ((long long)n > kNoAllocMaxRows) {
    std::fprintf(stderr,
                 "bksp_gpu_true_residual_noalloc: the operator has %d rows; "
                 "this entry point's static scratch holds at most %lld rows "
                 "(use bksp_gpu_true_residual)\n", n, kNoAllocMaxRows);
    return INVALID_PARAMETERS;
  }
  // The scratch is picked by the current device, so the operator must live
  // on that device: a kernel on one GPU reading another GPU's operator
  // through this GPU's scratch would fault or silently cross the link.
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != m->device) {
    cudaGetLastError();
    std::fprintf(stderr,
                 "bksp_gpu_true_residual_noalloc: the operator lives on device "
                 "%d but device %d is current\n", m->device, cur);
    return INVALID_PARAMETERS;
  }
  cudaStream_t st = nullptr;
  if (stream) {
    st = static_cast<cudaStream_t>(stream);
  } else {
    // The calling thread's library stream; its first use on a thread
    // creates it, which can fail (and throws inside the library).
    try {
      st = Ctx::get().st;
    } catch (const std::exception&) {
      cudaGetLastError();
      return INVALID_PARAMETERS;
    }
  }
  double* base = scratch_for_current_device();
  if (!base) return INVALID_PARAMETERS;
  double* r = base;
  double* part = base + kPartOff;
  double* S = base + kSOff;
  Ctl* ctl = reinterpret_cast<Ctl*>(base + kCtlOff);
  unsigned* ticket = reinterpret_cast<unsigned*>(base + kTicketOff);
  // What must start at zero: the control block (done flag) and the ticket.
  if (cudaMemsetAsync(ctl, 0, sizeof(double) * 64, st) != cudaSuccess) {
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
  SpmvH<double> io;
  std::memset(&io, 0, sizeof(io));
  io.x = x;
  io.y = r;
  io.b = b;
  io.mode = 1;
  io.nd = 2;
  io.dot[0][0] = 0; io.dot[0][1] = 0;   // (r, r)
  io.dot[1][0] = 1; io.dot[1][1] = 1;   // (b, b)
  Red rd{part, ticket, S, ctl, kD, E_NONE, 0, 0};
  const CsrH A = m->A.h64();
  const int g = A.nrb < kMaxBlocks ? (A.nrb > 0 ? A.nrb : 1) : kMaxBlocks;
  k_spmv<double, double, 2><<<g, kThreads, 0, st>>>(A, io, rd);
  double dots[2] = {0.0, 0.0};
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(dots, S + kD, sizeof(dots), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return INVALID_PARAMETERS;
  }
  *res = std::sqrt(dots[0]) / std::sqrt(dots[1]);
  return 0;
}
