// Persistent groups (runtime.h: PersistGroup): the host half of the
// persistent loop.  Members hand in their recorded iterations; the last to
// arrive lays the operation table out in device memory and makes one
// cooperative launch of k_persist for all of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "runtime.h"

namespace bk {

void prog_push(const ProgOpH& op) {
  static_cast<std::vector<ProgOpH>*>(g_prog_rec)->push_back(op);
}

void prog_unsupported(const char* what) {
  throw CudaError(std::string("no persistent form: ") + what);
}

void prog_require_aligned(const void* p) {
  if (reinterpret_cast<uintptr_t>(p) & 15u) prog_unsupported("unaligned vector");
}

PersistGroup*& persist_group() {
  thread_local PersistGroup* g = nullptr;
  return g;
}

// Polls per barrier wait before a CTA gives up: BKSP_GPU_SPIN_LIMIT, else
// 2^24 (seconds of waiting; a phase takes microseconds to milliseconds).
static long long default_spin_limit() {
  static const long long v = [] {
    const char* e = std::getenv("BKSP_GPU_SPIN_LIMIT");
    const long long x = e ? std::atoll(e) : 0;
    return x > 0 ? x : (1LL << 24);
  }();
  return v;
}

struct PersistGroup::Impl {
  struct Member {
    SolveState* ss;
    cudaStream_t st;
    std::vector<ProgOpH> ops;
    cudaEvent_t ready = nullptr;
  };
  int expected = 0;
  int withdrawn = 0;
  bool launched = false;
  std::vector<Member> members;
  cudaEvent_t done = nullptr;
  std::mutex mu;
  std::condition_variable cv;
};

PersistGroup::PersistGroup(int expected) : p_(new Impl) {
  p_->expected = expected;
}

PersistGroup::~PersistGroup() {
  for (auto& m : p_->members)
    if (m.ready) cudaEventDestroy(m.ready);
  if (p_->done) cudaEventDestroy(p_->done);
  delete p_;
}

void PersistGroup::withdraw(cudaStream_t st) {
  std::lock_guard<std::mutex> lk(p_->mu);
  ++p_->withdrawn;
  if (!p_->launched &&
      (int)p_->members.size() + p_->withdrawn >= p_->expected)
    launch_locked(st);
}

CtlH PersistGroup::join(SolveState& ss, std::vector<ProgOpH>& ops,
                        cudaStream_t st) {
  std::unique_lock<std::mutex> lk(p_->mu);
  if (p_->launched) throw CudaError("persistent group already launched");
  Impl::Member m;
  m.ss = &ss;
  m.st = st;
  m.ops.swap(ops);
  BK_CHECK(cudaEventCreateWithFlags(&m.ready, cudaEventDisableTiming));
  BK_CHECK(cudaEventRecord(m.ready, st));   // this member's set-up is queued
  p_->members.push_back(std::move(m));
  if ((int)p_->members.size() + p_->withdrawn >= p_->expected)
    launch_locked(st);
  else
    p_->cv.wait(lk, [&] { return p_->launched; });
  if (status != 0)
    throw CudaError(status == 1 ? "persistent loop: a grid barrier wait ran out"
                                : "persistent loop: launch failed");
  BK_CHECK(cudaStreamWaitEvent(st, p_->done, 0));
  lk.unlock();
  return ss.read(st);
}

// Called with the lock held, by the member (or withdrawing thread) that
// completes the group.
void PersistGroup::launch_locked(cudaStream_t st) {
  Impl& g = *p_;
  g.launched = true;
  try {
    const int nsys = (int)g.members.size();
    if (nsys == 0) {
      g.cv.notify_all();
      return;
    }
    if (nsys > kPersistMaxSys) throw CudaError("persistent group too large");
    int max_ops = 0;
    for (auto& m : g.members) max_ops = std::max(max_ops, (int)m.ops.size());
    // Grid: at least kUnitsPerCta units of the widest phase per CTA (a
    // CTA streams its units back to back; below that the barrier costs more
    // than the extra parallelism gains), at most every CTA that fits.
    constexpr long long kUnitsPerCta = 4;
    long long widest = 1;
    for (int k = 0; k < max_ops; ++k) {
      long long u = 0;
      for (auto& m : g.members)
        if (k < (int)m.ops.size()) u += m.ops[k].units;
      widest = std::max(widest, u);
    }
    int cap = persist_max_grid();
    if (max_grid > 0) cap = std::min(cap, max_grid);
    grid = (int)std::max<long long>(1, std::min<long long>((widest + kUnitsPerCta - 1) / kUnitsPerCta, cap));
    if (absent_cta >= 0) grid = std::max(grid, std::min(cap, absent_cta + 2));
    // Device layout: operations, their headers, control-block pointers,
    // counts, barrier.
    const size_t nop = (size_t)nsys * max_ops;
    const size_t ops_b = sizeof(ProgOpH) * nop;
    const size_t hdr_b = sizeof(OpHdrH) * nop;
    const size_t ctl_b = sizeof(CtlH*) * nsys;
    const size_t cnt_b = sizeof(int) * nsys;
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t off_hdr = up16(ops_b), off_ctl = off_hdr + up16(hdr_b),
                 off_cnt = off_ctl + up16(ctl_b), off_bar = off_cnt + up16(cnt_b);
    const size_t total = off_bar + up16(sizeof(PBarH));
    std::vector<unsigned char> host(total, 0);
    for (int s = 0; s < nsys; ++s) {
      auto& m = g.members[s];
      std::memcpy(host.data() + sizeof(ProgOpH) * (size_t)s * max_ops,
                  m.ops.data(), sizeof(ProgOpH) * m.ops.size());
      for (size_t k = 0; k < m.ops.size(); ++k) {
        const OpHdrH h{m.ops[k].units, m.ops[k].rd.guard, m.ops[k].rd.S};
        std::memcpy(host.data() + off_hdr + sizeof(OpHdrH) * ((size_t)s * max_ops + k),
                    &h, sizeof(h));
      }
      CtlH* c = m.ss->ctl;
      std::memcpy(host.data() + off_ctl + sizeof(CtlH*) * s, &c, sizeof(c));
      const int n = (int)m.ops.size();
      std::memcpy(host.data() + off_cnt + sizeof(int) * s, &n, sizeof(n));
    }
    for (auto& m : g.members) BK_CHECK(cudaStreamWaitEvent(st, m.ready, 0));
    unsigned char* dev = static_cast<unsigned char*>(dalloc(total, st));
    // Pageable source: the copy is staged before the call returns.
    BK_CHECK(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice, st));
    PersistH p;
    p.ops = reinterpret_cast<const ProgOpH*>(dev);
    p.hdr = reinterpret_cast<const OpHdrH*>(dev + off_hdr);
    p.ctl = reinterpret_cast<CtlH* const*>(dev + off_ctl);
    p.nops = reinterpret_cast<const int*>(dev + off_cnt);
    p.nsys = nsys;
    p.max_ops = max_ops;
    p.bar = reinterpret_cast<PBarH*>(dev + off_bar);
    p.spin_limit = spin_limit > 0 ? spin_limit : default_spin_limit();
    p.absent_cta = absent_cta;
    const cudaError_t le = launch_persist(p, grid, st);
    PBarH bar{};
    if (le == cudaSuccess) {
      BK_CHECK(cudaMemcpyAsync(&bar, p.bar, sizeof(bar), cudaMemcpyDeviceToHost, st));
    } else {
      cudaGetLastError();
    }
    BK_CHECK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    BK_CHECK(cudaEventRecord(g.done, st));
    BK_CHECK(cudaStreamSynchronize(st));
    dfree(dev, st);
    if (le != cudaSuccess) {
      status = 2;
      if (std::getenv("BKSP_GPU_VERBOSE"))
        std::fprintf(stderr, "bksp: persistent launch (%d CTAs): %s\n", grid,
                     cudaGetErrorString(le));
    } else if (bar.err) {
      status = 1;
      err_phase = bar.err_phase;
    }
  } catch (const std::exception& e) {
    status = 2;
    if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
    if (!g.done && cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming) == cudaSuccess)
      cudaEventRecord(g.done, st);
    cudaGetLastError();
  }
  g.cv.notify_all();
}

}  // namespace bk
