// Learned SPAI preconditioner, host side: model lifecycle, slot analysis of
// an operator, inference, training loop (Adam), gradient access for tests,
// checkpoint files.  No counterpart in the reference.
#include "spai.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <algorithm>

#include "capi_internal.h"

using namespace bk;

namespace bk {

void SpaiSlots::release(cudaStream_t st) {
  dfree(slot_entry, st);
  dfree(feat, st);
  dfree(dinv, st);
  slot_entry = nullptr;
  feat = nullptr;
  dinv = nullptr;
  ok = false;
}

void spai_build_slots(const DevCsr& A, SpaiSlots& s, cudaStream_t st) {
  s.ok = false;
  // The operator's distinct diagonal offsets come from its structure scan.
  if (A.scan.flags & (kScanManyOffs | kScanBadCol)) return;
  const int noff = A.scan.noff;
  if (noff > kSlots) return;   // more diagonals than slots
  std::vector<int> neg, pos;
  bool has0 = false;
  for (int q = 0; q < noff; ++q) {
    const int o = A.scan.off[q];
    if (o < 0) neg.push_back(o);
    else if (o > 0) pos.push_back(o);
    else has0 = true;
  }
  if (!has0 || neg.size() > (size_t)kCenterSlot ||
      pos.size() > (size_t)(kSlots - 1 - kCenterSlot))
    return;
  std::sort(neg.begin(), neg.end(), [](int a, int b) { return a > b; });
  std::sort(pos.begin(), pos.end());
  int so[kSlots] = {}, sl[kSlots] = {}, ns = 0;
  so[ns] = 0; sl[ns++] = kCenterSlot;
  for (size_t r = 0; r < neg.size(); ++r) { so[ns] = neg[r]; sl[ns++] = kCenterSlot - 1 - (int)r; }
  for (size_t r = 0; r < pos.size(); ++r) { so[ns] = pos[r]; sl[ns++] = kCenterSlot + 1 + (int)r; }
  s.slot_entry = dalloc_n<int>((long long)A.n * kSlots, st);
  launch_spai_slot_map(A.n, A.rowptr, A.col, so, sl, ns, s.slot_entry, st);
  BK_CHECK(cudaGetLastError());
  s.ok = true;
}

static void ensure_features(bksp_gpu_matrix* m, cudaStream_t st) {
  SpaiSlots& s = m->spai;
  if (!s.ok) throw CudaError("learned preconditioner: operator is not stencil-like");
  if (s.feat) return;
  const int n = m->A.n;
  s.feat = dalloc_n<float>((long long)n * kSlots, st);
  s.dinv = dalloc_n<float>(n, st);
  launch_spai_features(n, m->A.rowptr, m->A.v64, s.slot_entry, s.feat, s.dinv, st);
  BK_CHECK(cudaGetLastError());
}

long long spai_scratch_floats(const bksp_gpu_matrix* m, bool symmetric) {
  const long long csr = pad64((long long)m->A.nnz + 8);
  return csr + (long long)m->A.ndia * pad64(m->A.n) + (symmetric ? csr : 0);
}

DevCsr spai_apply(bksp_gpu_spai_model* model, bksp_gpu_matrix* m, float* mvals,
                  cudaStream_t st, bool symmetric) {
  ensure_features(m, st);
  const int n = m->A.n;
  const long long csr = pad64((long long)m->A.nnz + 8);
  float* pred = symmetric
                    ? mvals + csr + (long long)m->A.ndia * pad64(n)
                    : mvals;
  BK_CHECK(cudaMemsetAsync(pred, 0, sizeof(float) * ((size_t)m->A.nnz + 8), st));
  launch_spai_infer(n, model->w, m->spai.feat, m->spai.dinv, m->spai.slot_entry,
                    pred, st);
  // features, slot map and 1/a_ii read per row; M's values written
  byte_count() += (long long)n * (8LL * kSlots + 4) + 4LL * m->A.nnz;
  if (symmetric) {
    BK_CHECK(cudaMemsetAsync(mvals, 0, sizeof(float) * ((size_t)m->A.nnz + 8), st));
    launch_spai_symmetrize(n, m->A.rowptr, m->A.col, pred, mvals, st);
    byte_count() += 4LL * (n + 1) + 12LL * m->A.nnz;
  }
  BK_CHECK(cudaGetLastError());
  DevCsr v;
  v.n = n;
  v.nnz = m->A.nnz;
  v.nrb = m->A.nrb;
  v.rowptr = m->A.rowptr;
  v.col = m->A.col;
  v.rb = m->A.rb;
  v.variant = m->A.variant;
  v.v32 = mvals;
  if (m->A.ndia > 0) {
    // M has A's pattern: A's diagonals and row masks, M's values.
    v.ndia = m->A.ndia;
    for (int d = 0; d < kDiaMax; ++d) v.doff[d] = m->A.doff[d];
    v.dmask = m->A.dmask;
    v.owns_dmask = false;
    const long long dn = (long long)v.ndia * pad64(n);
    v.d32 = mvals + pad64((long long)m->A.nnz + 8);
    BK_CHECK(cudaMemsetAsync(v.d32, 0, sizeof(float) * dn, st));
    launch_csr2dia_f(v.hview(v.v32, v.d32), v.v32, v.d32, nullptr, st);
    BK_CHECK(cudaGetLastError());
  }
  return v;
}

}  // namespace bk

namespace {

// Initial parameters: He-scaled uniform hidden layers, zero output weights
// and an output bias selecting the diagonal slot, so the untrained model is
// Jacobi (m_ii = 1 / a_ii, all other m_ij = 0).
std::vector<float> init_params(unsigned seed) {
  constexpr int S = kSlots, H = kHidden;
  std::vector<float> p(kSpaiParams, 0.0f);
  std::mt19937 g(seed);
  auto fill = [&](int off, int cnt, int fan_in) {
    const float a = std::sqrt(6.0f / (float)fan_in);
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < cnt; ++i) p[off + i] = u(g);
  };
  const int oW1 = 0, ob1 = H * S, oW2 = ob1 + H, ob2 = oW2 + H * H;
  const int oW3 = ob2 + H, ob3 = oW3 + S * H;
  fill(oW1, H * S, S);
  fill(oW2, H * H, H);
  for (int i = 0; i < H; ++i) { p[ob1 + i] = 0.01f; p[ob2 + i] = 0.01f; }
  for (int i = 0; i < S * H; ++i) p[oW3 + i] = 0.0f;
  p[ob3 + kCenterSlot] = 1.0f;
  return p;
}

int fail(const std::exception& e) {
  if (std::getenv("BKSP_GPU_VERBOSE")) std::fprintf(stderr, "bksp: %s\n", e.what());
  cudaGetLastError();
  return INVALID_PARAMETERS;
}

// Probe block Z (probes x np, column-major, Rademacher) and AZ = A Z (FP32).
struct Probes {
  float* Z = nullptr;
  float* AZ = nullptr;
  long long np = 0;
  int k = 0;
  void make(bksp_gpu_matrix* m, int probes, uint32_t seed, const float* Zhost,
            cudaStream_t st) {
    np = pad64(m->A.n);
    k = probes;
    Z = dalloc_n<float>(np * k, st);
    AZ = dalloc_n<float>(np * k, st);
    BK_CHECK(cudaMemsetAsync(AZ, 0, sizeof(float) * np * k, st));
    if (Zhost) {
      BK_CHECK(cudaMemsetAsync(Z, 0, sizeof(float) * np * k, st));
      for (int c = 0; c < k; ++c)
        BK_CHECK(cudaMemcpyAsync(Z + c * np, Zhost + (size_t)c * m->A.n,
                                 sizeof(float) * m->A.n, cudaMemcpyHostToDevice, st));
    } else {
      launch_spai_probes(m->A.n, k, np, seed, Z, st);
    }
    SolveState ss;   // SpMV needs a (never-finished) control block
    ss.create(0, st);
    ss.start(0, 1, 0.0, st);
    for (int c = 0; c < k; ++c)
      spmv(m->A, spmv_io<float>(Z + c * np, AZ + c * np), ss.red(kD, E_NONE), st);
    BK_CHECK(cudaGetLastError());
    ss.release(st);
  }
  void release(cudaStream_t st) {
    dfree(Z, st);
    dfree(AZ, st);
  }
};

constexpr int kChunkRows = 1 << 16;   // rows per gradient step (mini-batch)

// One gradient evaluation over rows [r0, r0 + cnt) (+ Adam step if step > 0).
void grad_chunk(bksp_gpu_spai_model* md, bksp_gpu_matrix* m, const Probes& pr,
                int r0, int cnt, int step, float lr, float* gpart, float* lpart,
                cudaStream_t st) {
  const float scale = 1.0f / ((float)cnt * (float)pr.k);
  SpaiSlots& s = m->spai;
  launch_spai_grad(cnt, md->w, s.feat + (size_t)r0 * kSlots, s.dinv + r0,
                   s.slot_entry + (size_t)r0 * kSlots, m->A.col, pr.Z + r0,
                   pr.AZ, pr.k, pr.np, scale, gpart, lpart, st);
  launch_spai_reduce_adam(spai_grad_blocks(cnt), gpart, lpart, md->grad, md->loss,
                          scale, md->w, md->am, md->av, step, lr, st);
  BK_CHECK(cudaGetLastError());
}

}  // namespace

extern "C" {

int bksp_gpu_spai_nparams(void) { return kSpaiParams; }

int bksp_gpu_spai_create(unsigned seed, bksp_gpu_spai_model** out) {
  if (!out) return INVALID_PARAMETERS;
  *out = nullptr;
  bksp_gpu_spai_model* md = new bksp_gpu_spai_model();
  try {
    cudaStream_t st = Ctx::get().st;
    md->device = Ctx::get().device;
    md->w = dalloc_n<float>(kSpaiParams, st);
    md->am = dalloc_n<float>(kSpaiParams, st);
    md->av = dalloc_n<float>(kSpaiParams, st);
    md->grad = dalloc_n<float>(kSpaiParams, st);
    md->loss = dalloc_n<double>(1, st);
    std::vector<float> p = init_params(seed);
    BK_CHECK(cudaMemcpyAsync(md->w, p.data(), sizeof(float) * kSpaiParams,
                             cudaMemcpyHostToDevice, st));
    BK_CHECK(cudaMemsetAsync(md->am, 0, sizeof(float) * kSpaiParams, st));
    BK_CHECK(cudaMemsetAsync(md->av, 0, sizeof(float) * kSpaiParams, st));
    BK_CHECK(cudaMemsetAsync(md->grad, 0, sizeof(float) * kSpaiParams, st));
    BK_CHECK(cudaStreamSynchronize(st));
    *out = md;
    return 0;
  } catch (const std::exception& e) {
    delete md;
    return fail(e);
  }
}

int bksp_gpu_spai_destroy(bksp_gpu_spai_model* md) {
  if (!md) return 0;
  cudaStream_t st = Ctx::get().st;
  dfree(md->w, st);
  dfree(md->am, st);
  dfree(md->av, st);
  dfree(md->grad, st);
  dfree(md->loss, st);
  cudaStreamSynchronize(st);
  delete md;
  return 0;
}

// get (set = 0) or set (set = 1) the kSpaiParams parameters (host floats).
int bksp_gpu_spai_params(bksp_gpu_spai_model* md, float* host, int set) {
  if (!md || !host) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = Ctx::get().st;
    if (set)
      BK_CHECK(cudaMemcpyAsync(md->w, host, sizeof(float) * kSpaiParams,
                               cudaMemcpyHostToDevice, st));
    else
      BK_CHECK(cudaMemcpyAsync(host, md->w, sizeof(float) * kSpaiParams,
                               cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Loss ||(I - M A) Z||_F^2 / (n * probes) and its gradient (host, may be
// NULL) for the probe block Z (probes x n, column-major host floats; NULL:
// seeded Rademacher probes).  No parameter update.
int bksp_gpu_spai_loss_grad(bksp_gpu_spai_model* md, bksp_gpu_matrix* m,
                            const float* Zhost, int probes, unsigned seed,
                            double* loss, float* grad) {
  if (!md || !m || probes < 1 || !m->A.v32) return INVALID_PARAMETERS;
  if (!m->spai.ok) return INVALID_PARAMETERS;
  if (m->A.n > kChunkRows) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = Ctx::get().st;
    ensure_features(m, st);
    Probes pr;
    pr.make(m, probes, seed, Zhost, st);
    const int n = m->A.n;
    float* gpart = dalloc_n<float>((long long)spai_grad_blocks(n) * kSpaiParams, st);
    float* lpart = dalloc_n<float>(spai_grad_blocks(n), st);
    grad_chunk(md, m, pr, 0, n, 0, 0.0f, gpart, lpart, st);
    if (loss)
      BK_CHECK(cudaMemcpyAsync(loss, md->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (grad)
      BK_CHECK(cudaMemcpyAsync(grad, md->grad, sizeof(float) * kSpaiParams,
                               cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    dfree(gpart, st);
    dfree(lpart, st);
    pr.release(st);
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Adam training on the rows of `nsys` operators (each created with
// BKSP_GPU_FP32), fresh Rademacher probes per epoch and operator, one Adam
// step per chunk of at most 65,536 rows.  *loss_out: mean loss of the last
// epoch.
int bksp_gpu_spai_train(bksp_gpu_spai_model* md, bksp_gpu_matrix* const* sys,
                        int nsys, int epochs, int probes, float lr,
                        unsigned seed, double* loss_out) {
  if (!md || !sys || nsys < 1 || epochs < 0 || probes < 1) return INVALID_PARAMETERS;
  for (int s = 0; s < nsys; ++s)
    if (!sys[s] || !sys[s]->A.v32 || !sys[s]->spai.ok) return INVALID_PARAMETERS;
  try {
    cudaStream_t st = Ctx::get().st;
    float* gpart = dalloc_n<float>((long long)spai_grad_blocks(kChunkRows) * kSpaiParams, st);
    float* lpart = dalloc_n<float>(spai_grad_blocks(kChunkRows), st);
    double last = 0.0;
    for (int e = 0; e < epochs; ++e) {
      double sum = 0.0;
      int cnt = 0;
      for (int s = 0; s < nsys; ++s) {
        bksp_gpu_matrix* m = sys[s];
        ensure_features(m, st);
        Probes pr;
        pr.make(m, probes, seed * 7919u + (uint32_t)(e * nsys + s) * 104729u, nullptr, st);
        for (int r0 = 0; r0 < m->A.n; r0 += kChunkRows) {
          const int c = std::min(kChunkRows, m->A.n - r0);
          grad_chunk(md, m, pr, r0, c, ++md->step, lr, gpart, lpart, st);
          double l = 0.0;
          BK_CHECK(cudaMemcpyAsync(&l, md->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
          BK_CHECK(cudaStreamSynchronize(st));
          sum += l;
          cnt++;
        }
        pr.release(st);
      }
      last = cnt ? sum / cnt : 0.0;
    }
    if (loss_out) *loss_out = last;
    dfree(gpart, st);
    dfree(lpart, st);
    BK_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Checkpoint: one text header line, then kSpaiParams little-endian floats.
int bksp_gpu_spai_save(bksp_gpu_spai_model* md, const char* path) {
  if (!md || !path) return INVALID_PARAMETERS;
  std::vector<float> p(kSpaiParams);
  if (bksp_gpu_spai_params(md, p.data(), 0) != 0) return INVALID_PARAMETERS;
  FILE* f = std::fopen(path, "wb");
  if (!f) return INVALID_PARAMETERS;
  std::fprintf(f, "{\"format\": \"bksp-spai\", \"version\": 1, \"slots\": %d, "
                  "\"hidden\": %d, \"params\": %d, \"dtype\": \"f32le\"}\n",
               kSlots, kHidden, kSpaiParams);
  const size_t w = std::fwrite(p.data(), sizeof(float), p.size(), f);
  std::fclose(f);
  return w == p.size() ? 0 : INVALID_PARAMETERS;
}

int bksp_gpu_spai_load(const char* path, bksp_gpu_spai_model** out) {
  if (!path || !out) return INVALID_PARAMETERS;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return INVALID_PARAMETERS;
  char line[512];
  int slots = 0, hidden = 0, params = 0;
  if (!std::fgets(line, sizeof(line), f) ||
      !std::strstr(line, "\"bksp-spai\"")) {
    std::fclose(f);
    return INVALID_PARAMETERS;
  }
  const char* a = std::strstr(line, "\"slots\": ");
  const char* b = std::strstr(line, "\"hidden\": ");
  const char* c = std::strstr(line, "\"params\": ");
  if (a) slots = std::atoi(a + 9);
  if (b) hidden = std::atoi(b + 10);
  if (c) params = std::atoi(c + 10);
  if (slots != kSlots || hidden != kHidden || params != kSpaiParams) {
    std::fclose(f);
    return INVALID_PARAMETERS;
  }
  std::vector<float> p(kSpaiParams);
  const size_t r = std::fread(p.data(), sizeof(float), p.size(), f);
  std::fclose(f);
  if (r != p.size()) return INVALID_PARAMETERS;
  bksp_gpu_spai_model* md = nullptr;
  if (bksp_gpu_spai_create(0, &md) != 0) return INVALID_PARAMETERS;
  if (bksp_gpu_spai_params(md, p.data(), 1) != 0) {
    bksp_gpu_spai_destroy(md);
    return INVALID_PARAMETERS;
  }
  *out = md;
  return 0;
}

}  // extern "C"
