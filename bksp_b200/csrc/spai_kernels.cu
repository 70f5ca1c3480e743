// Learned sparse-approximate-inverse preconditioner: kernels of the per-row
// MLP (no reference counterpart; bksp has no preconditioners).
//
// A row i of a stencil-like matrix is described by its entries on up to
// kSlots diagonals ("slots", ordered near-to-far: slot 3 is the diagonal,
// slots 2,1,0 the negative offsets nearest first, slots 4..7 the positive
// ones).  Features f_i[s] = a_{i,j_s} / a_ii (slot 3: the row sum / a_ii).
// The MLP  f -> relu(W1 f + b1) -> relu(W2 h1 + b2) -> W3 h2 + b3 = o
// predicts the SPAI row on A's pattern: m_{i,j_s} = o_s / a_ii.
//
// Training minimises  L = sum_i ||(Z - M W)_i||^2 / (rows * probes)  with
// W = A Z for random probe blocks Z, i.e. ||(I - M A) Z||_F^2 scaled; the
// loss decomposes by rows of M, so each thread owns one row end to end
// (forward, residual, backward) and a CTA reduces its rows' weight
// gradients through shared memory into per-CTA partials, which the Adam
// kernel sums in a fixed order (deterministic).
#include <mutex>
#include <cuda_runtime.h>
#include <stdint.h>

#include "spai_api.h"

namespace bk {

namespace {

constexpr int S = kSlots;   // 8
constexpr int H = kHidden;  // 64

// Parameter layout (floats): W1[H][S], b1[H], W2[H][H], b2[H], W3[S][H], b3[S].
constexpr int oW1 = 0, ob1 = oW1 + H * S, oW2 = ob1 + H, ob2 = oW2 + H * H,
              oW3 = ob2 + H, ob3 = oW3 + S * H, kP = ob3 + S;
static_assert(kP == kSpaiParams, "parameter count");

__device__ __forceinline__ void load_params(float* sw, const float* w) {
  for (int p = threadIdx.x; p < kP; p += blockDim.x) sw[p] = w[p];
}

// Forward pass of two rows for inference.  The second hidden layer's
// activations are folded into the output as they are produced
// (o_s += W3[s][a] relu(z_a), a ascending -- the same fused multiply-adds in
// the same order as the training pass), so h2 needs no registers, and every
// weight read from shared memory serves both rows (half the shared-memory
// traffic per fused multiply-add).
__device__ __forceinline__ void forward_infer2(const float* sw, const float (&f0)[S],
                                               const float (&f1)[S], float (&o0)[S],
                                               float (&o1)[S]) {
  float h0[H], h1[H];
#pragma unroll
  for (int a = 0; a < H; ++a) {
    float z0 = sw[ob1 + a], z1 = z0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const float wv = sw[oW1 + a * S + s];
      z0 = fmaf(wv, f0[s], z0);
      z1 = fmaf(wv, f1[s], z1);
    }
    h0[a] = fmaxf(z0, 0.0f);
    h1[a] = fmaxf(z1, 0.0f);
  }
#pragma unroll
  for (int s = 0; s < S; ++s) o0[s] = o1[s] = sw[ob3 + s];
#pragma unroll 2
  for (int a = 0; a < H; ++a) {
    float z0 = sw[ob2 + a], z1 = z0;
#pragma unroll
    for (int b = 0; b < H; ++b) {
      const float wv = sw[oW2 + a * H + b];
      z0 = fmaf(wv, h0[b], z0);
      z1 = fmaf(wv, h1[b], z1);
    }
    const float r0 = fmaxf(z0, 0.0f), r1 = fmaxf(z1, 0.0f);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const float wv = sw[oW3 + s * H + a];
      o0[s] = fmaf(wv, r0, o0[s]);
      o1[s] = fmaf(wv, r1, o1[s]);
    }
  }
}

// Forward pass writing the activations to a per-row stage `my` (f at 0,
// h1 at S, h2 at S + H): bounded register use for the training kernel.
__device__ __forceinline__ void forward_staged(const float* sw,
                                               const float (&f)[S], float* my,
                                               float (&o)[S]) {
  float h1[H];
#pragma unroll
  for (int a = 0; a < H; ++a) {
    float z = sw[ob1 + a];
#pragma unroll
    for (int s = 0; s < S; ++s) z = fmaf(sw[oW1 + a * S + s], f[s], z);
    h1[a] = fmaxf(z, 0.0f);
    my[S + a] = h1[a];
  }
#pragma unroll 1
  for (int a = 0; a < H; ++a) {
    float z = sw[ob2 + a];
#pragma unroll
    for (int b = 0; b < H; ++b) z = fmaf(sw[oW2 + a * H + b], h1[b], z);
    my[S + H + a] = fmaxf(z, 0.0f);
  }
#pragma unroll
  for (int s = 0; s < S; ++s) o[s] = sw[ob3 + s];
#pragma unroll 4
  for (int b = 0; b < H; ++b) {
    const float hb = my[S + H + b];
#pragma unroll
    for (int s = 0; s < S; ++s) o[s] = fmaf(sw[oW3 + s * H + b], hb, o[s]);
  }
}

}  // namespace

// Features and 1/a_ii of every row.  slot_entry[i*S + s]: CSR index of the
// row's entry on slot s, or -1.
__global__ void k_spai_features(int n, const int* __restrict__ rowptr,
                                const double* __restrict__ val,
                                const int* __restrict__ slot_entry,
                                float* __restrict__ feat,
                                float* __restrict__ dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ed = slot_entry[i * S + kCenterSlot];
  const double d = ed >= 0 ? val[ed] : 0.0;
  const double di = d != 0.0 ? 1.0 / d : 0.0;
  double rowsum = 0.0;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) rowsum += val[k];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int e = slot_entry[i * S + s];
    float v = 0.0f;
    if (s == kCenterSlot) v = (float)(rowsum * di);
    else if (e >= 0) v = (float)(val[e] * di);
    feat[i * S + s] = v;
  }
  dinv[i] = (float)di;
}

// Inference: M values on A's pattern (entries without a slot get 0).  Each
// thread evaluates rows i and i + blockDim.x of its CTA's 2 * blockDim.x.
constexpr int kInferThreads = 128;

__global__ void __launch_bounds__(kInferThreads)
k_spai_infer(int n, const float* __restrict__ w, const float* __restrict__ feat,
             const float* __restrict__ dinv, const int* __restrict__ slot_entry,
             float* __restrict__ mval) {
  __shared__ float sw[kP];
  load_params(sw, w);
  __syncthreads();
  const int i0 = blockIdx.x * (2 * kInferThreads) + threadIdx.x;
  const int i1 = i0 + kInferThreads;
  if (i0 >= n) return;
  const bool two = i1 < n;
  float f0[S], f1[S], o0[S], o1[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    f0[s] = feat[(long long)i0 * S + s];
    f1[s] = two ? feat[(long long)i1 * S + s] : 0.0f;
  }
  forward_infer2(sw, f0, f1, o0, o1);
  const float d0 = dinv[i0];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int e = slot_entry[(long long)i0 * S + s];
    if (e >= 0) mval[e] = o0[s] * d0;
  }
  if (two) {
    const float d1 = dinv[i1];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int e = slot_entry[(long long)i1 * S + s];
      if (e >= 0) mval[e] = o1[s] * d1;
    }
  }
}

// One training pass over rows [0, n): loss partial and weight-gradient
// partials per CTA.  Z and AZ are column-major probe blocks (probes x ldz).
// `col` maps a slot's CSR entry to its column.
constexpr int kTrainThreads = 128;
// Per-row stage: f, h1, h2, dh1, dh2, do; odd stride (273 floats) so each
// thread's own row is bank-conflict free.
constexpr int kStage = S + H + H + H + H + S + 1;

__global__ void __launch_bounds__(kTrainThreads)
k_spai_grad(int n, const float* __restrict__ w, const float* __restrict__ feat,
            const float* __restrict__ dinv, const int* __restrict__ slot_entry,
            const int* __restrict__ col, const float* __restrict__ Z,
            const float* __restrict__ AZ, int probes, long long ldz,
            float scale, float* __restrict__ gpart, float* __restrict__ lpart) {
  extern __shared__ float smem[];
  float* sw = smem;                      // kP
  float* st = smem + kP;                 // kTrainThreads x kStage
  load_params(sw, w);
  __syncthreads();
  const int t = threadIdx.x;
  const int i = blockIdx.x * kTrainThreads + t;
  float* my = st + t * kStage;
  float loss = 0.0f;
  if (i < n) {
    float o[S];
    {
      // Activations go to the stage (also needed by the CTA reduction
      // below); the backward pass reads them back.
      float f[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        f[s] = feat[i * S + s];
        my[s] = f[s];
      }
      forward_staged(sw, f, my, o);
    }
    const float di = dinv[i];
    int cj[S];
    float m[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int e = slot_entry[i * S + s];
      cj[s] = e >= 0 ? col[e] : -1;
      m[s] = e >= 0 ? o[s] * di : 0.0f;
    }
    float dm[S];
#pragma unroll
    for (int s = 0; s < S; ++s) dm[s] = 0.0f;
    for (int c = 0; c < probes; ++c) {
      const float* azc = AZ + (long long)c * ldz;
      float r = Z[(long long)c * ldz + i];
      float wv[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        wv[s] = cj[s] >= 0 ? azc[cj[s]] : 0.0f;
        r = fmaf(-m[s], wv[s], r);
      }
      loss = fmaf(r, r, loss);
#pragma unroll
      for (int s = 0; s < S; ++s) dm[s] = fmaf(-2.0f * r, wv[s], dm[s]);
    }
    float dout[S];
#pragma unroll
    for (int s = 0; s < S; ++s) dout[s] = cj[s] >= 0 ? dm[s] * di * scale : 0.0f;
    float dh2[H];
#pragma unroll
    for (int b = 0; b < H; ++b) {
      float z = 0.0f;
#pragma unroll
      for (int s = 0; s < S; ++s) z = fmaf(sw[oW3 + s * H + b], dout[s], z);
      dh2[b] = my[S + H + b] > 0.0f ? z : 0.0f;
      my[S + 3 * H + b] = dh2[b];
    }
#pragma unroll 1
    for (int b = 0; b < H; ++b) {
      float z = 0.0f;
#pragma unroll
      for (int a = 0; a < H; ++a) z = fmaf(sw[oW2 + a * H + b], dh2[a], z);
      my[S + 2 * H + b] = my[S + b] > 0.0f ? z : 0.0f;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) my[S + 4 * H + s] = dout[s];
  } else {
    for (int q = 0; q < kStage; ++q) my[q] = 0.0f;
  }
  __syncthreads();
  // CTA reduction of the outer products into this CTA's gradient partial.
  const int rows = kTrainThreads;
  for (int p = t; p < kP; p += kTrainThreads) {
    float g = 0.0f;
    if (p < ob1) {                       // W1[a][s] += dh1[a] f[s]
      const int a = p / S, s = p % S;
      for (int r = 0; r < rows; ++r)
        g = fmaf(st[r * kStage + S + 2 * H + a], st[r * kStage + s], g);
    } else if (p < oW2) {                // b1[a] += dh1[a]
      const int a = p - ob1;
      for (int r = 0; r < rows; ++r) g += st[r * kStage + S + 2 * H + a];
    } else if (p < ob2) {                // W2[a][b] += dh2[a] h1[b]
      const int a = (p - oW2) / H, b = (p - oW2) % H;
      for (int r = 0; r < rows; ++r)
        g = fmaf(st[r * kStage + S + 3 * H + a], st[r * kStage + S + b], g);
    } else if (p < oW3) {                // b2[a] += dh2[a]
      const int a = p - ob2;
      for (int r = 0; r < rows; ++r) g += st[r * kStage + S + 3 * H + a];
    } else if (p < ob3) {                // W3[s][b] += do[s] h2[b]
      const int s = (p - oW3) / H, b = (p - oW3) % H;
      for (int r = 0; r < rows; ++r)
        g = fmaf(st[r * kStage + S + 4 * H + s], st[r * kStage + S + H + b], g);
    } else {                             // b3[s] += do[s]
      const int s = p - ob3;
      for (int r = 0; r < rows; ++r) g += st[r * kStage + S + 4 * H + s];
    }
    gpart[(long long)blockIdx.x * kP + p] = g;
  }
  // Loss partial (fixed-order block tree).
  __shared__ float lw[kTrainThreads / 32];
  float v = loss;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((t & 31) == 0) lw[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    float s = 0.0f;
    for (int k = 0; k < kTrainThreads / 32; ++k) s += lw[k];
    lpart[blockIdx.x] = s;
  }
}

// Sum the per-CTA partials (fixed order) into grad[] and loss; optionally
// apply one Adam step (step >= 1).
__global__ void k_spai_reduce_adam(int nblk, const float* __restrict__ gpart,
                                   const float* __restrict__ lpart,
                                   float* __restrict__ grad, double* loss,
                                   float loss_scale, float* w, float* am,
                                   float* av, int step, float lr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {
    double l = 0.0;
    for (int b = 0; b < nblk; ++b) l += (double)lpart[b];
    *loss = l * (double)loss_scale;
  }
  if (p >= kP) return;
  float g = 0.0f;
  for (int b = 0; b < nblk; ++b) g += gpart[(long long)b * kP + p];
  grad[p] = g;
  if (step <= 0) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float m = b1 * am[p] + (1.0f - b1) * g;
  const float v = b2 * av[p] + (1.0f - b2) * g * g;
  am[p] = m;
  av[p] = v;
  const float mh = m / (1.0f - powf(b1, (float)step));
  const float vh = v / (1.0f - powf(b2, (float)step));
  w[p] -= lr * mh / (sqrtf(vh) + eps);
}

// Rademacher probes: Z[c][i] = +-1 from a counter hash (seeded).
__global__ void k_spai_probes(int n, int probes, long long ldz, uint32_t seed,
                              float* __restrict__ Z) {
  const long long total = (long long)probes * ldz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long i = q % ldz;
    uint32_t h = (uint32_t)q * 2654435761u ^ seed;
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    Z[q] = i < n ? ((h & 1u) ? 1.0f : -1.0f) : 0.0f;
  }
}

// ---------------------------------------------------------------- launches

void launch_spai_features(int n, const int* rowptr, const double* val,
                          const int* slot_entry, float* feat, float* dinv,
                          cudaStream_t st) {
  ++launch_count();
  k_spai_features<<<(n + 255) / 256, 256, 0, st>>>(n, rowptr, val, slot_entry,
                                                  feat, dinv);
}

struct SlotTable {
  int so[kSlots], sl[kSlots];
  int ns;
};

__global__ void __launch_bounds__(256)
k_spai_slot_map(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                SlotTable t, int* __restrict__ slot_entry) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int e[kSlots];
#pragma unroll
  for (int s = 0; s < kSlots; ++s) e[s] = -1;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    const int o = col[k] - i;
#pragma unroll
    for (int q = 0; q < kSlots; ++q)
      if (q < t.ns && t.so[q] == o && e[t.sl[q]] < 0) e[t.sl[q]] = k;
  }
#pragma unroll
  for (int s = 0; s < kSlots; ++s) slot_entry[(long long)i * kSlots + s] = e[s];
}

// out = (M + M^T) / 2 on M's pattern, which is A's pattern and symmetric
// for the symmetric operators this serves (CG): entry (i, j) averages with
// the first stored (j, i); an entry without a transposed partner keeps its
// own value.  One thread per row.
__global__ void __launch_bounds__(256)
k_spai_symmetrize(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                  const float* __restrict__ in, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    const int j = col[k];
    float v = in[k];
    if (j != i && j >= 0 && j < n) {
      for (int kk = rowptr[j]; kk < rowptr[j + 1]; ++kk) {
        if (col[kk] == i) {
          v = (float)(0.5 * ((double)in[k] + (double)in[kk]));
          break;
        }
      }
    }
    out[k] = v;
  }
}

void launch_spai_symmetrize(int n, const int* rowptr, const int* col,
                            const float* in, float* out, cudaStream_t st) {
  ++launch_count();
  k_spai_symmetrize<<<(n + 255) / 256, 256, 0, st>>>(n, rowptr, col, in, out);
}

void launch_spai_slot_map(int n, const int* rowptr, const int* col,
                          const int* so, const int* sl, int ns, int* slot_entry,
                          cudaStream_t st) {
  ++launch_count();
  SlotTable t{};
  for (int q = 0; q < ns && q < kSlots; ++q) {
    t.so[q] = so[q];
    t.sl[q] = sl[q];
  }
  t.ns = ns < kSlots ? ns : kSlots;
  k_spai_slot_map<<<(n + 255) / 256, 256, 0, st>>>(n, rowptr, col, t, slot_entry);
}

void launch_spai_infer(int n, const float* w, const float* feat,
                       const float* dinv, const int* slot_entry, float* mval,
                       cudaStream_t st) {
  ++launch_count();
  const int rows_per_cta = 2 * kInferThreads;
  k_spai_infer<<<(n + rows_per_cta - 1) / rows_per_cta, kInferThreads, 0, st>>>(
      n, w, feat, dinv, slot_entry, mval);
}

int spai_grad_blocks(int n) { return (n + kTrainThreads - 1) / kTrainThreads; }

void launch_spai_grad(int n, const float* w, const float* feat,
                      const float* dinv, const int* slot_entry, const int* col,
                      const float* Z, const float* AZ, int probes,
                      long long ldz, float scale, float* gpart, float* lpart,
                      cudaStream_t st) {
  ++launch_count();
  const size_t sm = sizeof(float) * (kP + kTrainThreads * kStage);
  // The shared-memory attribute is per device: set it once on each.
  static std::mutex mu;
  static unsigned long long devs_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && !((devs_set >> dev) & 1ull)) {
      cudaFuncSetAttribute(k_spai_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
      devs_set |= 1ull << dev;
    }
  }
  k_spai_grad<<<spai_grad_blocks(n), kTrainThreads, sm, st>>>(
      n, w, feat, dinv, slot_entry, col, Z, AZ, probes, ldz, scale, gpart, lpart);
}

void launch_spai_reduce_adam(int nblk, const float* gpart, const float* lpart,
                             float* grad, double* loss, float loss_scale,
                             float* w, float* am, float* av, int step, float lr,
                             cudaStream_t st) {
  ++launch_count();
  k_spai_reduce_adam<<<(kP + 255) / 256, 256, 0, st>>>(
      nblk, gpart, lpart, grad, loss, loss_scale, w, am, av, step, lr);
}

void launch_spai_probes(int n, int probes, long long ldz, uint32_t seed,
                        float* Z, cudaStream_t st) {
  ++launch_count();
  k_spai_probes<<<148 * 4, 256, 0, st>>>(n, probes, ldz, seed, Z);
}

}  // namespace bk
