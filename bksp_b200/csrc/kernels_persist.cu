// The persistent loop: one cooperative kernel that runs a solve's recorded
// iteration (kernel_api.h: ProgOpH) for every system of a batch until each
// has converged or spent its budget.
//
// Execution.  Phase k of a trip runs operation k of every system still
// iterating (not done, trip below its cap, guard slot non-zero).  The
// phase's work is the concatenation of those systems' units (kPersistUnit
// rows or elements each); CTA b takes units b, b + G, b + 2G, ... of it, so
// a phase spreads over the whole grid however the rows divide between
// systems, and systems that have converged cost nothing.  A grid barrier
// ends the phase; scalar epilogues run inside the phase, by the last CTA
// that worked on the system (per-system arrival ticket), exactly as the
// last block of a stand-alone launch runs them.
//
// Determinism.  A CTA's contribution to a system is published in the slot
// given by its position among that system's contributors ((b - first unit)
// mod G), and the last arrival sums the slots in slot order, so the sums do
// not depend on arrival order.  Per element the arithmetic is the
// stand-alone kernels' (k_spmv_dia's row order, k_lincomb's term order).
//
// Memory.  Vectors are written in one phase and read in later ones by other
// SMs, so every vector load here goes through L2 (ld.global.cg); only the
// operator's values, columns and masks, which no phase writes, use the
// read-only path.
//
// Waits.  The only waits are the grid barriers; each gives up after
// spin_limit polls, records the phase, and every CTA then returns (a CTA
// that sees the error flag stops waiting), so the kernel always ends.
#include <cstdio>
#include <mutex>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_spmv.cuh"
#include "kernel_api.h"
#include "launch_util.h"

namespace bk {

namespace {

constexpr int kPAcc = kPersistGramMax * (kPersistGramMax + 1) / 2;   // 15

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T>
__device__ __forceinline__ T ldv(const T* p) { return __ldcg(p); }

// Scalar-slot coefficient, read through L2 (slots change between phases).
__device__ __forceinline__ double pcf(const Cf& c, const double* S) {
  switch (c.op) {
    case 1: return c.k;
    case 2: return c.k * __ldcg(S + c.s);
    case 3: return c.k / __ldcg(S + c.s);
    case 4: return c.k * __ldcg(S + c.s) / __ldcg(S + c.s2);
    case 5: return c.k * __ldcg(S + c.s) * __ldcg(S + c.s2);
    default: return 0.0;
  }
}

// ------------------------------------------------------------- barrier

__device__ bool pbarrier(const PersistH& P, int phase) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    PBarH* b = P.bar;
    int ok = 1;
    if ((int)blockIdx.x == P.absent_cta) {
      ok = 0;   // test hook: this CTA never arrives
    } else {
      // The generation cannot move before this CTA arrives, so reading it
      // first and then arriving cannot miss the release.
      const unsigned g0 = ld_acquire_u32(&b->gen);
      __threadfence();
      const unsigned t = atomicAdd(&b->count, 1u);
      if (t == gridDim.x - 1) {
        atomicExch(&b->count, 0u);
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        long long polls = 0;
        while (ld_acquire_u32(&b->gen) == g0) {
          if (ld_relaxed_i32(&b->err)) {
            ok = 0;
            break;
          }
          if (++polls > P.spin_limit) {
            if (atomicCAS(&b->err, 0, 1) == 0) b->err_phase = phase;
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
      if (ok && ld_relaxed_i32(&b->err)) ok = 0;
    }
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// ------------------------------------------------------- shared state

struct PShared {
  int u[kPersistMaxSys];           // units of each system in this phase
  long long pre[kPersistMaxSys + 1];   // exclusive prefix of u
  long long wsum[kWarps];
  ProgOpH op;                      // the current system's operation
  double cs[kLcMaxOut][kLcMaxIn];  // its linear-combination coefficients
  unsigned pm[kLcMaxOut];          // ... and which terms are present
  double red[kPAcc][kWarps];
  double acc[kPAcc][kThreads];     // per-thread partial dots of the system
  int flag;
};

// Fold a unit's partial dots into the thread's running sums.
template <int N>
__device__ __forceinline__ void add_acc(PShared& sh, const double (&a)[N], int nd) {
#pragma unroll
  for (int d = 0; d < N; ++d)
    if (d < nd) sh.acc[d][threadIdx.x] += a[d];
}

// Exclusive prefix sum of sh.u[0..nsys) into sh.pre[0..nsys].
__device__ void scan_units(PShared& sh, int nsys) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per = (nsys + kThreads - 1) / kThreads;
  const int a = threadIdx.x * per;
  const int e = a + per < nsys ? a + per : nsys;
  long long loc = 0;
  for (int i = a; i < e; ++i) loc += sh.u[i];
  long long v = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) sh.wsum[warp] = v;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < kWarps ? sh.wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < kWarps) sh.wsum[lane] = w;
  }
  __syncthreads();
  long long base = (warp ? sh.wsum[warp - 1] : 0) + v - loc;
  for (int i = a; i < e; ++i) {
    sh.pre[i] = base;
    base += sh.u[i];
  }
  if (threadIdx.x == 0) sh.pre[nsys] = sh.wsum[kWarps - 1];
  __syncthreads();
}

// ------------------------------------------------------------ units

// Diagonal-form SpMV on rows [unit * kPersistUnit, +kPersistUnit): four
// consecutive rows per thread, k_spmv_dia's arithmetic.
template <typename T>
__device__ __noinline__ void u_spmv_dia(PShared& sh, const CsrH& A,
                                        const SpmvH<T>& io, long long unit) {
  const int n = A.n;
  const int i0 = (int)(unit * kPersistUnit) + 4 * (int)threadIdx.x;
  if (i0 >= n) return;
  double acc[3] = {0.0, 0.0, 0.0};
  const T* __restrict__ V = static_cast<const T*>(A.dia.val);
  const long long stride = A.dia.stride;
  const unsigned m = __ldg(reinterpret_cast<const unsigned*>(A.dia.mask + i0));
  T bv[4], w0[4], w1[4], sum[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const bool in = i0 + e < n;
    bv[e] = (io.b && in) ? ldv(io.b + i0 + e) : T(0);
    w0[e] = (io.w0 && in) ? ldv(io.w0 + i0 + e) : T(0);
    w1[e] = (io.w1 && in) ? ldv(io.w1 + i0 + e) : T(0);
    sum[e] = T(0);
  }
#pragma unroll
  for (int d = 0; d < kDiaMax; ++d) {
    if (d < A.dia.nd) {
      const int o = A.dia.off[d];
      T v[4], xv[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        v[e] = __ldg(V + d * stride + i0 + e);
        const int j = i0 + e + o;
        xv[e] = (j >= 0 && j < n) ? ldv(io.x + j) : T(0);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if ((m >> (8 * e + d)) & 1u) sum[e] = add_rn(sum[e], mul_rn(v[e], xv[e]));
    }
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (i0 + e < n) {
      const T y = io.mode == 1 ? add_rn(bv[e], -sum[e]) : sum[e];
      io.y[i0 + e] = y;
      if (io.y2) io.y2[i0 + e] = y;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < io.nd)
          acc[d] += (double)spmv_operand(io.dot[d][0], y, bv[e], w0[e], w1[e]) *
                    (double)spmv_operand(io.dot[d][1], y, bv[e], w0[e], w1[e]);
    }
  }
  add_acc<3>(sh, acc, io.nd);
}

// CSR SpMV, one thread per row (rows unit * kPersistUnit + t + 256 e): the
// row's entries in stored order, y = 0; y += a_k x_k without FMA.
template <typename T>
__device__ __noinline__ void u_spmv_csr(PShared& sh, const CsrH& A,
                                        const SpmvH<T>& io, long long unit) {
  const T* __restrict__ val = static_cast<const T*>(A.val);
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
  for (int e = 0; e < kPersistUnit / kThreads; ++e) {
    const int i = (int)(unit * kPersistUnit) + e * kThreads + (int)threadIdx.x;
    if (i >= A.n) break;
    const int k0 = __ldg(A.rowptr + i), k1 = __ldg(A.rowptr + i + 1);
    T sum = T(0);
    for (int k = k0; k < k1; ++k)
      sum = add_rn(sum, mul_rn(__ldg(val + k), ldv(io.x + __ldg(A.col + k))));
    const T bv = io.b ? ldv(io.b + i) : T(0);
    const T w0 = io.w0 ? ldv(io.w0 + i) : T(0);
    const T w1 = io.w1 ? ldv(io.w1 + i) : T(0);
    const T y = io.mode == 1 ? add_rn(bv, -sum) : sum;
    io.y[i] = y;
    if (io.y2) io.y2[i] = y;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < io.nd)
        acc[d] += (double)spmv_operand(io.dot[d][0], y, bv, w0, w1) *
                  (double)spmv_operand(io.dot[d][1], y, bv, w0, w1);
  }
  add_acc<3>(sh, acc, io.nd);
}

// Linear combination on one unit: rep = unit / chunks, elements
// [chunk * kPersistUnit, +kPersistUnit) of that repetition; per element
// k_lincomb's arithmetic (first present term a rounded product, the others
// fused multiply-adds, in input order).
// Two-element packets (float2 / double2) for the linear combination: its
// six outputs, three dot operand pairs and four inputs in flight stay in
// registers.
template <typename T> struct Pair;
template <> struct Pair<float> { using V = float2; };
template <> struct Pair<double> { using V = double2; };

template <typename T>
__device__ __forceinline__ void unpack2(const typename Pair<T>::V& p, T* e) {
  e[0] = p.x;
  e[1] = p.y;
}

template <typename T>
__device__ __noinline__ void u_lincomb(PShared& sh, const LcH<T>& d,
                                       long long unit) {
  double acc[3] = {0.0, 0.0, 0.0};
  using PV = typename Pair<T>::V;
  constexpr int P = 2;
  constexpr int PER = kPersistUnit / (kThreads * P);   // packets per thread
  const long long chunks = (d.n + kPersistUnit - 1) / kPersistUnit;
  const long long rep = unit / chunks, chunk = unit - rep * chunks;
  const long long off = rep * d.stride;
  const long long npk = d.n / P;
#pragma unroll 1
  for (int h = 0; h < PER; ++h) {
    const long long q = chunk * (kPersistUnit / P) + h * kThreads + threadIdx.x;
    if (q >= npk) break;
    T r[kLcMaxOut][P];
    bool first[kLcMaxOut];
#pragma unroll
    for (int o = 0; o < kLcMaxOut; ++o) first[o] = true;
    T da[3][P], db[3][P];
    // Inputs in groups of four: the group's loads are in flight together,
    // then folded in input order.
#pragma unroll 1
    for (int i0 = 0; i0 < d.nin; i0 += 4) {
      T v[4][P];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = i0 + j;
        if (i < d.nin) {
          const T* p = d.in[i] + ((d.in_rep_mask >> i) & 1u ? off : 0);
          unpack2<T>(ldv(reinterpret_cast<const PV*>(p) + q), v[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = i0 + j;
        if (i < d.nin) {
#pragma unroll
          for (int o = 0; o < kLcMaxOut; ++o) {
            if ((sh.pm[o] >> i) & 1u) {
              const T cf = (T)sh.cs[o][i];
#pragma unroll
              for (int e = 0; e < P; ++e)
                r[o][e] = first[o] ? mul_rn(cf, v[j][e]) : fma_rn(cf, v[j][e], r[o][e]);
              first[o] = false;
            }
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            if (k < d.nd && d.dot[k][0] == i)
#pragma unroll
              for (int e = 0; e < P; ++e) da[k][e] = v[j][e];
            if (k < d.nd && d.dot[k][1] == i)
#pragma unroll
              for (int e = 0; e < P; ++e) db[k][e] = v[j][e];
          }
        }
      }
    }
#pragma unroll
    for (int o = 0; o < kLcMaxOut; ++o) {
      if (o < d.nout) {
        if (first[o])
#pragma unroll
          for (int e = 0; e < P; ++e) r[o][e] = T(0);
        T* p = d.out[o] + ((d.out_rep_mask >> o) & 1u ? off : 0);
        PV w;
        w.x = r[o][0];
        w.y = r[o][1];
        reinterpret_cast<PV*>(p)[q] = w;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k < d.nd && d.dot[k][0] == d.nin + o)
#pragma unroll
            for (int e = 0; e < P; ++e) da[k][e] = r[o][e];
          if (k < d.nd && d.dot[k][1] == d.nin + o)
#pragma unroll
            for (int e = 0; e < P; ++e) db[k][e] = r[o][e];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (k < d.nd)
#pragma unroll
        for (int e = 0; e < P; ++e) acc[k] += (double)da[k][e] * (double)db[k][e];
  }
  add_acc<3>(sh, acc, d.nd);
}

// Pairwise Gram products <v_i, v_j>, i <= j < M, on one unit.
template <typename T, int M>
__device__ __noinline__ void u_gram_m(PShared& sh, const GramH<T>& g,
                                      long long unit) {
  constexpr int NP = M * (M + 1) / 2;
  double acc[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) acc[q] = 0.0;
  using PV = typename Pack<T>::V;
  constexpr int P = Pack<T>::N;
  constexpr int PER = kPersistUnit / (kThreads * P);
  const long long npk = g.n / P;
#pragma unroll 1
  for (int h = 0; h < PER; ++h) {
    const long long q = unit * (kPersistUnit / P) + h * kThreads + threadIdx.x;
    if (q >= npk) break;
    T v[M][P];
#pragma unroll
    for (int i = 0; i < M; ++i) unpack<T>(ldv(reinterpret_cast<const PV*>(g.v[i]) + q), v[i]);
    int idx = 0;
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
      for (int j = i; j < M; ++j) {
        double s = 0.0;
#pragma unroll
        for (int e = 0; e < P; ++e) s += (double)v[i][e] * (double)v[j][e];
        acc[idx++] += s;
      }
  }
  add_acc<NP>(sh, acc, NP);
}

template <typename T>
__device__ void u_gram(PShared& sh, const GramH<T>& g, long long unit) {
  switch (g.m) {
    case 1: u_gram_m<T, 1>(sh, g, unit); break;
    case 2: u_gram_m<T, 2>(sh, g, unit); break;
    case 3: u_gram_m<T, 3>(sh, g, unit); break;
    case 4: u_gram_m<T, 4>(sh, g, unit); break;
    default: u_gram_m<T, 5>(sh, g, unit); break;
  }
}

__device__ __noinline__ void u_d2f(PShared& sh, const MxD2fH& a, long long unit) {
  double acc[1] = {0.0};
#pragma unroll 1
  for (int e = 0; e < kPersistUnit / kThreads; ++e) {
    const long long i = unit * kPersistUnit + e * kThreads + threadIdx.x;
    if (i >= a.n) break;
    const float v = (float)ldv(a.in + i);
    const float wv = (a.nd > 0 && a.w) ? ldv(a.w + i) : v;   // before any store
    a.o0[i] = v;
    if (a.o1) a.o1[i] = v;
    if (a.o2) a.o2[i] = v;
    if (a.nd > 0) acc[0] += (double)wv * (double)v;
  }
  add_acc<1>(sh, acc, a.nd);
}

__device__ __noinline__ void u_accum(const MxAccH& a, long long unit) {
#pragma unroll 1
  for (int e = 0; e < kPersistUnit / kThreads; ++e) {
    const long long i = unit * kPersistUnit + e * kThreads + threadIdx.x;
    if (i >= a.n) break;
    a.x[i] = ldv(a.x + i) + (double)ldv(a.t + i);
    a.y[i] = 0.0f;
  }
}

// Dots an operation reduces.
__device__ __forceinline__ int op_dots(const ProgOpH& op) {
  switch (op.kind) {
    case kOpSpmvDiaD: case kOpSpmvCsrD: return op.u.sd.io.nd;
    case kOpSpmvDiaF: case kOpSpmvCsrF: return op.u.sf.io.nd;
    case kOpLcD: return op.u.ld.nd;
    case kOpLcF: return op.u.lf.nd;
    case kOpGramD: return op.u.gd.m * (op.u.gd.m + 1) / 2;
    case kOpGramF: return op.u.gf.m * (op.u.gf.m + 1) / 2;
    case kOpMxD2f: return op.u.d2f.nd;
    default: return 0;
  }
}

// Load system `sys`'s operation k into shared memory and prepare it.
__device__ void load_op(PShared& sh, const PersistH& P, int sys, int k) {
  __syncthreads();   // the previous operation's readers are done
  const int4* src = reinterpret_cast<const int4*>(P.ops + (long long)sys * P.max_ops + k);
  int4* dst = reinterpret_cast<int4*>(&sh.op);
  constexpr int W = (int)(sizeof(ProgOpH) / sizeof(int4));
  static_assert(sizeof(ProgOpH) % sizeof(int4) == 0, "operation record size");
  for (int w = threadIdx.x; w < W; w += kThreads) dst[w] = __ldcg(src + w);
  __syncthreads();
  const ProgOpH& op = sh.op;
  if (op.kind == kOpLcD || op.kind == kOpLcF) {
    const int nin = op.kind == kOpLcD ? op.u.ld.nin : op.u.lf.nin;
    const int nout = op.kind == kOpLcD ? op.u.ld.nout : op.u.lf.nout;
    for (int t = threadIdx.x; t < kLcMaxOut * kLcMaxIn; t += kThreads) {
      const int o = t / kLcMaxIn, i = t % kLcMaxIn;
      const Cf& c = op.kind == kOpLcD ? op.u.ld.c[o][i] : op.u.lf.c[o][i];
      sh.cs[o][i] = (o < nout && i < nin) ? pcf(c, op.rd.S) : 0.0;
    }
    if (threadIdx.x < kLcMaxOut) {
      unsigned m = 0;
      for (int i = 0; i < kLcMaxIn; ++i) {
        const Cf& c = op.kind == kOpLcD ? op.u.ld.c[threadIdx.x][i] : op.u.lf.c[threadIdx.x][i];
        if ((int)threadIdx.x < nout && i < nin && c.op) m |= 1u << i;
      }
      sh.pm[threadIdx.x] = m;
    }
    __syncthreads();
  }
}

__device__ void run_unit(PShared& sh, long long unit) {
  const ProgOpH& op = sh.op;
  switch (op.kind) {
    case kOpSpmvDiaD: u_spmv_dia<double>(sh, op.u.sd.A, op.u.sd.io, unit); break;
    case kOpSpmvDiaF: u_spmv_dia<float>(sh, op.u.sf.A, op.u.sf.io, unit); break;
    case kOpSpmvCsrD: u_spmv_csr<double>(sh, op.u.sd.A, op.u.sd.io, unit); break;
    case kOpSpmvCsrF: u_spmv_csr<float>(sh, op.u.sf.A, op.u.sf.io, unit); break;
    case kOpLcD: u_lincomb<double>(sh, op.u.ld, unit); break;
    case kOpLcF: u_lincomb<float>(sh, op.u.lf, unit); break;
    case kOpGramD: u_gram<double>(sh, op.u.gd, unit); break;
    case kOpGramF: u_gram<float>(sh, op.u.gf, unit); break;
    case kOpMxD2f: u_d2f(sh, op.u.d2f, unit); break;
    case kOpMxAccum: u_accum(op.u.acc, unit); break;
    default: break;
  }
}

// This CTA's contribution to the current system's reductions: block sums
// into the CTA's slot, and the last contributor finishes the sums and runs
// the epilogue.  `first` is the system's first unit in the phase, `units`
// its unit count.
__device__ void flush(PShared& sh, long long first, long long units) {
  const Red rd = sh.op.rd;
  const int nd = op_dots(sh.op);
  if (nd == 0 && rd.epi == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 0; d < nd; ++d) {
    const double v = warp_sum(sh.acc[d][threadIdx.x]);
    if (lane == 0) sh.red[d][warp] = v;
  }
  __syncthreads();
  const long long G = gridDim.x;
  const int C = (int)(units < G ? units : G);
  if (threadIdx.x == 0) {
    double tot[kPAcc];
#pragma unroll
    for (int d = 0; d < kPAcc; ++d) {
      tot[d] = 0.0;
      if (d < nd)
        for (int w = 0; w < kWarps; ++w) tot[d] += sh.red[d][w];
    }
    if (C == 1) {
      for (int d = 0; d < nd; ++d) rd.S[rd.out + d] = tot[d];
      sh.flag = 0;
      if (rd.epi) run_epilogue(rd);
    } else {
      long long j = ((long long)blockIdx.x - first) % G;
      if (j < 0) j += G;
      for (int d = 0; d < nd; ++d) rd.part[d * kMaxBlocks + j] = tot[d];
      unsigned t;
      asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                   : "=r"(t) : "l"(rd.ticket) : "memory");
      sh.flag = (t == (unsigned)C - 1) ? 1 : 0;
    }
  }
  __syncthreads();
  if (!sh.flag) return;
  __threadfence();
  // Last contributor: slot-ordered sums (thread-strided, then warps in
  // order), as finish_reduction does over a launch's blocks.
#pragma unroll
  for (int d = 0; d < kPAcc; ++d) {
    if (d < nd) {
      double v = 0.0;
      for (int b = threadIdx.x; b < C; b += kThreads) v += __ldcg(rd.part + d * kMaxBlocks + b);
      v = warp_sum(v);
      if (lane == 0) sh.red[d][warp] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < nd; ++d) {
      double s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += sh.red[d][w];
      rd.S[rd.out + d] = s;
    }
    *rd.ticket = 0u;
    if (rd.epi) run_epilogue(rd);
  }
  __syncthreads();
}

// One phase: operation k of every system still iterating at trip `trip`.
__device__ void phase(PShared& sh, const PersistH& P, int k, int trip) {
  for (int s = threadIdx.x; s < P.nsys; s += kThreads) {
    int u = 0;
    const CtlH* c = P.ctl[s];
    if (k < P.nops[s] && !finished(c) && trip < c->trip_cap) {
      const ProgOpH* op = P.ops + (long long)s * P.max_ops + k;
      const short g = op->rd.guard;
      if (g <= 0 || __ldcg(op->rd.S + g) != 0.0) u = op->units;
    }
    sh.u[s] = u;
  }
  __syncthreads();
  scan_units(sh, P.nsys);
  const long long T = sh.pre[P.nsys];
  int cur = -1, sys = 0;
  for (long long g = blockIdx.x; g < T; g += gridDim.x) {
    while (sh.pre[sys + 1] <= g) ++sys;
    if (sys != cur) {
      if (cur >= 0) flush(sh, sh.pre[cur], sh.u[cur]);
      cur = sys;
      load_op(sh, P, sys, k);
#pragma unroll
      for (int d = 0; d < kPAcc; ++d) sh.acc[d][threadIdx.x] = 0.0;
    }
    run_unit(sh, g - sh.pre[sys]);
  }
  if (cur >= 0) flush(sh, sh.pre[cur], sh.u[cur]);
}

__global__ void __launch_bounds__(kThreads, 1) k_persist(const PersistH P) {
  __shared__ PShared sh;
  __shared__ int any;
  for (int trip = 0;; ++trip) {
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < P.nsys; s += kThreads) {
      CtlH* c = P.ctl[s];
      if (!finished(c) && trip < c->trip_cap) {
        any = 1;
        if (blockIdx.x == 0) c->trips = trip + 1;
      }
    }
    __syncthreads();
    if (!any) break;
    for (int k = 0; k < P.max_ops; ++k) {
      phase(sh, P, k, trip);
      if (!pbarrier(P, trip * P.max_ops + k)) return;
    }
  }
  // Systems that ran out of trips end as the graph loop's control node
  // ends them.
  if (blockIdx.x == 0) {
    for (int s = threadIdx.x; s < P.nsys; s += kThreads) {
      CtlH* c = P.ctl[s];
      if (!finished(c)) {
        c->done = 1;
        c->ret = kNotConverged;
      }
    }
  }
}

}  // namespace

int persist_max_grid() {
  static std::mutex mu;
  static int cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && cache[dev] > 0) return cache[dev];
  int sms = kSMs, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist, kThreads, 0) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  long long g = (long long)per_sm * sms;
  if (g > kMaxBlocks) g = kMaxBlocks;
  if (dev >= 0 && dev < 64) cache[dev] = (int)g;
  return (int)g;
}

cudaError_t launch_persist(const PersistH& p, int grid, cudaStream_t st) {
  ++launch_count();
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_persist, p);
}

}  // namespace bk
