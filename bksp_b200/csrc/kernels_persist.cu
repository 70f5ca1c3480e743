// The persistent loop: one cooperative kernel that runs a solve's recorded
// iteration (kernel_api.h: ProgOpH) for every system of a batch until each
// has converged or spent its budget.
//
// Execution.  Phase k of a trip runs operation k of every system still
// iterating (not done, trip below its cap, guard slot non-zero).  The
// phase's work is the concatenation of those systems' units (kPersistUnit
// rows or elements each); CTA b takes the contiguous share [T b / G,
// T (b + 1) / G) of its T units, so a phase spreads over the whole grid
// however the rows divide between systems, a CTA meets few systems (one
// operation record to load per system it meets), and systems that have
// converged cost nothing.  A grid barrier ends the phase (a grid of one CTA
// needs only a CTA barrier); scalar epilogues run inside the phase, by the
// last CTA that worked on the system (per-system arrival ticket), as the
// last block of a stand-alone launch runs them.
//
// Determinism.  A CTA's contribution to a system is published in the slot
// given by its position among that system's contributors (CTA b minus the
// CTA holding the system's first unit), and the last arrival sums the slots
// in slot order; within a CTA, per-warp running sums are added in warp
// order.  Sums therefore do not depend on arrival order.  Per element the
// arithmetic is the stand-alone kernels' (k_spmv_dia's and the CSR
// kernels' row order, k_lincomb's term order).
//
// Memory.  Vectors are written in one phase and read in later ones by other
// SMs, so every vector load here goes through L2 (ld.global.cg); only the
// operator's values, columns and masks, which no phase writes, use the
// read-only path.  Every vector operand is 16-byte aligned with a padded
// length (the recording wrappers check), so streams move 16-byte packets.
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

constexpr int kPT = kPersistThreads;       // threads per CTA
constexpr int kPW = kPT / 32;              // warps per CTA
constexpr int kEPT = kPersistUnit / kPT;   // rows / elements per thread and unit
static_assert(kEPT == 4, "four rows or elements per thread and unit");
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

// Four consecutive vector elements p[i .. i+3] through L2 (p + i 16-byte
// aligned), and their store.
__device__ __forceinline__ void ld4(const float* p, long long i, float (&v)[4]) {
  const float4 a = __ldcg(reinterpret_cast<const float4*>(p + i));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void ld4(const double* p, long long i, double (&v)[4]) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p + i));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p + i + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, long long i, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p + i) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, long long i, const double (&v)[4]) {
  *reinterpret_cast<double2*>(p + i) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + i + 2) = make_double2(v[2], v[3]);
}
// Read-only operator values (never written by a phase).
__device__ __forceinline__ void ldg4(const float* p, long long i, float (&v)[4]) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(p + i));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void ldg4(const double* p, long long i, double (&v)[4]) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p + i));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p + i + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

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

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------- barrier

__device__ bool pbarrier(const PersistH& P, int phase) {
  __shared__ int ok_s;
  if (gridDim.x == 1) {   // one CTA: its own barrier orders its memory
    __threadfence_block();
    __syncthreads();
    return true;
  }
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
          __nanosleep(32);
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
  int u[kPersistMaxSys];               // units of each system in this phase
  long long pre[kPersistMaxSys + 1];   // exclusive prefix of u
  CtlH* ctl[kPersistMaxSys];           // each system's control block
  int cap[kPersistMaxSys];             // ... and its trip cap
  long long wsum[kPW];
  ProgOpH op;                          // the current system's operation
  double cs[kLcMaxOut][kLcMaxIn];      // its linear-combination coefficients
  unsigned pm[kLcMaxOut];              // ... and which terms are present
  double acc[kPAcc][kPW];              // per-warp running sums of its dots
  double red[kPAcc][kPW];
  int flag;
};

// The CTA's shared state, at namespace scope so that every function
// addresses it as shared memory (no generic pointer that a global store
// could alias).
__shared__ PShared sh;

template <typename T> __device__ __forceinline__ const SpmvH<T>& sh_io();
template <> __device__ __forceinline__ const SpmvH<double>& sh_io<double>() { return sh.op.u.sd.io; }
template <> __device__ __forceinline__ const SpmvH<float>& sh_io<float>() { return sh.op.u.sf.io; }
template <typename T> __device__ __forceinline__ const CsrH& sh_A();
template <> __device__ __forceinline__ const CsrH& sh_A<double>() { return sh.op.u.sd.A; }
template <> __device__ __forceinline__ const CsrH& sh_A<float>() { return sh.op.u.sf.A; }
template <typename T> __device__ __forceinline__ const LcH<T>& sh_lc();
template <> __device__ __forceinline__ const LcH<double>& sh_lc<double>() { return sh.op.u.ld; }
template <> __device__ __forceinline__ const LcH<float>& sh_lc<float>() { return sh.op.u.lf; }
template <typename T> __device__ __forceinline__ const GramH<T>& sh_gram();
template <> __device__ __forceinline__ const GramH<double>& sh_gram<double>() { return sh.op.u.gd; }
template <> __device__ __forceinline__ const GramH<float>& sh_gram<float>() { return sh.op.u.gf; }

// Fold a unit's per-thread partial dots into the warp's running sums (lane
// 0 adds the warp's total: one fixed order).
template <int N>
__device__ __forceinline__ void add_acc(const double (&a)[N], int nd) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    if (d < nd) {
      const double v = warp_sum_d(a[d]);
      if (lane == 0) sh.acc[d][warp] += v;
    }
  }
}

// Exclusive prefix sum of sh.u[0..nsys) into sh.pre[0..nsys].
__device__ void scan_units(int nsys) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per = (nsys + kPT - 1) / kPT;
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
    long long w = lane < kPW ? sh.wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < kPW) sh.wsum[lane] = w;
  }
  __syncthreads();
  long long base = (warp ? sh.wsum[warp - 1] : 0) + v - loc;
  for (int i = a; i < e; ++i) {
    sh.pre[i] = base;
    base += sh.u[i];
  }
  if (threadIdx.x == 0) sh.pre[nsys] = sh.wsum[kPW - 1];
  __syncthreads();
}

// ------------------------------------------------------------ units

// x[j0 .. j0+3] for a diagonal of offset o, zero outside [0, n): one
// 16-byte packet when the offset keeps j0 on a packet boundary and all
// four exist, else element loads (k_spmv_dia's load_x, through L2).
template <typename T>
__device__ __forceinline__ void load_xd(const T* x, int j0, int o, int n, T (&v)[4]) {
  constexpr int P = 16 / (int)sizeof(T);
  if ((o & (P - 1)) == 0 && j0 >= 0 && j0 + 4 <= n) {
    ld4(x, j0, v);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int j = j0 + e;
      v[e] = (j >= 0 && j < n) ? __ldcg(x + j) : T(0);
    }
  }
}

template <typename T>
__device__ __forceinline__ void load_opnd4(const T* p, int i0, int n, T (&v)[4]) {
  if (!p) {
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = T(0);
  } else if (i0 + 4 <= n) {
    ld4(p, i0, v);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = i0 + e < n ? __ldcg(p + i0 + e) : T(0);
  }
}

// Diagonal-form SpMV on rows [unit * kPersistUnit, +kPersistUnit): four
// consecutive rows per thread, k_spmv_dia's arithmetic.
template <typename T>
__device__ __forceinline__ void u_spmv_dia(long long unit) {
  const CsrH& A = sh_A<T>();
  const SpmvH<T>& io = sh_io<T>();
  const int n = A.n;
  const int i0 = (int)(unit * kPersistUnit) + kEPT * (int)threadIdx.x;
  double acc[3] = {0.0, 0.0, 0.0};
  if (i0 < n) {
    const T* __restrict__ V = static_cast<const T*>(A.dia.val);
    const long long stride = A.dia.stride;
    const unsigned m = __ldg(reinterpret_cast<const unsigned*>(A.dia.mask + i0));
    T bv[4], w0[4], w1[4], sum[4];
    load_opnd4<T>(io.b, i0, n, bv);
    load_opnd4<T>(io.nd ? io.w0 : nullptr, i0, n, w0);
    load_opnd4<T>(io.nd ? io.w1 : nullptr, i0, n, w1);
#pragma unroll
    for (int e = 0; e < 4; ++e) sum[e] = T(0);
    // Diagonals in groups of four: the group's loads are in flight
    // together, then added in ascending diagonal order.
#pragma unroll 1
    for (int d0 = 0; d0 < A.dia.nd; d0 += 4) {
      T v[4][4], xv[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int d = d0 + j;
        if (d < A.dia.nd) {
          const int o = A.dia.off[d];
          ldg4(V + d * stride, i0, v[j]);
          load_xd<T>(io.x, i0 + o, o, n, xv[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int d = d0 + j;
        if (d < A.dia.nd)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if ((m >> (8 * e + d)) & 1u) sum[e] = add_rn(sum[e], mul_rn(v[j][e], xv[j][e]));
      }
    }
    T y[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) y[e] = io.mode == 1 ? add_rn(bv[e], -sum[e]) : sum[e];
    if (i0 + 4 <= n) {
      st4(io.y, i0, y);
      if (io.y2) st4(io.y2, i0, y);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (i0 + e < n) {
          io.y[i0 + e] = y[e];
          if (io.y2) io.y2[i0 + e] = y[e];
        }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (i0 + e < n)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (d < io.nd)
            acc[d] += (double)spmv_operand(io.dot[d][0], y[e], bv[e], w0[e], w1[e]) *
                      (double)spmv_operand(io.dot[d][1], y[e], bv[e], w0[e], w1[e]);
  }
  add_acc<3>(acc, io.nd);
}

// CSR SpMV, one thread per row (rows unit * kPersistUnit + t + kPT e): the
// row's entries in stored order, y = 0; y += a_k x_k without FMA.
template <typename T>
__device__ __forceinline__ void u_spmv_csr(long long unit) {
  const CsrH& A = sh_A<T>();
  const SpmvH<T>& io = sh_io<T>();
  const T* __restrict__ val = static_cast<const T*>(A.val);
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
  for (int e = 0; e < kEPT; ++e) {
    const int i = (int)(unit * kPersistUnit) + e * kPT + (int)threadIdx.x;
    if (i >= A.n) break;
    const int k0 = __ldg(A.rowptr + i), k1 = __ldg(A.rowptr + i + 1);
    T sum = T(0);
    for (int k = k0; k < k1; ++k)
      sum = add_rn(sum, mul_rn(__ldg(val + k), __ldcg(io.x + __ldg(A.col + k))));
    const T bv = io.b ? __ldcg(io.b + i) : T(0);
    const T w0 = io.w0 ? __ldcg(io.w0 + i) : T(0);
    const T w1 = io.w1 ? __ldcg(io.w1 + i) : T(0);
    const T y = io.mode == 1 ? add_rn(bv, -sum) : sum;
    io.y[i] = y;
    if (io.y2) io.y2[i] = y;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < io.nd)
        acc[d] += (double)spmv_operand(io.dot[d][0], y, bv, w0, w1) *
                  (double)spmv_operand(io.dot[d][1], y, bv, w0, w1);
  }
  add_acc<3>(acc, io.nd);
}

// Linear combination on one unit: rep = unit / chunks, elements
// [chunk * kPersistUnit, +kPersistUnit) of that repetition, four per thread
// (processed as two halves of two); per element k_lincomb's arithmetic
// (first present term a rounded product, the others fused multiply-adds,
// in input order).  Inputs are read in groups of four loads in flight.
template <typename T>
__device__ __forceinline__ void u_lincomb(long long unit) {
  const LcH<T>& d = sh_lc<T>();
  double acc[3] = {0.0, 0.0, 0.0};
  const long long chunks = (d.n + kPersistUnit - 1) / kPersistUnit;
  const long long rep = unit / chunks, chunk = unit - rep * chunks;
  const long long off = rep * d.stride;
  const long long i0 = chunk * kPersistUnit + kEPT * (long long)threadIdx.x;
  if (i0 < d.n) {
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const long long ih = i0 + 2 * h;
      T r[kLcMaxOut][2];
      bool first[kLcMaxOut];
#pragma unroll
      for (int o = 0; o < kLcMaxOut; ++o) first[o] = true;
      T da[3][2], db[3][2];
#pragma unroll 1
      for (int g = 0; g < d.nin; g += 4) {
        T v[4][2];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int i = g + j;
          if (i < d.nin) {
            const T* p = d.in[i] + ((d.in_rep_mask >> i) & 1u ? off : 0) + ih;
            if constexpr (sizeof(T) == 8) {
              const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
              v[j][0] = a.x; v[j][1] = a.y;
            } else {
              const float2 a = __ldcg(reinterpret_cast<const float2*>(p));
              v[j][0] = a.x; v[j][1] = a.y;
            }
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int i = g + j;
          if (i < d.nin) {
#pragma unroll
            for (int o = 0; o < kLcMaxOut; ++o) {
              if ((sh.pm[o] >> i) & 1u) {
                const T cf = (T)sh.cs[o][i];
#pragma unroll
                for (int e = 0; e < 2; ++e)
                  r[o][e] = first[o] ? mul_rn(cf, v[j][e]) : fma_rn(cf, v[j][e], r[o][e]);
                first[o] = false;
              }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              if (k < d.nd && d.dot[k][0] == i) { da[k][0] = v[j][0]; da[k][1] = v[j][1]; }
              if (k < d.nd && d.dot[k][1] == i) { db[k][0] = v[j][0]; db[k][1] = v[j][1]; }
            }
          }
        }
      }
#pragma unroll
      for (int o = 0; o < kLcMaxOut; ++o) {
        if (o < d.nout) {
          if (first[o]) { r[o][0] = T(0); r[o][1] = T(0); }
          T* p = d.out[o] + ((d.out_rep_mask >> o) & 1u ? off : 0) + ih;
          if constexpr (sizeof(T) == 8)
            *reinterpret_cast<double2*>(p) = make_double2(r[o][0], r[o][1]);
          else
            *reinterpret_cast<float2*>(p) = make_float2(r[o][0], r[o][1]);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            if (k < d.nd && d.dot[k][0] == d.nin + o) { da[k][0] = r[o][0]; da[k][1] = r[o][1]; }
            if (k < d.nd && d.dot[k][1] == d.nin + o) { db[k][0] = r[o][0]; db[k][1] = r[o][1]; }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (k < d.nd)
#pragma unroll
          for (int e = 0; e < 2; ++e) acc[k] += (double)da[k][e] * (double)db[k][e];
    }
  }
  add_acc<3>(acc, d.nd);
}

// Pairwise Gram products <v_i, v_j>, i <= j < M, on one unit.
template <typename T, int M>
__device__ __forceinline__ void u_gram_m(long long unit) {
  const GramH<T>& g = sh_gram<T>();
  constexpr int NP = M * (M + 1) / 2;
  double acc[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) acc[q] = 0.0;
  const long long i0 = unit * kPersistUnit + kEPT * (long long)threadIdx.x;
  if (i0 < g.n) {
    T v[M][4];
#pragma unroll
    for (int i = 0; i < M; ++i) ld4(g.v[i], i0, v[i]);
    int idx = 0;
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
      for (int j = i; j < M; ++j) {
        double s = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) s += (double)v[i][e] * (double)v[j][e];
        acc[idx++] += s;
      }
  }
  add_acc<NP>(acc, NP);
}

template <typename T>
__device__ void u_gram(long long unit) {
  switch (sh_gram<T>().m) {
    case 1: u_gram_m<T, 1>(unit); break;
    case 2: u_gram_m<T, 2>(unit); break;
    case 3: u_gram_m<T, 3>(unit); break;
    case 4: u_gram_m<T, 4>(unit); break;
    default: u_gram_m<T, 5>(unit); break;
  }
}

__device__ __forceinline__ void u_d2f(long long unit) {
  const MxD2fH& a = sh.op.u.d2f;
  double acc[1] = {0.0};
  const long long i0 = unit * kPersistUnit + kEPT * (long long)threadIdx.x;
  if (i0 < a.n) {
    double in[4];
    ld4(a.in, i0, in);
    float v[4], wv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = (float)in[e];
    if (a.nd > 0 && a.w) ld4(a.w, i0, wv);   // before any store
    else
#pragma unroll
      for (int e = 0; e < 4; ++e) wv[e] = v[e];
    st4(a.o0, i0, v);
    if (a.o1) st4(a.o1, i0, v);
    if (a.o2) st4(a.o2, i0, v);
    if (a.nd > 0)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[0] += (double)wv[e] * (double)v[e];
  }
  add_acc<1>(acc, a.nd);
}

__device__ __forceinline__ void u_accum(long long unit) {
  const MxAccH& a = sh.op.u.acc;
  const long long i0 = unit * kPersistUnit + kEPT * (long long)threadIdx.x;
  if (i0 >= a.n) return;
  double x[4];
  float t[4];
  ld4(a.x, i0, x);
  ld4(a.t, i0, t);
#pragma unroll
  for (int e = 0; e < 4; ++e) x[e] += (double)t[e];
  st4(a.x, i0, x);
  const float z[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  st4(a.y, i0, z);
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
__device__ void load_op(const PersistH& P, int sys, int k) {
  __syncthreads();   // the previous operation's readers are done
  const int4* src = reinterpret_cast<const int4*>(P.ops + (long long)sys * P.max_ops + k);
  int4* dst = reinterpret_cast<int4*>(&sh.op);
  constexpr int W = (int)(sizeof(ProgOpH) / sizeof(int4));
  static_assert(sizeof(ProgOpH) % sizeof(int4) == 0, "operation record size");
  for (int w = threadIdx.x; w < W; w += kPT) dst[w] = __ldcg(src + w);
  if (threadIdx.x < kPAcc * kPW) (&sh.acc[0][0])[threadIdx.x] = 0.0;
  __syncthreads();
  const ProgOpH& op = sh.op;
  if (op.kind == kOpLcD || op.kind == kOpLcF) {
    const int nin = op.kind == kOpLcD ? op.u.ld.nin : op.u.lf.nin;
    const int nout = op.kind == kOpLcD ? op.u.ld.nout : op.u.lf.nout;
    for (int t = threadIdx.x; t < kLcMaxOut * kLcMaxIn; t += kPT) {
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

// Units [a, b) of the current operation: one dispatch per run of units,
// then the operation's loop.
__device__ void run_units(long long a, long long b) {
  switch (sh.op.kind) {
    case kOpSpmvDiaD: for (long long u = a; u < b; ++u) u_spmv_dia<double>(u); break;
    case kOpSpmvDiaF: for (long long u = a; u < b; ++u) u_spmv_dia<float>(u); break;
    case kOpSpmvCsrD: for (long long u = a; u < b; ++u) u_spmv_csr<double>(u); break;
    case kOpSpmvCsrF: for (long long u = a; u < b; ++u) u_spmv_csr<float>(u); break;
    case kOpLcD: for (long long u = a; u < b; ++u) u_lincomb<double>(u); break;
    case kOpLcF: for (long long u = a; u < b; ++u) u_lincomb<float>(u); break;
    case kOpGramD: for (long long u = a; u < b; ++u) u_gram<double>(u); break;
    case kOpGramF: for (long long u = a; u < b; ++u) u_gram<float>(u); break;
    case kOpMxD2f: for (long long u = a; u < b; ++u) u_d2f(u); break;
    case kOpMxAccum: for (long long u = a; u < b; ++u) u_accum(u); break;
    default: break;
  }
}

// CTA whose share of T units (over G CTAs, CTA b taking [T b / G,
// T (b + 1) / G)) holds unit g.
__device__ __forceinline__ long long owner(long long g, long long T, long long G) {
  return ((g + 1) * G + T - 1) / T - 1;
}

// This CTA's contribution to the current system's reductions: warp sums
// into the CTA's slot, and the last contributor finishes the sums and runs
// the epilogue.  `first` is the system's first unit in the phase, `units`
// its unit count, T / G the phase's units and CTAs.
__device__ void flush(long long first, long long units, long long T,
                      long long G) {
  const Red rd = sh.op.rd;
  const int nd = op_dots(sh.op);
  if (nd == 0 && rd.epi == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();   // every warp's running sums are in
  // Contributors: the CTAs whose shares meet [first, first + units), in
  // CTA order; shares are never empty (T >= G), so each one arrives.
  const long long b_lo = owner(first, T, G);
  const int C = (int)(owner(first + units - 1, T, G) - b_lo + 1);
  if (threadIdx.x == 0) {
    double tot[kPAcc];
#pragma unroll
    for (int d = 0; d < kPAcc; ++d) {
      tot[d] = 0.0;
      if (d < nd)
        for (int w = 0; w < kPW; ++w) tot[d] += sh.acc[d][w];
    }
    if (C == 1) {
      for (int d = 0; d < nd; ++d) rd.S[rd.out + d] = tot[d];
      sh.flag = 0;
      if (rd.epi) run_epilogue(rd);
    } else {
      const long long j = (long long)blockIdx.x - b_lo;
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
  for (int d = 0; d < nd; ++d) {
    double v = 0.0;
    for (int b = threadIdx.x; b < C; b += kPT) v += __ldcg(rd.part + d * kMaxBlocks + b);
    v = warp_sum_d(v);
    if (lane == 0) sh.red[d][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < nd; ++d) {
      double s = 0.0;
      for (int w = 0; w < kPW; ++w) s += sh.red[d][w];
      rd.S[rd.out + d] = s;
    }
    *rd.ticket = 0u;
    if (rd.epi) run_epilogue(rd);
  }
  __syncthreads();
}

// One phase: operation k of every system still iterating at trip `trip`.
__device__ void phase(const PersistH& P, int k, int trip) {
  for (int s = threadIdx.x; s < P.nsys; s += kPT) {
    int u = 0;
    if (!finished(sh.ctl[s]) && trip < sh.cap[s]) {
      const OpHdrH h = P.hdr[(long long)s * P.max_ops + k];
      if (h.units > 0 && (h.guard <= 0 || __ldcg(h.S + h.guard) != 0.0)) u = h.units;
    }
    sh.u[s] = u;
  }
  __syncthreads();
  scan_units(P.nsys);
  const long long T = sh.pre[P.nsys];
  const long long G = T < (long long)gridDim.x ? T : (long long)gridDim.x;
  if ((long long)blockIdx.x >= G) return;
  // This CTA's contiguous share of the phase's units.
  const long long g0 = T * blockIdx.x / G, g1 = T * (blockIdx.x + 1) / G;
  int sys = 0;
  for (long long g = g0; g < g1;) {
    while (sh.pre[sys + 1] <= g) ++sys;
    const long long end = sh.pre[sys + 1] < g1 ? sh.pre[sys + 1] : g1;
    load_op(P, sys, k);
    run_units(g - sh.pre[sys], end - sh.pre[sys]);
    flush(sh.pre[sys], sh.u[sys], T, G);
    g = end;
  }
}

__global__ void __launch_bounds__(kPT, 1) k_persist(const PersistH P) {
  __shared__ int any;
  for (int s = threadIdx.x; s < P.nsys; s += kPT) {
    CtlH* c = P.ctl[s];
    sh.ctl[s] = c;
    sh.cap[s] = c->trip_cap;
  }
  __syncthreads();
  for (int trip = 0;; ++trip) {
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < P.nsys; s += kPT) {
      if (!finished(sh.ctl[s]) && trip < sh.cap[s]) {
        any = 1;
        if (blockIdx.x == 0) sh.ctl[s]->trips = trip + 1;
      }
    }
    __syncthreads();
    if (!any) break;
    for (int k = 0; k < P.max_ops; ++k) {
      phase(P, k, trip);
      if (!pbarrier(P, trip * P.max_ops + k)) return;
    }
  }
  // Systems that ran out of trips end as the graph loop's control node
  // ends them.
  if (blockIdx.x == 0) {
    for (int s = threadIdx.x; s < P.nsys; s += kPT) {
      CtlH* c = sh.ctl[s];
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
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist, kPT, 0) !=
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
  cfg.blockDim = dim3((unsigned)kPT);
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
