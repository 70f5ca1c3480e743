// Fused level-1 kernels (linear combinations with dots, pairwise Gram
// products) and their launch wrappers (kernel_api.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "dev_common.cuh"
#include "epilogues.cuh"
#include "k_vec.cuh"
#include "kernel_api.h"
#include "launch_util.h"

namespace bk {

// ------------------------------------------------------ linear combination

template <typename T, int MI, int MO>
static void lc_nd(const LcH<T>& d, const RedH& rd, cudaStream_t st) {
  const long long q = d.n / Pack<T>::N;
  switch (d.nd) {
    case 0: launch_k(k_lincomb<T, MI, MO, 0>, grid_wave(k_lincomb<T, MI, MO, 0>, q), kThreads, 0, st, d, rd); break;
    case 1: launch_k(k_lincomb<T, MI, MO, 1>, grid_wave(k_lincomb<T, MI, MO, 1>, q), kThreads, 0, st, d, rd); break;
    case 2: launch_k(k_lincomb<T, MI, MO, 2>, grid_wave(k_lincomb<T, MI, MO, 2>, q), kThreads, 0, st, d, rd); break;
    default: launch_k(k_lincomb<T, MI, MO, 3>, grid_wave(k_lincomb<T, MI, MO, 3>, q), kThreads, 0, st, d, rd); break;
  }
}

template <typename T>
static void lc_dispatch(const LcH<T>& d, const RedH& rd, cudaStream_t st) {
  if (d.nin <= 4 && d.nout <= 2) lc_nd<T, 4, 2>(d, rd, st);
  else if (d.nin <= 8 && d.nout <= 4) lc_nd<T, 8, 4>(d, rd, st);
  else if (d.nout <= 4) lc_nd<T, 24, 4>(d, rd, st);
  else if (d.nin <= 16) lc_nd<T, 16, 6>(d, rd, st);
  else lc_nd<T, 24, 6>(d, rd, st);
}

// Every input and output once per repetition it is advanced in, else once.
template <typename T>
static long long lc_bytes(const LcH<T>& d) {
  long long vecs = 0;
  for (int i = 0; i < d.nin; ++i) vecs += (d.in_rep_mask >> i) & 1u ? d.reps : 1;
  for (int o = 0; o < d.nout; ++o) vecs += (d.out_rep_mask >> o) & 1u ? d.reps : 1;
  return vecs * d.n * (long long)sizeof(T);
}

// Persistent-loop form: units run over (repetition, chunk).
template <typename T>
static void lc_record(const LcH<T>& d, const RedH& rd) {
  if (d.nd > 3) prog_unsupported("linear combination with more than three dots");
  if (d.n % 4 || (d.reps > 1 && d.stride % 4)) prog_unsupported("unpadded vector");
  for (int i = 0; i < d.nin; ++i) prog_require_aligned(d.in[i]);
  for (int o = 0; o < d.nout; ++o) prog_require_aligned(d.out[o]);
  ProgOpH op;
  std::memset(&op, 0, sizeof(op));
  if constexpr (sizeof(T) == 8) {
    op.kind = kOpLcD;
    op.u.ld = d;
  } else {
    op.kind = kOpLcF;
    op.u.lf = d;
  }
  op.units = prog_units(d.n) * (d.reps > 0 ? d.reps : 1);
  op.rd = rd;
  prog_push(op);
}

void launch_lincomb_d(const LcH<double>& d, const RedH& rd, cudaStream_t st) {
  byte_count() += lc_bytes(d);
  if (g_prog_rec) return lc_record<double>(d, rd);
  ++launch_count();
  lc_dispatch<double>(d, rd, st);
}
void launch_lincomb_f(const LcH<float>& d, const RedH& rd, cudaStream_t st) {
  byte_count() += lc_bytes(d);
  if (g_prog_rec) return lc_record<float>(d, rd);
  ++launch_count();
  lc_dispatch<float>(d, rd, st);
}

// ------------------------------------------------------ pairwise Gram

template <typename T>
static void gram_dispatch(const GramH<T>& g, const RedH& rd, cudaStream_t st) {
  byte_count() += (long long)g.m * g.n * (long long)sizeof(T);
  if (g_prog_rec) {
    if (g.m > kPersistGramMax) prog_unsupported("Gram of more than five vectors");
    if (g.n % 4) prog_unsupported("unpadded vector");
    for (int i = 0; i < g.m; ++i) prog_require_aligned(g.v[i]);
    ProgOpH op;
    std::memset(&op, 0, sizeof(op));
    if constexpr (sizeof(T) == 8) {
      op.kind = kOpGramD;
      op.u.gd = g;
    } else {
      op.kind = kOpGramF;
      op.u.gf = g;
    }
    op.units = prog_units(g.n);
    op.rd = rd;
    prog_push(op);
    return;
  }
  ++launch_count();
  const long long q = (g.n / Pack<T>::N + 1) / 2;   // two packets per thread
  switch (g.m) {
#define BK_GRAM(M)                                                        \
  case M:                                                                 \
    launch_k(k_gram_vec<T, M>, grid_wave(k_gram_vec<T, M>, q), kThreads, 0, st, g, rd); \
    break;
    BK_GRAM(2) BK_GRAM(3) BK_GRAM(4) BK_GRAM(5) BK_GRAM(6) BK_GRAM(7) BK_GRAM(8)
    default:
      launch_k(k_gram_vec<T, 9>, grid_wave(k_gram_vec<T, 9>, q), kThreads, 0, st, g, rd);
      break;
#undef BK_GRAM
  }
}
void launch_gram_d(const GramH<double>& g, const RedH& rd, cudaStream_t st) {
  gram_dispatch<double>(g, rd, st);
}
void launch_gram_f(const GramH<float>& g, const RedH& rd, cudaStream_t st) {
  gram_dispatch<float>(g, rd, st);
}

}  // namespace bk
