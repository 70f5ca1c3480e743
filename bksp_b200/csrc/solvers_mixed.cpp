// Mixed-precision, right-preconditioned BiCGSTAB(l) -- the fast path of the
// BiCGSTAB(l) family (no reference counterpart: the reference computes in
// FP64 only).  The recurrences are those of src/bicgstabl.c:54-126 applied
// to A M y = b (x = x0 + M y), with
//   * A and M values and all Krylov vectors in FP32 (half the bytes of the
//     FP64 path), dot products and every scalar in FP64;
//   * reliable updates: when the recursive residual has fallen by `delta`
//     since the last replacement, or `period` outer iterations have passed,
//     or it is below the target, the FP32 correction is folded into the
//     FP64 solution (x += M y, y = 0), the FP64 true residual b - A x is
//     computed with the FP64 matrix and replaces r0 -- all inside the
//     captured iteration, behind a device-side guard;
//   * convergence is decided on that FP64 true residual only.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "solvers.h"

namespace bk {

namespace {

template <typename T>
T* zeros(long long n, cudaStream_t st) {
  T* p = dalloc_n<T>(n, st);
  BK_CHECK(cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, st));
  return p;
}

constexpr int Y = 0, B = 1, W0 = 2;
constexpr int OUT = Lc<float>::OUT;

template <typename T>
void set_dot(SpmvH<T>& io, int k, int a, int b) {
  io.dot[k][0] = (unsigned char)a;
  io.dot[k][1] = (unsigned char)b;
  io.nd = std::max(io.nd, k + 1);
}

}  // namespace

MixedOut bicgstabl_mixed(const DevCsr& A, const DevCsr* M, const double* b,
                         int l, double* x, int max_iter, const MixedOpts& o,
                         SolveState& ss, cudaStream_t st) {
  if (l < 1 || l > kBlMaxL) throw CudaError("bicgstabl: l out of range");
  if (!A.v32 || (M && !M->v32)) throw CudaError("mixed solve: FP32 values missing");
  MixedOut out;
  const long long np = pad64(A.n);
  float* w = zeros<float>((2 * (l + 1) + 3) * np, st);
  auto R = [&](int i) { return w + i * np; };
  auto P = [&](int i) { return w + (l + 1 + i) * np; };
  float* rs = w + 2 * (l + 1) * np;
  float* y = rs + np;
  float* t = y + np;
  double* r64 = zeros<double>(np, st);

  ss.start(0, max_iter, 0.0, st);
  ss.set_scalar(kL, (double)l, st);
  ss.set_scalar(kMxTarget, o.target, st);
  ss.set_scalar(kMxDelta, o.delta, st);
  ss.set_scalar(kMxPeriod, (double)std::max(1, o.period), st);

  // r64 = b - A x0 (FP64), ||b||; r0 = p0 = rs = fl32(r64), (rs, r0).
  // (A + o.shift I throughout when a shift is given.)
  {
    SpmvH<double> io = spmv_io<double>(x, r64);
    io.b = b;
    io.mode = 1;
    io.shift = o.shift;
    set_dot(io, 0, Y, Y);
    set_dot(io, 1, B, B);
    spmv(A, io, ss.red(kD, E_MX_INIT), st);
    launch_mx_d2f(r64, R(0), P(0), rs, nullptr, 1, np, ss.red(kD, E_MX_INIT2), st);
  }

  // v -> A M v (FP32), optional dot (rs, A M v) into the epilogue `epi`.
  auto op = [&](const float* v, float* dst, bool dot, short epi, cudaStream_t s) {
    const float* src = v;
    if (M) {
      spmv(*M, spmv_io<float>(v, t), ss.red(kD, E_NONE), s);
      src = t;
    }
    SpmvH<float> io = spmv_io<float>(src, dst);
    io.shift = o.shift;
    if (dot) {
      io.w0 = rs;
      set_dot(io, 0, W0, Y);
    }
    spmv(A, io, ss.red(kD, epi), s);
  };

  auto body = [&](cudaStream_t s) {
    for (int j = 0; j < l; ++j) {
      {  // p_i = beta p_i + r_i
        Lc<float> u(np);
        const int ip = u.in(P(0), true), ir = u.in(R(0), true);
        const int op_ = u.out(P(0), true);
        u.term(op_, ip, cf_slot(kBlBeta)).term(op_, ir, cf_const(1));
        u.batch(j + 1, np);
        u.launch(ss.red(kD, E_NONE), s);
      }
      op(P(j), P(j + 1), true, E_BL_ALPHA, s);
      if (j + 2 <= kLcMaxOut) {   // r_i -= alpha p_{i+1}, y += alpha p_0
        Lc<float> u(np);
        const int iy = u.in(y), ip0 = u.in(P(0));
        const int oy = u.out(y);
        u.term(oy, iy, cf_const(1)).term(oy, ip0, cf_slot(kBlAlpha));
        for (int i = 0; i <= j; ++i) {
          const int ir = u.in(R(i)), ip = u.in(P(i + 1));
          const int orr = u.out(R(i));
          u.term(orr, ir, cf_const(1)).term(orr, ip, cf_slot(kBlAlpha, -1));
        }
        u.launch(ss.red(kD, E_NONE), s);
      } else {
        Lc<float> u(np);
        const int ir = u.in(R(0), true), ip = u.in(P(1), true);
        const int orr = u.out(R(0), true);
        u.term(orr, ir, cf_const(1)).term(orr, ip, cf_slot(kBlAlpha, -1));
        u.batch(j + 1, np);
        u.launch(ss.red(kD, E_NONE), s);
        Lc<float> v(np);
        const int iy = v.in(y), i0 = v.in(P(0));
        const int oy = v.out(y);
        v.term(oy, iy, cf_const(1)).term(oy, i0, cf_slot(kBlAlpha));
        v.launch(ss.red(kD, E_NONE), s);
      }
      op(R(j), R(j + 1), j + 1 < l, j + 1 < l ? E_BL_BETA : E_NONE, s);
    }
    // MR part, FP64 dots of FP32 vectors.
    if (o.fast_mr) {
      GramH<float> g;
      std::memset(&g, 0, sizeof(g));
      for (int i = 0; i <= l; ++i) g.v[i] = R(i);
      g.n = np;
      g.m = l + 1;
      launch_gram_f(g, ss.red(kGramOut, E_BLF_MR), s);
    } else {
      // modified Gram-Schmidt, as the reference
      for (int j = 1; j <= l; ++j) {
        if (j == 1) {
          Lc<float> u(np);
          const int i1 = u.in(R(1)), i0 = u.in(R(0));
          u.dot(i1, i1).dot(i0, i1);
          u.launch(ss.red(kD, E_BL_SIG, 0, 1), s);
          continue;
        }
        {
          Lc<float> u(np);
          const int ij = u.in(R(j)), i1 = u.in(R(1));
          u.dot(ij, i1);
          u.launch(ss.red(kD, E_BL_TAU, 1, (short)j), s);
        }
        for (int i = 1; i < j; ++i) {
          Lc<float> u(np);
          const int ij = u.in(R(j)), ii = u.in(R(i));
          const int oj = u.out(R(j));
          u.term(oj, ij, cf_const(1))
              .term(oj, ii, cf_slot((short)(kBlTau + i * l + j), -1));
          if (i + 1 < j) {
            const int in = u.in(R(i + 1));
            u.dot(OUT + oj, in);
            u.launch(ss.red(kD, E_BL_TAU, (short)(i + 1), (short)j), s);
          } else {
            const int i0 = u.in(R(0));
            u.dot(OUT + oj, OUT + oj).dot(i0, OUT + oj);
            u.launch(ss.red(kD, E_BL_SIG, 0, (short)j), s);
          }
        }
      }
    }
    {  // update y, r0, p0; recursive residual test / replacement trigger
      Lc<float> u(np);
      const int iy = u.in(y);
      int ir[kBlMaxL + 1], ip[kBlMaxL + 1];
      for (int i = 0; i <= l; ++i) ir[i] = u.in(R(i));
      for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
      const int irs = u.in(rs);
      const int oy = u.out(y), orr = u.out(R(0)), op_ = u.out(P(0));
      u.term(oy, iy, cf_const(1)).term(oy, ir[0], cf_slot(kBlOmega + 1));
      u.term(orr, ir[0], cf_const(1));
      u.term(op_, ip[0], cf_const(1))
          .term(op_, ip[l], cf_slot((short)(kBlOmega + l), -1));
      for (int i = 1; i < l; ++i)
        u.term(op_, ip[i], cf_slot((short)(kBlOmega + i), -1));
      if (o.fast_mr) {     // coefficients on the unorthogonalised r_i
        for (int i = 1; i <= l; ++i) {
          u.term(orr, ir[i], cf_slot((short)(kBlfCr + i), -1));
          u.term(oy, ir[i], cf_slot((short)(kBlfCx + i)));
        }
      } else {
        u.term(orr, ir[l], cf_slot((short)(kBlOmegaD + l), -1));
        for (int i = 1; i < l; ++i) {
          u.term(orr, ir[i], cf_slot((short)(kBlOmegaD + i), -1));
          u.term(oy, ir[i], cf_slot((short)(kBlOmegaDD + i)));
        }
      }
      u.dot(OUT + orr, OUT + orr).dot(irs, OUT + orr);
      u.launch(ss.red(kD, E_MX_CHECK), s);
    }
    // Reliable update, guarded by S[kMxDoRep]; in the captured iteration
    // these kernels sit in a conditional node that E_MX_CHECK opens only
    // when a replacement is due.
    cond_block(ss, s, [&](cudaStream_t s2) {
      const float* corr = y;
      if (M) {
        spmv(*M, spmv_io<float>(y, t), ss.red_if(kMxDoRep, kD, E_NONE), s2);
        corr = t;
      }
      launch_mx_accum(x, corr, y, np, ss.red_if(kMxDoRep, kD, E_NONE), s2);
      {
        SpmvH<double> io = spmv_io<double>(x, r64);
        io.b = b;
        io.mode = 1;
        io.shift = o.shift;
        set_dot(io, 0, Y, Y);
        spmv(A, io, ss.red_if(kMxDoRep, kD, E_MX_TRUE), s2);
      }
      launch_mx_d2f(r64, R(0), nullptr, nullptr, rs, 1, np,
                    ss.red_if(kMxDoRep, kD, E_MX_REBETA), s2);
    });
  };
  const CtlH c = run_loop(ss, body, st);
  // Fold any correction not yet accumulated (budget exhausted / breakdown).
  const float* corr = y;
  if (M) {
    spmv(*M, spmv_io<float>(y, t), ss.red_after(kD, E_NONE), st);
    corr = t;
  }
  launch_mx_accum(x, corr, y, np, ss.red_after(kD, E_NONE), st);
  BK_CHECK(cudaGetLastError());
  out.ret = c.ret;
  out.iters = c.hist_len;
  out.replacements = (int)ss.get_scalar(kMxReps, st);
  // The conditional node's kernels ran only in the iterations with a
  // replacement (run_loop counted them in every trip).
  if (ss.has_cond) {
    const long long idle = std::max(0, c.trips - out.replacements);
    launch_count() -= ss.cond_kernels * idle;
    byte_count() -= ss.cond_bytes * idle;
  }
  ss.has_cond = false;
  out.true_res = ss.get_scalar(kMxTrue, st);
  dfree(w, st);
  dfree(r64, st);
  return out;
}

MixedOut cg_mixed_fused(const DevCsr& A, const DevCsr* M, const double* b,
                        double* x, int max_iter, const MixedOpts& o,
                        SolveState& ss, cudaStream_t st) {
  MixedOut out;
  const long long np = pad64(A.n);
  float* w = zeros<float>(7 * np, st);
  float* R[2] = {w, w + np};
  float* P[2] = {w + 2 * np, w + 3 * np};
  float *z = w + 4 * np, *q = w + 5 * np, *y = w + 6 * np;
  double* r64 = zeros<double>(np, st);

  ss.start(0, max_iter, 0.0, st);
  ss.set_scalar(kMxTarget, o.target, st);
  ss.set_scalar(kMxDelta, o.delta, st);
  ss.set_scalar(kMxPeriod, (double)std::max(1, o.period), st);
  ss.set_scalar(kBeta, 0.0, st);   // first p = z + 0 * 0
  {
    SpmvH<double> io = spmv_io<double>(x, r64);
    io.b = b;
    io.mode = 1;
    set_dot(io, 0, Y, Y);
    set_dot(io, 1, B, B);
    spmv(A, io, ss.red(kD, E_MX_INIT), st);
  }
  // r = fl32(r64); z = M r and rho = (r, z) (z = r without M).
  auto restart = [&](float* r, const RedH& conv, const RedH& beta, cudaStream_t s) {
    if (M) {
      launch_mx_d2f(r64, r, nullptr, nullptr, nullptr, 0, np, conv, s);
      SpmvH<float> io = spmv_io<float>(r, z);
      io.w0 = r;
      set_dot(io, 0, W0, Y);
      spmv(*M, io, beta, s);
    } else {
      launch_mx_d2f(r64, r, nullptr, nullptr, nullptr, 1, np, beta, s);
    }
  };
  restart(R[0], ss.red(kD, E_NONE), ss.red(kD, E_MCG_RHO0), st);

  auto half = [&](int h, cudaStream_t s) {
    float *pa = P[h], *pb = P[1 - h], *ra = R[h], *rb = R[1 - h];
    {  // p = z + beta p_old (stored to pb), q = A p, alpha = rho / (p, q)
      SpmvFuseH<float> f;
      std::memset(&f, 0, sizeof(f));
      f.xa = M ? z : ra;
      f.ca = cf_const(1);
      f.xb = pa;
      f.cb = cf_slot(kBeta);
      f.xe = pb;
      f.y = q;
      f.nd = 1;
      f.dot[0][0] = 1;
      f.dot[0][1] = 0;
      launch_spmv_fused_f(A.h32(), f, ss.red(kD, E_MCG_ALPHA), s);
    }
    if (M) {  // r = r_old - alpha q (stored to rb), z = M r, y += alpha p
      SpmvFuseH<float> f;
      std::memset(&f, 0, sizeof(f));
      f.xa = ra;
      f.ca = cf_const(1);
      f.xb = q;
      f.cb = cf_slot(kAlpha, -1);
      f.xe = rb;
      f.y = z;
      f.f0 = y;
      f.c0 = cf_const(1);
      f.f1 = pb;
      f.c1 = cf_slot(kAlpha);
      f.fo = y;
      f.nd = 2;
      f.dot[0][0] = 1; f.dot[0][1] = 1;   // (r, r)
      f.dot[1][0] = 1; f.dot[1][1] = 0;   // (r, z)
      launch_spmv_fused_f(M->h32(), f, ss.red(kD, E_MCG_RES, 2, (short)h), s);
    } else {
      Lc<float> u(np);
      const int iy = u.in(y), ip = u.in(pb), ir = u.in(ra), iq = u.in(q);
      const int oy = u.out(y), orr = u.out(rb);
      u.term(oy, iy, cf_const(1)).term(oy, ip, cf_slot(kAlpha));
      u.term(orr, ir, cf_const(1)).term(orr, iq, cf_slot(kAlpha, -1));
      u.dot(OUT + orr, OUT + orr);
      u.launch(ss.red(kD, E_MCG_RES, 1, (short)h), s);
    }
    cond_block(ss, s, [&](cudaStream_t s2) {   // the h-th node of the body
      launch_mx_accum(x, y, y, np, ss.red_if(kMxDoRep, kD, E_NONE), s2);
      SpmvH<double> io = spmv_io<double>(x, r64);
      io.b = b;
      io.mode = 1;
      set_dot(io, 0, Y, Y);
      spmv(A, io, ss.red_if(kMxDoRep, kD, E_MX_TRUE), s2);
      restart(rb, ss.red_if(kMxDoRep, kD, E_NONE),
              ss.red_if(kMxDoRep, kD, E_MCG_BETA), s2);
    });
  };
  auto body = [&](cudaStream_t s) {
    half(0, s);
    half(1, s);
  };
  const CtlH c = run_loop(ss, body, st);
  launch_mx_accum(x, y, y, np, ss.red_after(kD, E_NONE), st);
  BK_CHECK(cudaGetLastError());
  out.ret = c.ret;
  out.iters = c.hist_len;
  out.replacements = (int)ss.get_scalar(kMxReps, st);
  if (ss.has_cond) {
    // two conditional nodes per body: the idle ones launched nothing
    const long long idle = std::max(0, 2 * c.trips - out.replacements);
    launch_count() -= ss.cond_kernels / 2 * idle;
    byte_count() -= ss.cond_bytes / 2 * idle;
  }
  ss.has_cond = false;
  out.true_res = ss.get_scalar(kMxTrue, st);
  dfree(w, st);
  dfree(r64, st);
  return out;
}

// Mixed-precision preconditioned CG with reliable updates (no reference
// counterpart; the recurrence is src/cg.c:35-54 with a symmetric
// preconditioner z = M r): FP32 values of A and M and FP32 vectors r, z, p,
// q = A p and the correction y (solution space), FP64 dots, scalars and
// solution.  Every replacement folds y into the FP64 x, recomputes the
// FP64 true residual b - A x with the FP64 operator and restarts r from it
// (p kept); convergence is decided on that true residual.
namespace {

// The same method with each iteration in two launches, for operators (and
// preconditioners) in diagonal form: the product q = A p forms p = z + beta
// p_old on the fly (and stores it), the preconditioner product z = M r
// forms r = r_old - alpha q on the fly (storing it) and carries y += alpha
// p along; p and r alternate between two buffers, two iterations per loop
// body.
bool cg_fusable(const DevCsr& A, const DevCsr* M) {
  static const bool off = [] {
    const char* e = std::getenv("BKSP_GPU_FUSE");
    return e && std::strcmp(e, "0") == 0;
  }();
  return !off && A.ndia > 0 && A.d32 &&
         (!M || (M->ndia > 0 && M->d32));
}

}  // namespace

MixedOut cg_mixed(const DevCsr& A, const DevCsr* M, const double* b, double* x,
                  int max_iter, const MixedOpts& o, SolveState& ss,
                  cudaStream_t st) {
  if (!A.v32 || (M && !M->v32)) throw CudaError("mixed solve: FP32 values missing");
  if (cg_fusable(A, M)) return cg_mixed_fused(A, M, b, x, max_iter, o, ss, st);
  MixedOut out;
  const long long np = pad64(A.n);
  float* w = zeros<float>(5 * np, st);
  float *r = w, *z = w + np, *p = w + 2 * np, *q = w + 3 * np, *y = w + 4 * np;
  double* r64 = zeros<double>(np, st);
  const short unprec = M ? 0 : 1;

  ss.start(0, max_iter, 0.0, st);
  ss.set_scalar(kMxTarget, o.target, st);
  ss.set_scalar(kMxDelta, o.delta, st);
  ss.set_scalar(kMxPeriod, (double)std::max(1, o.period), st);

  // r64 = b - A x0 (FP64), ||b||, true residual; r = fl32(r64); z = M r,
  // p = z, rho = (r, z).
  {
    SpmvH<double> io = spmv_io<double>(x, r64);
    io.b = b;
    io.mode = 1;
    set_dot(io, 0, Y, Y);
    set_dot(io, 1, B, B);
    spmv(A, io, ss.red(kD, E_MX_INIT), st);
  }
  auto precondition = [&](const RedH& rd, cudaStream_t s) {
    // z = M r, p-independent; (r, z) into the epilogue of rd
    SpmvH<float> io = spmv_io<float>(r, z);
    io.w0 = r;
    set_dot(io, 0, W0, Y);
    spmv(*M, io, rd, s);
  };
  if (M) {
    launch_mx_d2f(r64, r, nullptr, nullptr, nullptr, 0, np, ss.red(kD, E_NONE), st);
    SpmvH<float> io = spmv_io<float>(r, z);
    io.y2 = p;
    io.w0 = r;
    set_dot(io, 0, W0, Y);
    spmv(*M, io, ss.red(kD, E_MCG_RHO0), st);
  } else {
    launch_mx_d2f(r64, r, p, nullptr, nullptr, 1, np, ss.red(kD, E_MCG_RHO0), st);
  }

  auto body = [&](cudaStream_t s) {
    {  // q = A p, alpha = rho / (p, q)
      SpmvH<float> io = spmv_io<float>(p, q);
      io.w0 = p;
      set_dot(io, 0, W0, Y);
      spmv(A, io, ss.red(kD, E_MCG_ALPHA), s);
    }
    {  // y += alpha p, r -= alpha q, (r, r): replacement decision
      Lc<float> u(np);
      const int iy = u.in(y), ip = u.in(p), ir = u.in(r), iq = u.in(q);
      const int oy = u.out(y), orr = u.out(r);
      u.term(oy, iy, cf_const(1)).term(oy, ip, cf_slot(kAlpha));
      u.term(orr, ir, cf_const(1)).term(orr, iq, cf_slot(kAlpha, -1));
      u.dot(OUT + orr, OUT + orr);
      u.launch(ss.red(kD, E_MCG_RES, unprec), s);
    }
    cond_block(ss, s, [&](cudaStream_t s2) {
      // x += y (FP64), y = 0; r64 = b - A x; r = fl32(r64)
      launch_mx_accum(x, y, y, np, ss.red_if(kMxDoRep, kD, E_NONE), s2);
      SpmvH<double> io = spmv_io<double>(x, r64);
      io.b = b;
      io.mode = 1;
      set_dot(io, 0, Y, Y);
      spmv(A, io, ss.red_if(kMxDoRep, kD, E_MX_TRUE), s2);
      if (M)
        launch_mx_d2f(r64, r, nullptr, nullptr, nullptr, 0, np,
                      ss.red_if(kMxDoRep, kD, E_NONE), s2);
      else
        launch_mx_d2f(r64, r, nullptr, nullptr, nullptr, 1, np,
                      ss.red_if(kMxDoRep, kD, E_MCG_BETA), s2);
    });
    if (M) precondition(ss.red(kD, E_MCG_BETA), s);
    {  // p = z + beta p
      Lc<float> u(np);
      const int iz = u.in(M ? z : r), ip = u.in(p);
      const int op_ = u.out(p);
      u.term(op_, iz, cf_const(1)).term(op_, ip, cf_slot(kBeta));
      u.launch(ss.red(kD, E_NONE), s);
    }
  };
  const CtlH c = run_loop(ss, body, st);
  // Fold the correction not yet accumulated.
  launch_mx_accum(x, y, y, np, ss.red_after(kD, E_NONE), st);
  BK_CHECK(cudaGetLastError());
  out.ret = c.ret;
  out.iters = c.hist_len;
  out.replacements = (int)ss.get_scalar(kMxReps, st);
  if (ss.has_cond) {
    const long long idle = std::max(0, c.trips - out.replacements);
    launch_count() -= ss.cond_kernels * idle;
    byte_count() -= ss.cond_bytes * idle;
  }
  ss.has_cond = false;
  out.true_res = ss.get_scalar(kMxTrue, st);
  dfree(w, st);
  dfree(r64, st);
  return out;
}

// FP64 ||b - (A + shift I) x|| / ||b|| of padded device vectors.
static double shifted_residual(const DevCsr& A, const double* b, const double* x,
                               double shift, cudaStream_t st) {
  const long long np = pad64(A.n);
  double* r = dalloc_n<double>(np, st);
  SolveState t;
  t.create(0, st);
  t.start(0, 1, 0.0, st);
  SpmvH<double> io = spmv_io<double>(x, r);
  io.b = b;
  io.mode = 1;
  io.shift = shift;
  set_dot(io, 0, Y, Y);
  set_dot(io, 1, B, B);
  spmv(A, io, t.red(kD, E_NONE), st);
  const double rr = t.get_scalar(kD, st), bb = t.get_scalar(kD + 1, st);
  t.release(st);
  dfree(r, st);
  return std::sqrt(rr) / std::sqrt(bb);
}

MixedOut shbicgstabl_mixed(const DevCsr& A, const double* b, int l,
                           const double* sigma_host, int ns, double* x,
                           double target, int max_iter, SolveState& ss,
                           cudaStream_t st) {
  if (!A.v32) throw CudaError("mixed solve: FP32 values missing");
  MixedOut out;
  const SolveOut o = shbicgstabl(A, b, l, sigma_host, ns, x, target, max_iter, ss,
                                 st, /*fp32_ps=*/true);
  out.ret = o.ret;
  out.iters = 0;
  const long long np = pad64(A.n);
  double worst = 0.0;
  for (int k = -1; k < ns; ++k) {
    const double sg = k < 0 ? 0.0 : sigma_host[k];
    double* xk = x + (long long)(k + 1) * np;
    double res = shifted_residual(A, b, xk, sg, st);
    if (!(res <= target)) {
      MixedOpts mo;
      mo.target = target;
      mo.shift = sg;
      SolveState ps;
      ps.create(0, st);
      const MixedOut p = bicgstabl_mixed(A, nullptr, b, l, xk, max_iter, mo, ps, st);
      ps.release(st);
      out.iters += p.iters;
      out.replacements += p.replacements;
      res = p.true_res;
      if (p.ret < 0 && out.ret >= 0) out.ret = kNotConverged;
    }
    worst = std::isfinite(res) ? std::max(worst, res) : res;
  }
  out.true_res = worst;
  return out;
}

}  // namespace bk
