// Host drivers of the single-right-hand-side FP64 methods.  Each driver is
// the reference routine's statement sequence regrouped into fused launches;
// the comments cite the reference lines each launch covers.  All scalar
// statements run in the epilogues (epilogues.cuh) on the device.
#include "solvers.h"

#include <algorithm>
#include <cstring>

namespace bk {

namespace {

template <typename T>
T* zeros(long long n, cudaStream_t st) {
  T* p = dalloc_n<T>(n, st);
  BK_CHECK(cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, st));
  return p;
}

// Reference convention when no iteration runs (max_iter <= first index):
// error stays 0, so the routine returns its first index unless tol <= 0.
bool no_iterations(int iter0, int max_iter, double tol, SolveOut& o) {
  if (max_iter > iter0) return false;
  o.ret = tol > 0.0 ? iter0 : kNotConverged;
  o.iters = 0;
  return true;
}

SolveOut finish(const CtlH& c) {
  SolveOut o;
  o.ret = c.ret;
  o.iters = c.hist_len;
  return o;
}

template <typename T>
SpmvH<T> residual_io(const T* x, T* r, const T* b) {
  SpmvH<T> io = spmv_io<T>(x, r);
  io.b = b;
  io.mode = 1;
  return io;
}

inline void set_dot(SpmvH<double>& io, int k, int a, int b) {
  io.dot[k][0] = (unsigned char)a;
  io.dot[k][1] = (unsigned char)b;
  io.nd = std::max(io.nd, k + 1);
}

constexpr int Y = 0, B = 1, W0 = 2, W1 = 3;   // SpMV dot operand codes
constexpr int OUT = Lc<double>::OUT;

}  // namespace

// ------------------------------------------------------------------- CG
SolveOut cg(const DevCsr& A, const double* b, double* x, double tol,
            int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>(3 * np, st);
  double *r = w, *p = w + np, *t = w + 2 * np;
  ss.start(0, max_iter, tol, st);
  // src/cg.c:23-30: r = b - A x, p = r, (r, r), ||b||.
  SpmvH<double> io = residual_io<double>(x, r, b);
  io.y2 = p;
  set_dot(io, 0, B, B);
  set_dot(io, 1, Y, Y);
  spmv(A, io, ss.red(kD, E_CG_INIT), st);
  if (!no_iterations(0, max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      // :35-39  t = A p, alpha = (r,r) / (t,p)
      SpmvH<double> a = spmv_io<double>(p, t);
      a.w0 = p;
      set_dot(a, 0, Y, W0);
      spmv(A, a, ss.red(kD, E_CG_ALPHA), s);
      // :42-50, :56  x += alpha p, r -= alpha t, beta, error test
      Lc<double> u(np);
      const int ix = u.in(x), ip = u.in(p), ir = u.in(r), it = u.in(t);
      const int ox = u.out(x), orr = u.out(r);
      u.term(ox, ix, cf_const(1)).term(ox, ip, cf_slot(kAlpha));
      u.term(orr, ir, cf_const(1)).term(orr, it, cf_slot(kAlpha, -1));
      u.dot(OUT + orr, OUT + orr);
      u.launch(ss.red(kD, E_CG_CHECK), s);
      // :53-54  p = beta p + r
      Lc<double> q(np);
      const int jp = q.in(p), jr = q.in(r);
      const int op = q.out(p);
      q.term(op, jp, cf_slot(kBeta)).term(op, jr, cf_const(1));
      q.launch(ss.red(kD, E_NONE), s);
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// ------------------------------------------------------------------- CR
SolveOut cr(const DevCsr& A, const double* b, double* x, double tol,
            int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>(4 * np, st);
  double *r = w, *p = w + np, *ap = w + 2 * np, *t = w + 3 * np;
  ss.start(1, max_iter, tol, st);
  // src/cr.c:24-34: r = b - A x, p = r, t = A r, ap = t, (r, t), ||b||.
  SpmvH<double> io = residual_io<double>(x, r, b);
  io.y2 = p;
  set_dot(io, 0, B, B);
  spmv(A, io, ss.red(kD, E_CR_INIT1), st);
  SpmvH<double> i2 = spmv_io<double>(r, t);
  i2.y2 = ap;
  i2.w0 = r;
  set_dot(i2, 0, W0, Y);
  set_dot(i2, 1, Y, Y);
  spmv(A, i2, ss.red(kD, E_CR_INIT2), st);
  if (!no_iterations(1, max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      // :39-45  alpha (computed by the previous epilogue), x, r updates
      Lc<double> u(np);
      const int ix = u.in(x), ip = u.in(p), ir = u.in(r), ia = u.in(ap);
      const int ox = u.out(x), orr = u.out(r);
      u.term(ox, ix, cf_const(1)).term(ox, ip, cf_slot(kAlpha));
      u.term(orr, ir, cf_const(1)).term(orr, ia, cf_slot(kAlpha, -1));
      u.dot(OUT + orr, OUT + orr);
      u.launch(ss.red(kD, E_CR_SAVE_RR), s);
      // :48-53  t = A r, beta = (r, t) / rdot_old
      SpmvH<double> a = spmv_io<double>(r, t);
      a.w0 = r;
      set_dot(a, 0, W0, Y);
      spmv(A, a, ss.red(kD, E_CR_BETA), s);
      // :57-67  p = beta p + r, ap = beta ap + t, error test, next alpha
      Lc<double> q(np);
      const int jp = q.in(p), jr = q.in(r), ja = q.in(ap), jt = q.in(t);
      const int op = q.out(p), oa = q.out(ap);
      q.term(op, jp, cf_slot(kBeta)).term(op, jr, cf_const(1));
      q.term(oa, ja, cf_slot(kBeta)).term(oa, jt, cf_const(1));
      q.dot(OUT + oa, OUT + oa);
      q.launch(ss.red(kD, E_CR_CHECK), s);
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// ----------------------------------------------------------------- BiCG
SolveOut bicg(const DevCsr& A, const DevCsr& At, const double* b, double* x,
              double tol, int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>(6 * np, st);
  double *r = w, *sr = w + np, *p = w + 2 * np, *sp = w + 3 * np,
         *ap = w + 4 * np, *atp = w + 5 * np;
  ss.start(0, max_iter, tol, st);
  // src/bicg.c:20-29: r = sr = p = sp = b - A x, (r, sr), ||b||.
  SpmvH<double> io = residual_io<double>(x, r, b);
  io.y2 = p;
  set_dot(io, 0, B, B);
  set_dot(io, 1, Y, Y);
  spmv(A, io, ss.red(kD, E_BICG_INIT), st);
  {
    Lc<double> c(np);
    const int ir = c.in(r);
    const int o1 = c.out(sr), o2 = c.out(sp);
    c.term(o1, ir, cf_const(1)).term(o2, ir, cf_const(1));
    c.launch(ss.red(kD, E_NONE), st);
  }
  if (!no_iterations(0, max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      // :34-42  ap = A p, atp = A^T sp, alpha = rdot_old / (ap, sp)
      SpmvH<double> a = spmv_io<double>(p, ap);
      a.w0 = sp;
      set_dot(a, 0, Y, W0);
      spmv(A, a, ss.red(kD, E_BICG_ALPHA), s);
      spmv(At, spmv_io<double>(sp, atp), ss.red(kD, E_NONE), s);
      // :45-56, :66-69  x, r, sr updates, beta, error test
      Lc<double> u(np);
      const int ix = u.in(x), ip = u.in(p), ir = u.in(r), ia = u.in(ap),
                is = u.in(sr), iat = u.in(atp);
      const int ox = u.out(x), orr = u.out(r), os = u.out(sr);
      u.term(ox, ix, cf_const(1)).term(ox, ip, cf_slot(kAlpha));
      u.term(orr, ir, cf_const(1)).term(orr, ia, cf_slot(kAlpha, -1));
      u.term(os, is, cf_const(1)).term(os, iat, cf_slot(kAlpha, -1));
      u.dot(OUT + orr, OUT + os).dot(OUT + orr, OUT + orr);
      u.launch(ss.red(kD, E_BICG_CHECK), s);
      // :59-64  p = beta p + r, sp = beta sp + sr
      Lc<double> q(np);
      const int jp = q.in(p), jr = q.in(r), js = q.in(sp), jsr = q.in(sr);
      const int op = q.out(p), osp = q.out(sp);
      q.term(op, jp, cf_slot(kBeta)).term(op, jr, cf_const(1));
      q.term(osp, js, cf_slot(kBeta)).term(osp, jsr, cf_const(1));
      q.launch(ss.red(kD, E_NONE), s);
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// ------------------------------------------------------------- BiCGSTAB
SolveOut bicgstab(const DevCsr& A, const double* b, double* x, double tol,
                  int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>(6 * np, st);
  double *r = w, *rs = w + np, *s_ = w + 2 * np, *p = w + 3 * np,
         *ap = w + 4 * np, *as = w + 5 * np;
  ss.start(0, max_iter, tol, st);
  // src/bicgstab.c:22-30: r = p = rs = b - A x, ||b||, rho = (rs, r).
  SpmvH<double> io = residual_io<double>(x, r, b);
  io.y2 = p;
  set_dot(io, 0, B, B);
  set_dot(io, 1, Y, Y);
  spmv(A, io, ss.red(kD, E_BS_INIT), st);
  {
    Lc<double> c(np);
    const int ir = c.in(r);
    const int o1 = c.out(rs);
    c.term(o1, ir, cf_const(1));
    c.launch(ss.red(kD, E_NONE), st);
  }
  if (!no_iterations(0, max_iter, tol, o)) {
    auto body = [&](cudaStream_t sm) {
      // :34-36  ap = A p, alpha = rho / (rs, ap)
      SpmvH<double> a = spmv_io<double>(p, ap);
      a.w0 = rs;
      set_dot(a, 0, W0, Y);
      spmv(A, a, ss.red(kD, E_BS_ALPHA), sm);
      // :38-39  s = r - alpha ap
      Lc<double> u(np);
      const int ir = u.in(r), ia = u.in(ap);
      const int os = u.out(s_);
      u.term(os, ir, cf_const(1)).term(os, ia, cf_slot(kAlpha, -1));
      u.launch(ss.red(kD, E_NONE), sm);
      // :41-43  as = A s, omega = (as, s) / (as, as)
      SpmvH<double> c = spmv_io<double>(s_, as);
      c.w0 = s_;
      set_dot(c, 0, Y, W0);
      set_dot(c, 1, Y, Y);
      spmv(A, c, ss.red(kD, E_BS_OMEGA), sm);
      // :45-53, :59-62  x, r updates, rho, beta, error test
      Lc<double> v(np);
      const int jx = v.in(x), jp = v.in(p), js = v.in(s_), jas = v.in(as),
                jrs = v.in(rs);
      const int ox = v.out(x), orr = v.out(r);
      v.term(ox, jx, cf_const(1)).term(ox, jp, cf_slot(kAlpha))
          .term(ox, js, cf_slot(kOmega1));
      v.term(orr, js, cf_const(1)).term(orr, jas, cf_slot(kOmega1, -1));
      v.dot(jrs, OUT + orr).dot(OUT + orr, OUT + orr);
      v.launch(ss.red(kD, E_BS_CHECK), sm);
      // :55-57  p = beta (p - omega ap) + r
      Lc<double> q(np);
      const int kp = q.in(p), ka = q.in(ap), kr = q.in(r);
      const int op = q.out(p);
      q.term(op, kp, cf_slot(kBeta)).term(op, ka, cf_prod(kBeta, kOmega1, -1))
          .term(op, kr, cf_const(1));
      q.launch(ss.red(kD, E_NONE), sm);
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// ---------------------------------------------------------- BiCGSTAB(l)
SolveOut bicgstabl(const DevCsr& A, const double* b, int l, double* x,
                   double tol, int max_iter, SolveState& ss, cudaStream_t st,
                   bool fast_mr) {
  SolveOut o;
  if (l < 1 || l > kBlMaxL) throw CudaError("bicgstabl: l out of range");
  const long long np = pad64(A.n);
  double* w = zeros<double>((2 * (l + 1) + 1) * np, st);
  auto R = [&](int i) { return w + i * np; };
  auto P = [&](int i) { return w + (l + 1 + i) * np; };
  double* rs = w + 2 * (l + 1) * np;
  ss.set_scalar(kL, (double)l, st);
  ss.start(0, max_iter, tol, st);
  // src/bicgstabl.c:45-51: r0 = p0 = rs = b - A x, ||b||; then the first
  // (rs, r0) of the BiCG part (:60).
  SpmvH<double> io = residual_io<double>(x, R(0), b);
  io.y2 = P(0);
  set_dot(io, 0, B, B);
  spmv(A, io, ss.red(kD, E_BL_INIT0), st);
  {
    Lc<double> c(np);
    const int ir = c.in(R(0));
    const int o1 = c.out(rs);
    c.term(o1, ir, cf_const(1));
    c.dot(OUT + o1, ir);
    c.launch(ss.red(kD, E_BL_BETA0), st);
  }
  if (!no_iterations(0, max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      // ---- BiCG part, :59-80
      for (int j = 0; j < l; ++j) {
        {  // :64-67  p_i = beta p_i + r_i, i = 0..j
          Lc<double> u(np);
          const int ip = u.in(P(0), true), ir = u.in(R(0), true);
          const int op = u.out(P(0), true);
          u.term(op, ip, cf_slot(kBlBeta)).term(op, ir, cf_const(1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
        }
        {  // :68-71  p_{j+1} = A p_j, alpha = gamma1 / (rs, p_{j+1})
          SpmvH<double> a = spmv_io<double>(P(j), P(j + 1));
          a.w0 = rs;
          set_dot(a, 0, W0, Y);
          spmv(A, a, ss.red(kD, E_BL_ALPHA), s);
        }
        if (j + 2 <= kLcMaxOut) {
          // :73-75 and :79 in one pass: r_i -= alpha p_{i+1} (i <= j),
          // x += alpha p_0
          Lc<double> u(np);
          const int ix = u.in(x), ip0 = u.in(P(0));
          const int ox = u.out(x);
          u.term(ox, ix, cf_const(1)).term(ox, ip0, cf_slot(kBlAlpha));
          for (int i = 0; i <= j; ++i) {
            const int ir = u.in(R(i)), ip = u.in(P(i + 1));
            const int orr = u.out(R(i));
            u.term(orr, ir, cf_const(1)).term(orr, ip, cf_slot(kBlAlpha, -1));
          }
          u.launch(ss.red(kD, E_NONE), s);
        } else {
          {  // :73-75  r_i -= alpha p_{i+1}, i = 0..j
            Lc<double> u(np);
            const int ir = u.in(R(0), true), ip = u.in(P(1), true);
            const int orr = u.out(R(0), true);
            u.term(orr, ir, cf_const(1)).term(orr, ip, cf_slot(kBlAlpha, -1));
            u.batch(j + 1, np);
            u.launch(ss.red(kD, E_NONE), s);
          }
          {  // :79  x += alpha p_0
            Lc<double> u(np);
            const int ix = u.in(x), ip = u.in(P(0));
            const int ox = u.out(x);
            u.term(ox, ix, cf_const(1)).term(ox, ip, cf_slot(kBlAlpha));
            u.launch(ss.red(kD, E_NONE), s);
          }
        }
        {  // :76  r_{j+1} = A r_j (+ (rs, r_{j+1}) for the next j, :60)
          SpmvH<double> a = spmv_io<double>(R(j), R(j + 1));
          if (j + 1 < l) {
            a.w0 = rs;
            set_dot(a, 0, W0, Y);
            spmv(A, a, ss.red(kD, E_BL_BETA), s);
          } else {
            spmv(A, a, ss.red(kD, E_NONE), s);
          }
        }
      }
      // ---- MR part, :84-109
      if (fast_mr) {
        GramH<double> g;
        std::memset(&g, 0, sizeof(g));
        for (int i = 0; i <= l; ++i) g.v[i] = R(i);
        g.n = np;
        g.m = l + 1;
        launch_gram_d(g, ss.red(kGramOut, E_BLF_MR), s);
      } else {
        // modified Gram-Schmidt on r_1..r_l, as the reference
        for (int j = 1; j <= l; ++j) {
          if (j == 1) {
            Lc<double> u(np);
            const int i1 = u.in(R(1)), i0 = u.in(R(0));
            u.dot(i1, i1).dot(i0, i1);
            u.launch(ss.red(kD, E_BL_SIG, 0, 1), s);
            continue;
          }
          {
            Lc<double> u(np);
            const int ij = u.in(R(j)), i1 = u.in(R(1));
            u.dot(ij, i1);
            u.launch(ss.red(kD, E_BL_TAU, 1, (short)j), s);
          }
          for (int i = 1; i < j; ++i) {
            Lc<double> u(np);
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
      // ---- update, :113-125, plus (rs, r0) for the next iteration (:60)
      {
        Lc<double> u(np);
        const int ix = u.in(x);
        int ir[kBlMaxL + 1], ip[kBlMaxL + 1];
        for (int i = 0; i <= l; ++i) ir[i] = u.in(R(i));
        for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
        const int irs = u.in(rs);
        const int ox = u.out(x), orr = u.out(R(0)), op = u.out(P(0));
        u.term(ox, ix, cf_const(1)).term(ox, ir[0], cf_slot(kBlOmega + 1));
        u.term(orr, ir[0], cf_const(1));
        u.term(op, ip[0], cf_const(1))
            .term(op, ip[l], cf_slot((short)(kBlOmega + l), -1));
        for (int i = 1; i < l; ++i)
          u.term(op, ip[i], cf_slot((short)(kBlOmega + i), -1));
        if (fast_mr) {       // coefficients on the unorthogonalised r_i
          for (int i = 1; i <= l; ++i) {
            u.term(orr, ir[i], cf_slot((short)(kBlfCr + i), -1));
            u.term(ox, ir[i], cf_slot((short)(kBlfCx + i)));
          }
        } else {
          u.term(orr, ir[l], cf_slot((short)(kBlOmegaD + l), -1));
          for (int i = 1; i < l; ++i) {
            u.term(orr, ir[i], cf_slot((short)(kBlOmegaD + i), -1));
            u.term(ox, ir[i], cf_slot((short)(kBlOmegaDD + i)));
          }
        }
        u.dot(OUT + orr, OUT + orr).dot(irs, OUT + orr);
        u.launch(ss.red(kD, E_BL_CHECK), s);
      }
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

}  // namespace bk
