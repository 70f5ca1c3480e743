// Host drivers of the shifted methods: the seed recurrence as fused
// launches (as in solvers.cpp) plus the fused all-shift kernel (k_shift.cuh)
// for every per-shift vector update.  Scalars, including all per-shift
// recurrences, run in the epilogues.
#include <algorithm>

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
constexpr int OUT = Lc<double>::OUT;

void set_dot(SpmvH<double>& io, int k, int a, int b) {
  io.dot[k][0] = (unsigned char)a;
  io.dot[k][1] = (unsigned char)b;
  io.nd = std::max(io.nd, k + 1);
}

bool no_iterations(int max_iter, double tol, SolveOut& o) {
  if (max_iter > 0) return false;
  o.ret = tol > 0.0 ? 0 : kNotConverged;
  return true;
}

}  // namespace

// ---------------------------------------------------------- shifted BiCG
SolveOut shbicg(const DevCsr& A, const DevCsr& At, const double* b,
                const double* sigma_host, int ns, double* x, double tol,
                int max_iter, SolveState& ss, cudaStream_t st) {
  if (ns < 0 || ns > kMaxShifts) throw CudaError("shbicg: too many shifts");
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>(6 * np, st);
  double *r = w, *sr = w + np, *p = w + 2 * np, *sp = w + 3 * np,
         *ap = w + 4 * np, *atp = w + 5 * np;
  double* ps = zeros<double>((long long)std::max(ns, 1) * np, st);
  ss.start(0, max_iter, tol, st);
  ss.set_scalar(kNs, (double)ns, st);
  ss.set_scalars(kShSigma, sigma_host, ns, st);
  // src/shbicg.c:21-46: r = sr = b - A x, ||b||; (r, sr) for iteration 0.
  SpmvH<double> io = spmv_io<double>(x, r);
  io.b = b;
  io.mode = 1;
  io.y2 = sr;
  set_dot(io, 0, B, B);
  set_dot(io, 1, Y, Y);
  spmv(A, io, ss.red(kD, E_SHB_INIT), st);
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      {  // :56-61  p = -beta p + r, sp = -beta sp + sr
        Lc<double> u(np);
        const int ip = u.in(p), ir = u.in(r), is = u.in(sp), isr = u.in(sr);
        const int op = u.out(p), osp = u.out(sp);
        u.term(op, ip, cf_slot(kShBetaS, -1)).term(op, ir, cf_const(1));
        u.term(osp, is, cf_slot(kShBetaS, -1)).term(osp, isr, cf_const(1));
        u.launch(ss.red(kD, E_NONE), s);
      }
      {  // :64-72  ap = A p, atp = A^T sp, alpha; shift scalars (:78-88)
        SpmvH<double> a = spmv_io<double>(p, ap);
        a.w0 = sr;
        set_dot(a, 0, Y, W0);
        spmv(A, a, ss.red(kD, E_SHB_ALPHA), s);
        spmv(At, spmv_io<double>(sp, atp), ss.red(kD, E_NONE), s);
      }
      {  // :75, :90-95  x, p_k, x_k
        ShiftArgsH sa{r, p, x, x + np, ps, np, ns, 0, 0, 0};
        launch_shift(sa, ss.red(kD, E_NONE), s);
      }
      {  // :99-115  r, sr updates, rotation, error test; next rho / beta
        Lc<double> u(np);
        const int ir = u.in(r), ia = u.in(ap), isr = u.in(sr), iat = u.in(atp);
        const int orr = u.out(r), osr = u.out(sr);
        u.term(orr, ir, cf_const(1)).term(orr, ia, cf_slot(kShAlphaS, -1));
        u.term(osr, isr, cf_const(1)).term(osr, iat, cf_slot(kShAlphaS, -1));
        u.dot(OUT + orr, OUT + osr).dot(OUT + orr, OUT + orr);
        u.launch(ss.red(kD, E_SHB_CHECK), s);
      }
    };
    const CtlH c = run_loop(ss, body, st);
    o.ret = c.ret;
    o.iters = c.hist_len;
  }
  dfree(w, st);
  dfree(ps, st);
  return o;
}

// --------------------------------------------------- shifted BiCGSTAB(l)
SolveOut shbicgstabl(const DevCsr& A, const double* b, int l,
                     const double* sigma_host, int ns, double* x, double tol,
                     int max_iter, SolveState& ss, cudaStream_t st,
                     bool fp32_ps) {
  if (l < 1 || l > kBlMaxL) throw CudaError("shbicgstabl: l out of range");
  if (ns < 0 || ns > kMaxShifts) throw CudaError("shbicgstabl: too many shifts");
  SolveOut o;
  const long long np = pad64(A.n);
  double* w = zeros<double>((2 * (l + 1) + 1) * np, st);
  auto R = [&](int i) { return w + i * np; };
  auto P = [&](int i) { return w + (l + 1 + i) * np; };
  double* rs = w + 2 * (l + 1) * np;
  const long long nps = (long long)std::max(ns, 1) * (l + 1) * np;
  double* ps = fp32_ps ? nullptr : zeros<double>(nps, st);
  float* ps32 = fp32_ps ? zeros<float>(nps, st) : nullptr;
  ss.start(0, max_iter, tol, st);
  ss.set_scalar(kL, (double)l, st);
  ss.set_scalar(kNs, (double)ns, st);
  ss.set_scalars(kShSigma, sigma_host, ns, st);
  // src/shbicgstabl.c:32-43: r0 = p0 = rs = b - A x, ||b||; (r0, rs).
  SpmvH<double> io = spmv_io<double>(x, R(0));
  io.b = b;
  io.mode = 1;
  io.y2 = P(0);
  set_dot(io, 0, B, B);
  set_dot(io, 1, Y, Y);
  spmv(A, io, ss.red(kD, E_SHL_INIT), st);
  {
    Lc<double> c(np);
    const int ir = c.in(R(0));
    const int o1 = c.out(rs);
    c.term(o1, ir, cf_const(1));
    c.launch(ss.red(kD, E_NONE), st);
  }
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      for (int j = 0; j < l; ++j) {
        {  // :95-98  p_i = -beta p_i + r_i
          Lc<double> u(np);
          const int ip = u.in(P(0), true), ir = u.in(R(0), true);
          const int op = u.out(P(0), true);
          u.term(op, ip, cf_slot(kBlBeta, -1)).term(op, ir, cf_const(1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
        }
        {  // :101-105  p_{j+1} = A p_j, alpha; shift scalars :111-121
          SpmvH<double> a = spmv_io<double>(P(j), P(j + 1));
          a.w0 = rs;
          set_dot(a, 0, W0, Y);
          spmv(A, a, ss.red(kD, E_SHL_ALPHA), s);
        }
        {  // :108, :123-133  x, p_k[0..j+1], x_k
          ShiftArgsH sa{R(0), P(0), x, x + np, ps, np, ns, l, j, 1, ps32};
          launch_shift(sa, ss.red(kD, E_NONE), s);
        }
        {  // :137-139  r_i -= alpha p_{i+1}
          Lc<double> u(np);
          const int ir = u.in(R(0), true), ip = u.in(P(1), true);
          const int orr = u.out(R(0), true);
          u.term(orr, ir, cf_const(1)).term(orr, ip, cf_slot(kBlAlpha, -1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
        }
        {  // :142  r_{j+1} = A r_j (+ (r_{j+1}, rs) for the next j, :91)
          SpmvH<double> a = spmv_io<double>(R(j), R(j + 1));
          if (j + 1 < l) {
            a.w0 = rs;
            set_dot(a, 0, Y, W0);
            spmv(A, a, ss.red(kD, E_SHL_BETA), s);
          } else {
            spmv(A, a, ss.red(kD, E_NONE), s);
          }
        }
        {  // :146-161  p_k[j+1] completion, then scalar rotation
          ShiftArgsH sa{R(0), P(0), x, x + np, ps, np, ns, l, j, 2, ps32};
          launch_shift(sa, ss.red(kD, E_SHL_ROTATE, j + 1 < l ? 1 : 0), s);
        }
      }
      // MR part, :166-173 (modified Gram-Schmidt on r_1..r_l)
      for (int j = 0; j < l; ++j) {
        if (j == 0) {
          Lc<double> u(np);
          const int i1 = u.in(R(1)), i0 = u.in(R(0));
          u.dot(i1, i1).dot(i0, i1);
          u.launch(ss.red(kD, E_SHL_SIG, 0, 0), s);
          continue;
        }
        {
          Lc<double> u(np);
          const int ij = u.in(R(j + 1)), i1 = u.in(R(1));
          u.dot(ij, i1);
          u.launch(ss.red(kD, E_SHL_TAU, 0, (short)j), s);
        }
        for (int i = 0; i < j; ++i) {
          Lc<double> u(np);
          const int ij = u.in(R(j + 1)), ii = u.in(R(i + 1));
          const int oj = u.out(R(j + 1));
          u.term(oj, ij, cf_const(1))
              .term(oj, ii, cf_slot((short)(kBlTau + i * l + j), -1));
          if (i + 1 < j) {
            const int in = u.in(R(i + 2));
            u.dot(OUT + oj, in);
            u.launch(ss.red(kD, E_SHL_TAU, (short)(i + 1), (short)j), s);
          } else {
            const int i0 = u.in(R(0));
            u.dot(OUT + oj, OUT + oj).dot(i0, OUT + oj);
            u.launch(ss.red(kD, E_SHL_SIG, 0, (short)j), s);
          }
        }
      }
      {  // :194-199  seed x and p0
        Lc<double> u(np);
        const int ix = u.in(x);
        int ir[kBlMaxL + 1], ip[kBlMaxL + 1];
        for (int i = 0; i < l; ++i) ir[i] = u.in(R(i));
        for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
        const int ox = u.out(x), op = u.out(P(0));
        u.term(ox, ix, cf_const(1)).term(ox, ir[0], cf_slot(kBlOmega + 0));
        u.term(op, ip[0], cf_const(1))
            .term(op, ip[l], cf_slot((short)(kBlOmega + l - 1), -1));
        for (int i = 1; i < l; ++i) {
          u.term(op, ip[i], cf_slot((short)(kBlOmega + i - 1), -1));
          u.term(ox, ir[i], cf_slot((short)(kBlOmegaDD + i - 1)));
        }
        u.launch(ss.red(kD, E_NONE), s);
      }
      {  // :202-237  every shift's x_k and p_k[0]
        ShiftArgsH sa{R(0), P(0), x, x + np, ps, np, ns, l, 0, 3, ps32};
        launch_shift(sa, ss.red(kD, E_NONE), s);
      }
      {  // :240-247  seed r0, error test; next rho / beta (:88-92)
        Lc<double> u(np);
        int ir[kBlMaxL + 1];
        for (int i = 0; i <= l; ++i) ir[i] = u.in(R(i));
        const int irs = u.in(rs);
        const int orr = u.out(R(0));
        u.term(orr, ir[0], cf_const(1));
        for (int i = 1; i <= l; ++i)
          u.term(orr, ir[i], cf_slot((short)(kBlOmegaD + i - 1), -1));
        u.dot(OUT + orr, OUT + orr).dot(OUT + orr, irs);
        u.launch(ss.red(kD, E_SHL_CHECK), s);
      }
    };
    const CtlH c = run_loop(ss, body, st);
    o.ret = c.ret;
    o.iters = c.hist_len;
  }
  dfree(w, st);
  dfree(ps, st);
  dfree(ps32, st);
  return o;
}

}  // namespace bk
