// Host drivers of the complex methods.  Each driver is the reference
// routine's statement sequence regrouped into fused launches of the complex
// kernels (kernels_z.cu); the comments cite the reference lines each launch
// covers, and every scalar statement runs in the complex epilogues
// (zepilogues.cuh) on the device.
#include "zsolvers.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace bk {

namespace {

double2* zzeros(long long n, cudaStream_t st) {
  double2* p = dalloc_n<double2>(n, st);
  BK_CHECK(cudaMemsetAsync(p, 0, sizeof(double2) * (size_t)n, st));
  return p;
}

bool no_iterations(int max_iter, double tol, SolveOut& o) {
  if (max_iter > 0) return false;
  o.ret = tol > 0.0 ? 0 : kNotConverged;
  o.iters = 0;
  return true;
}

SolveOut finish(const CtlH& c) {
  SolveOut o;
  o.ret = c.ret;
  o.iters = c.hist_len;
  return o;
}

void set_z(SolveState& ss, short slot, double re, double im, cudaStream_t st) {
  const double v[2] = {re, im};
  ss.set_scalars(slot, v, 2, st);
}

constexpr int Y = 0, B = 1, W0 = 2;   // complex SpMV dot operand codes

ZSpmvH zio(const double2* x, double2* y) {
  ZSpmvH io;
  std::memset(&io, 0, sizeof(io));
  io.x = x;
  io.y = y;
  return io;
}

void zdot_io(ZSpmvH& io, int k, int a, int b) {
  io.dot[k][0] = (unsigned char)a;
  io.dot[k][1] = (unsigned char)b;
  io.dconj[k] = 1;
  io.nd = std::max(io.nd, k + 1);
}

}  // namespace

// ------------------------------------------------------------ operator

void ZDevCsr::release(cudaStream_t st) {
  dfree(rowptr, st);
  dfree(col, st);
  dfree(val, st);
  dfree(rb, st);
  dfree(sptr, st);
  dfree(scol, st);
  dfree(sval, st);
  rowptr = col = rb = sptr = scol = nullptr;
  val = sval = nullptr;
  nslice = 0;
}

void upload_zcsr(int n, const int* rowptr, const int* col, const double* val,
                 bool conj_transpose, ZDevCsr& out, cudaStream_t st) {
  if (n <= 0) throw CudaError("matrix: empty");
  const int nnz = rowptr[n];
  if (rowptr[0] != 0 || nnz < 0) throw CudaError("matrix: bad row pointer");
  for (int i = 0; i < n; ++i)
    if (rowptr[i + 1] < rowptr[i]) throw CudaError("matrix: bad row pointer");
  for (int k = 0; k < nnz; ++k)
    if (col[k] < 0 || col[k] >= n) throw CudaError("matrix: column index out of range");
  // A^H on the host (rows of A^H in the original row order).
  std::vector<int> trp, tc;
  std::vector<double> tv;
  const int* rp = rowptr;
  const int* cc = col;
  const double* vv = val;
  if (conj_transpose) {
    trp.assign(n + 1, 0);
    tc.resize(nnz);
    tv.resize(2 * (size_t)nnz);
    for (int k = 0; k < nnz; ++k) trp[col[k] + 1]++;
    for (int i = 0; i < n; ++i) trp[i + 1] += trp[i];
    std::vector<int> pos(trp.begin(), trp.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        const int p = pos[col[k]]++;
        tc[p] = i;
        tv[2 * (size_t)p] = val[2 * (size_t)k];
        tv[2 * (size_t)p + 1] = -val[2 * (size_t)k + 1];
      }
    rp = trp.data();
    cc = tc.data();
    vv = tv.data();
  }
  const long long padn = (long long)(nnz + 3) / 4 * 4 + 4;
  out.n = n;
  out.nnz = nnz;
  out.rowptr = dalloc_n<int>(n + 1, st);
  out.col = dalloc_n<int>(padn, st);
  out.val = dalloc_n<double2>(padn, st);
  BK_CHECK(cudaMemsetAsync(out.col, 0, sizeof(int) * padn, st));
  BK_CHECK(cudaMemsetAsync(out.val, 0, sizeof(double2) * padn, st));
  BK_CHECK(cudaMemcpyAsync(out.rowptr, rp, sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, st));
  if (nnz > 0) {
    BK_CHECK(cudaMemcpyAsync(out.col, cc, sizeof(int) * nnz,
                             cudaMemcpyHostToDevice, st));
    BK_CHECK(cudaMemcpyAsync(out.val, vv, sizeof(double2) * nnz,
                             cudaMemcpyHostToDevice, st));
  }
  std::vector<int> rb = make_row_blocks(n, rp);
  out.nrb = (int)rb.size() - 1;
  out.rb = dalloc_n<int>((long long)rb.size(), st);
  BK_CHECK(cudaMemcpyAsync(out.rb, rb.data(), sizeof(int) * rb.size(),
                           cudaMemcpyHostToDevice, st));
  // Sliced-ELL copy (32-row slices, entries column-major within a slice,
  // each row in CSR order, padding column -1), placed on the GPU, unless
  // padding would exceed half the entries.
  const int nslice = (n + 31) / 32;
  std::vector<int> sp((size_t)nslice + 1, 0);
  long long total = 0;
  for (int s = 0; s < nslice && total <= 0x7fffff00LL; ++s) {
    int w = 0;
    for (int r = s * 32; r < std::min(n, s * 32 + 32); ++r) w = std::max(w, rp[r + 1] - rp[r]);
    total += 32LL * w;
    sp[s + 1] = (int)std::min(total, 0x7fffff00LL);
  }
  if (total <= 0x7fffff00LL && total <= (long long)nnz * 3 / 2 + 64) {
    out.sptr = dalloc_n<int>(nslice + 1, st);
    out.scol = dalloc_n<int>(total, st);
    out.sval = dalloc_n<double2>(total, st);
    BK_CHECK(cudaMemcpyAsync(out.sptr, sp.data(), sizeof(int) * (nslice + 1),
                             cudaMemcpyHostToDevice, st));
    launch_csr2sell_z(out.rowptr, out.col, out.val, n, nslice, out.sptr,
                      out.scol, out.sval, st);
    BK_CHECK(cudaGetLastError());
    out.nslice = nslice;
  }
  // The host vectors above must outlive the copies.
  BK_CHECK(cudaStreamSynchronize(st));
}

// ------------------------------------------------------------- builder

ZLc::ZLc(long long n) {
  std::memset(&d, 0, sizeof(d));
  d.n = n;
  d.reps = 1;
}
int ZLc::in(const double2* p, bool rep) {
  if (d.nin >= kZLcIn) throw CudaError("complex lincomb: too many inputs");
  const int i = d.nin++;
  d.in[i] = p;
  if (rep) d.in_rep_mask |= 1u << i;
  return i;
}
int ZLc::out(double2* p, bool rep) {
  if (d.nout >= kZLcOut) throw CudaError("complex lincomb: too many outputs");
  const int o = d.nout++;
  d.out[o] = p;
  if (rep) d.out_rep_mask |= 1u << o;
  return o;
}
ZLc& ZLc::term(int o, int i, ZCfH c) {
  d.c[o][i] = c;
  return *this;
}
ZLc& ZLc::dot(int a, int b, bool conj) {
  if (d.nd >= kZDots) throw CudaError("complex lincomb: too many dots");
  d.dot[d.nd][0] = (unsigned char)a;
  d.dot[d.nd][1] = (unsigned char)b;
  d.dconj[d.nd] = conj ? 1 : 0;
  d.nd++;
  return *this;
}
ZLc& ZLc::batch(int reps, long long stride) {
  d.reps = reps;
  d.stride = stride;
  return *this;
}
void ZLc::launch(const RedH& rd, cudaStream_t st) { launch_zlc(d, rd, st); }

// ---------------------------------------------------------------- zbicg
SolveOut zbicg(const ZDevCsr& A, const ZDevCsr& AH, const double2* b,
               double2* x, double tol, int max_iter, SolveState& ss,
               cudaStream_t st) {
  SolveOut o;
  const long long np = pad64(A.n);
  double2* w = zzeros(6 * np, st);
  double2 *r = w, *sr = w + np, *p = w + 2 * np, *sp = w + 3 * np,
          *ap = w + 4 * np, *atp = w + 5 * np;
  ss.start(0, max_iter, tol, st);
  // src/bicg.c:108-117: r = sr = p = sp = b - A x, (sr, r), ||b||.
  ZSpmvH io = zio(x, r);
  io.b = b;
  io.mode = 1;
  io.y2 = p;
  zdot_io(io, 0, B, B);
  zdot_io(io, 1, Y, Y);
  launch_zspmv(A.h(), io, ss.red(kD, EZ_BICG_INIT), st);
  {
    ZLc c(np);
    const int ir = c.in(r);
    const int o1 = c.out(sr), o2 = c.out(sp);
    c.term(o1, ir, zcf_const(1)).term(o2, ir, zcf_const(1));
    c.launch(ss.red(kD, E_NONE), st);
  }
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      // :122-131  ap = A p, atp = A^H sp, alpha = r_dot_old / (sp, ap)
      ZSpmvH a = zio(p, ap);
      a.w0 = sp;
      zdot_io(a, 0, W0, Y);
      launch_zspmv(A.h(), a, ss.red(kD, EZ_BICG_ALPHA), s);
      launch_zspmv(AH.h(), zio(sp, atp), ss.red(kD, E_NONE), s);
      // :136-148, :158  x, r, sr updates, (sr, r), beta, error test
      ZLc u(np);
      const int ix = u.in(x), ip = u.in(p), ir = u.in(r), ia = u.in(ap),
                is = u.in(sr), iat = u.in(atp);
      const int ox = u.out(x), orr = u.out(r), os = u.out(sr);
      u.term(ox, ix, zcf_const(1)).term(ox, ip, zcf_slot(kZAlpha));
      u.term(orr, ir, zcf_const(1)).term(orr, ia, zcf_slot(kZAlpha, -1));
      u.term(os, is, zcf_const(1)).term(os, iat, zcf_conj(kZAlpha, -1));
      u.dot(ZLc::OUT + os, ZLc::OUT + orr).dot(ZLc::OUT + orr, ZLc::OUT + orr);
      u.launch(ss.red(kD, EZ_BICG_CHECK), s);
      // :151-156  p = beta p + r, sp = conj(beta) sp + sr
      ZLc q(np);
      const int jp = q.in(p), jr = q.in(r), js = q.in(sp), jsr = q.in(sr);
      const int op = q.out(p), osp = q.out(sp);
      q.term(op, jp, zcf_slot(kZBeta)).term(op, jr, zcf_const(1));
      q.term(osp, js, zcf_conj(kZBeta)).term(osp, jsr, zcf_const(1));
      q.launch(ss.red(kD, E_NONE), s);
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// ----------------------------------------------------------- zbicgstabl
SolveOut zbicgstabl(const ZDevCsr& A, const double2* b, int l, double2* x,
                    double tol, int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  if (l < 1 || l > kBlMaxL) throw CudaError("zbicgstabl: l out of range");
  const long long np = pad64(A.n);
  double2* w = zzeros((2 * (l + 1) + 1) * np, st);
  auto R = [&](int i) { return w + i * np; };
  auto P = [&](int i) { return w + (l + 1 + i) * np; };
  double2* rs = w + 2 * (l + 1) * np;
  ss.set_scalar(kL, (double)l, st);
  set_z(ss, kZOmega + 2 * l, 1.0, 0.0, st);   // src/bicgstabl.c:169
  set_z(ss, kZG0, 1.0, 0.0, st);              // :151
  ss.start(0, max_iter, tol, st);
  // :175-182: r0 = p0 = rs = b - A x, ||b||; then (rs, r0) and beta for the
  // first j (:187-192).
  ZSpmvH io = zio(x, R(0));
  io.b = b;
  io.mode = 1;
  io.y2 = P(0);
  zdot_io(io, 0, B, B);
  launch_zspmv(A.h(), io, ss.red(kD, EZ_SET_FNB), st);
  {
    ZLc c(np);
    const int ir = c.in(R(0));
    const int o1 = c.out(rs);
    c.term(o1, ir, zcf_const(1));
    c.dot(ZLc::OUT + o1, ir);
    c.launch(ss.red(kD, EZ_BL_BETA0), st);
  }
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      for (int j = 0; j < l; ++j) {          // BiCG part, :189-212
        {  // :194-197  p_i = beta p_i + r_i, i = 0..j
          ZLc u(np);
          const int ip = u.in(P(0), true), ir = u.in(R(0), true);
          const int op = u.out(P(0), true);
          u.term(op, ip, zcf_slot(kZBeta)).term(op, ir, zcf_const(1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
        }
        {  // :198-202  p_{j+1} = A p_j, alpha = gamma1 / (rs, p_{j+1})
          ZSpmvH a = zio(P(j), P(j + 1));
          a.w0 = rs;
          zdot_io(a, 0, W0, Y);
          launch_zspmv(A.h(), a, ss.red(kD, EZ_BL_ALPHA), s);
        }
        if (j + 2 <= kZLcOut) {   // :204-207 and :211 in one pass
          ZLc u(np);
          const int ix = u.in(x), ip0 = u.in(P(0));
          const int ox = u.out(x);
          u.term(ox, ix, zcf_const(1)).term(ox, ip0, zcf_slot(kZAlpha));
          for (int i = 0; i <= j; ++i) {
            const int ir = u.in(R(i)), ip = u.in(P(i + 1));
            const int orr = u.out(R(i));
            u.term(orr, ir, zcf_const(1)).term(orr, ip, zcf_slot(kZAlpha, -1));
          }
          u.launch(ss.red(kD, E_NONE), s);
        } else {
          ZLc u(np);
          const int ir = u.in(R(0), true), ip = u.in(P(1), true);
          const int orr = u.out(R(0), true);
          u.term(orr, ir, zcf_const(1)).term(orr, ip, zcf_slot(kZAlpha, -1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
          ZLc v(np);
          const int ix = v.in(x), ip0 = v.in(P(0));
          const int ox = v.out(x);
          v.term(ox, ix, zcf_const(1)).term(ox, ip0, zcf_slot(kZAlpha));
          v.launch(ss.red(kD, E_NONE), s);
        }
        {  // :208-209  r_{j+1} = A r_j (+ (rs, r_{j+1}) for the next j, :190)
          ZSpmvH a = zio(R(j), R(j + 1));
          if (j + 1 < l) {
            a.w0 = rs;
            zdot_io(a, 0, W0, Y);
            launch_zspmv(A.h(), a, ss.red(kD, EZ_BL_BETA), s);
          } else {
            launch_zspmv(A.h(), a, ss.red(kD, E_NONE), s);
          }
        }
      }
      // MR part, :216-226: modified Gram-Schmidt on r_1..r_l.
      for (int j = 1; j <= l; ++j) {
        if (j == 1) {
          ZLc u(np);
          const int i1 = u.in(R(1)), i0 = u.in(R(0));
          u.dot(i1, i1).dot(i1, i0);
          u.launch(ss.red(kD, EZ_BL_SIG, 0, 1), s);
          continue;
        }
        {
          ZLc u(np);
          const int i1 = u.in(R(1)), ij = u.in(R(j));
          u.dot(i1, ij);
          u.launch(ss.red(kD, EZ_BL_TAU, 1, (short)j), s);
        }
        for (int i = 1; i < j; ++i) {
          ZLc u(np);
          const int ij = u.in(R(j)), ii = u.in(R(i));
          const int oj = u.out(R(j));
          u.term(oj, ij, zcf_const(1))
              .term(oj, ii, zcf_slot((short)(kZTau + 2 * (j * l + i)), -1));
          if (i + 1 < j) {
            const int in = u.in(R(i + 1));
            u.dot(in, ZLc::OUT + oj);
            u.launch(ss.red(kD, EZ_BL_TAU, (short)(i + 1), (short)j), s);
          } else {
            const int i0 = u.in(R(0));
            u.dot(ZLc::OUT + oj, ZLc::OUT + oj).dot(ZLc::OUT + oj, i0);
            u.launch(ss.red(kD, EZ_BL_SIG, 0, (short)j), s);
          }
        }
      }
      {  // update, :247-258, error :260, (rs, r0) of the next iteration
        ZLc u(np);
        const int ix = u.in(x);
        int ir[kBlMaxL + 1], ip[kBlMaxL + 1];
        for (int i = 0; i <= l; ++i) ir[i] = u.in(R(i));
        for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
        const int irs = u.in(rs);
        const int ox = u.out(x), orr = u.out(R(0)), op = u.out(P(0));
        u.term(ox, ix, zcf_const(1)).term(ox, ir[0], zcf_slot((short)(kZOmega + 2)));
        u.term(orr, ir[0], zcf_const(1))
            .term(orr, ir[l], zcf_slot((short)(kZOmegaD + 2 * l), -1));
        u.term(op, ip[0], zcf_const(1))
            .term(op, ip[l], zcf_slot((short)(kZOmega + 2 * l), -1));
        for (int i = 1; i < l; ++i) {
          u.term(op, ip[i], zcf_slot((short)(kZOmega + 2 * i), -1));
          u.term(orr, ir[i], zcf_slot((short)(kZOmegaD + 2 * i), -1));
          u.term(ox, ir[i], zcf_slot((short)(kZOmegaDD + 2 * i)));
        }
        u.dot(ZLc::OUT + orr, ZLc::OUT + orr).dot(irs, ZLc::OUT + orr);
        u.launch(ss.red(kD, EZ_BL_CHECK), s);
      }
    };
    o = finish(run_loop(ss, body, st));
  }
  dfree(w, st);
  return o;
}

// --------------------------------------------------------- zshbicgstabl
SolveOut zshbicgstabl(const ZDevCsr& A, const double2* b, int l,
                      const double* sigma, int ns, double2* x, double tol,
                      int max_iter, SolveState& ss, cudaStream_t st) {
  SolveOut o;
  if (l < 1 || l > kBlMaxL) throw CudaError("zshbicgstabl: l out of range");
  if (ns < 0 || ns > kZMaxShifts) throw CudaError("zshbicgstabl: too many shifts");
  const long long np = pad64(A.n);
  double2* w = zzeros((2 * (l + 1) + 1) * np, st);
  auto R = [&](int i) { return w + i * np; };
  auto P = [&](int i) { return w + (l + 1 + i) * np; };
  double2* rs = w + 2 * (l + 1) * np;
  double2* PS = ns > 0 ? zzeros((long long)ns * (l + 1) * np, st) : nullptr;
  ss.set_scalar(kL, (double)l, st);
  ss.set_scalar(kNs, (double)ns, st);
  set_z(ss, kZOmega + 2 * (l - 1), 1.0, 0.0, st);   // src/shbicgstabl.c:316
  set_z(ss, kZAlphaOld, 1.0, 0.0, st);              // :331
  set_z(ss, kZRdot, 1.0, 0.0, st);                  // :332 rho_old
  if (ns > 0) {                                     // :361-367
    std::vector<double> one(2 * (size_t)ns);
    for (int k = 0; k < ns; ++k) { one[2 * k] = 1.0; one[2 * k + 1] = 0.0; }
    ss.set_scalars(kZShSigma, sigma, 2 * ns, st);
    ss.set_scalars(kZShPi, one.data(), 2 * ns, st);
    ss.set_scalars(kZShPiOld, one.data(), 2 * ns, st);
    ss.set_scalars(kZShTheta, one.data(), 2 * ns, st);
  }
  ss.start(0, max_iter, tol, st);
  auto shift = [&](int mode, int j, cudaStream_t s) {
    if (ns == 0) return;
    ZShiftH h{PS, x + np, R(0), np, ns, l, j, mode};
    launch_zshift(h, ss.red(kD, E_NONE), s);
  };
  // :322-329: r0 = p0 = rs = b - A x, ||b||; then rho_old, rho = (rs, r0)
  // and beta for the first step (:391-395).
  ZSpmvH io = zio(x, R(0));
  io.b = b;
  io.mode = 1;
  io.y2 = P(0);
  zdot_io(io, 0, B, B);
  launch_zspmv(A.h(), io, ss.red(kD, EZ_SH_INIT), st);
  {
    ZLc c(np);
    const int ir = c.in(R(0));
    const int o1 = c.out(rs);
    c.term(o1, ir, zcf_const(1));
    c.dot(ir, ir).dot(ZLc::OUT + o1, ir);
    c.launch(ss.red(kD, EZ_SH_CHECK, 1), st);
  }
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t s) {
      for (int j = 0; j < l; ++j) {          // BiCG part, :392-472
        {  // :398-402  p_i = -beta p_i + r_i
          ZLc u(np);
          const int ip = u.in(P(0), true), ir = u.in(R(0), true);
          const int op = u.out(P(0), true);
          u.term(op, ip, zcf_slot(kZBeta, -1)).term(op, ir, zcf_const(1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
        }
        {  // :405-410 p_{j+1} = A p_j, alpha; :416-442's per-shift scalars
          ZSpmvH a = zio(P(j), P(j + 1));
          a.w0 = rs;
          zdot_io(a, 0, W0, Y);
          launch_zspmv(A.h(), a, ss.red(kD, EZ_SH_ALPHA), s);
        }
        shift(0, j, s);                      // :429-441 (before r changes)
        if (j + 2 <= kZLcOut) {              // :413, :445-448
          ZLc u(np);
          const int ix = u.in(x), ip0 = u.in(P(0));
          const int ox = u.out(x);
          u.term(ox, ix, zcf_const(1)).term(ox, ip0, zcf_slot(kZAlpha));
          for (int i = 0; i <= j; ++i) {
            const int ir = u.in(R(i)), ip = u.in(P(i + 1));
            const int orr = u.out(R(i));
            u.term(orr, ir, zcf_const(1)).term(orr, ip, zcf_slot(kZAlpha, -1));
          }
          u.launch(ss.red(kD, E_NONE), s);
        } else {
          ZLc u(np);
          const int ir = u.in(R(0), true), ip = u.in(P(1), true);
          const int orr = u.out(R(0), true);
          u.term(orr, ir, zcf_const(1)).term(orr, ip, zcf_slot(kZAlpha, -1));
          u.batch(j + 1, np);
          u.launch(ss.red(kD, E_NONE), s);
          ZLc v(np);
          const int ix = v.in(x), ip0 = v.in(P(0));
          const int ox = v.out(x);
          v.term(ox, ix, zcf_const(1)).term(ox, ip0, zcf_slot(kZAlpha));
          v.launch(ss.red(kD, E_NONE), s);
        }
        {  // :451-452 r_{j+1} = A r_j; :466-471 (+ rho, beta of the next j)
          ZSpmvH a = zio(R(j), R(j + 1));
          if (j + 1 < l) {
            a.w0 = rs;
            zdot_io(a, 0, W0, Y);
            launch_zspmv(A.h(), a, ss.red(kD, EZ_SH_STEP, 1), s);
          } else {
            launch_zspmv(A.h(), a, ss.red(kD, EZ_SH_STEP, 0), s);
          }
        }
        shift(1, j, s);                      // :455-463
      }
      // MR part, :477-487 (r_1..r_l, the l - 1 index convention).
      for (int j = 0; j < l; ++j) {
        if (j == 0) {
          ZLc u(np);
          const int i1 = u.in(R(1)), i0 = u.in(R(0));
          u.dot(i1, i1).dot(i1, i0);
          u.launch(ss.red(kD, EZ_SH_SIG, 0, 0), s);
          continue;
        }
        {
          ZLc u(np);
          const int i1 = u.in(R(1)), ij = u.in(R(j + 1));
          u.dot(i1, ij);
          u.launch(ss.red(kD, EZ_SH_TAU, 0, (short)j), s);
        }
        for (int i = 0; i < j; ++i) {
          ZLc u(np);
          const int ij = u.in(R(j + 1)), ii = u.in(R(i + 1));
          const int oj = u.out(R(j + 1));
          u.term(oj, ij, zcf_const(1))
              .term(oj, ii, zcf_slot((short)(kZTau + 2 * (j * l + i)), -1));
          if (i + 1 < j) {
            const int in = u.in(R(i + 2));
            u.dot(in, ZLc::OUT + oj);
            u.launch(ss.red(kD, EZ_SH_TAU, (short)(i + 1), (short)j), s);
          } else {
            const int i0 = u.in(R(0));
            u.dot(ZLc::OUT + oj, ZLc::OUT + oj).dot(ZLc::OUT + oj, i0);
            u.launch(ss.red(kD, EZ_SH_SIG, 0, (short)j), s);
          }
        }
      }
      shift(2, 0, s);                        // :518-557 (before r0 changes)
      {  // :508-515 seed x, p0; :560-563 r0; :565 error; rho of the next
        ZLc u(np);
        const int ix = u.in(x);
        int ir[kBlMaxL + 1], ip[kBlMaxL + 1];
        for (int i = 0; i <= l; ++i) ir[i] = u.in(R(i));
        for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
        const int irs = u.in(rs);
        const int ox = u.out(x), orr = u.out(R(0)), op = u.out(P(0));
        u.term(ox, ix, zcf_const(1)).term(ox, ir[0], zcf_slot(kZOmega));
        u.term(op, ip[0], zcf_const(1))
            .term(op, ip[l], zcf_slot((short)(kZOmega + 2 * (l - 1)), -1));
        u.term(orr, ir[0], zcf_const(1));
        for (int i = 1; i < l; ++i) {
          u.term(op, ip[i], zcf_slot((short)(kZOmega + 2 * (i - 1)), -1));
          u.term(ox, ir[i], zcf_slot((short)(kZOmegaDD + 2 * (i - 1))));
        }
        for (int i = 1; i <= l; ++i)
          u.term(orr, ir[i], zcf_slot((short)(kZOmegaD + 2 * (i - 1)), -1));
        u.dot(ZLc::OUT + orr, ZLc::OUT + orr).dot(irs, ZLc::OUT + orr);
        u.launch(ss.red(kD, EZ_SH_CHECK, 0), s);
      }
    };
    o = finish(run_loop(ss, body, st));
  }
  if (PS) dfree(PS, st);
  dfree(w, st);
  return o;
}

// --------------------------------------------------------- block methods

namespace {

// Builder of one complex block launch (ZBlkH).
struct ZBlk {
  ZBlkH a;
  ZBlk(long long rows, int s) {
    std::memset(&a, 0, sizeof(a));
    a.n = rows;
    a.s = s;
    for (int o = 0; o < 2; ++o)
      for (int i = 0; i < 4; ++i) a.mslot[o][i] = -1;
  }
  static constexpr int OUTB = 4;   // operand code base of outputs (Grams, dots)
  int in(const double2* p) {
    if (a.nin >= 4) throw CudaError("complex block kernel: too many inputs");
    a.in[a.nin] = p;
    return a.nin++;
  }
  int out(double2* p) {
    if (a.nout >= 2) throw CudaError("complex block kernel: too many outputs");
    a.out[a.nout] = p;
    return a.nout++;
  }
  ZBlk& scal(int o, int i, ZCfH c) {
    a.c[o][i] = c;
    return *this;
  }
  // out[o] += k in[i] M, M the s-by-s matrix at slot m.
  ZBlk& mat(int o, int i, short m, double k = 1.0) {
    a.c[o][i] = zcf_const(k);
    a.mslot[o][i] = m;
    return *this;
  }
  // Gram G = U^T V (conj false) or U^H V to slot g; operands: input index
  // or OUTB + output index.
  ZBlk& gram(int u, int v, short g, bool conj) {
    a.gram[a.ng][0] = (unsigned char)code(u);
    a.gram[a.ng][1] = (unsigned char)code(v);
    a.gconj[a.ng] = conj ? 1 : 0;
    a.gslot[a.ng] = g;
    a.ng++;
    return *this;
  }
  ZBlk& dot(int u, int v) {
    a.dot[a.nd][0] = (unsigned char)code(u);
    a.dot[a.nd][1] = (unsigned char)code(v);
    a.nd++;
    return *this;
  }
  int code(int u) const { return u >= OUTB ? a.nin + (u - OUTB) : u; }
  void launch(const RedH& rd, cudaStream_t st) { launch_zblock(a, rd, st); }
};

ZSpmmH zspmm_args(const double2* X, double2* Y, int s, int alpha = 1,
                  const double2* C = nullptr) {
  ZSpmmH h{X, Y, C, s, alpha, C ? 1 : 0};
  return h;
}

struct ZBlockCtx {
  int n, s;
  long long np;
  SolveState& ss;
  cudaStream_t st;
  double* bpart = nullptr;
  std::vector<void*> owned;
  ZBlockCtx(int n_, int s_, SolveState& ss_, cudaStream_t st_)
      : n(n_), s(s_), np(pad64(n_)), ss(ss_), st(st_) {
    if (s < 1 || s > 16) throw CudaError("complex block width out of range");
    bpart = dalloc_n<double>(red2_doubles(kZBlkPart), st);
    BK_CHECK(cudaMemsetAsync(bpart + red2_ticket_offset(kZBlkPart), 0,
                             kRedGroups * sizeof(double), st));
  }
  ~ZBlockCtx() {
    for (void* p : owned) dfree(p, st);
    dfree(bpart, st);
  }
  RedH red(short out, short epi, short a0 = 0, short a1 = 0) const {
    return RedH{bpart, ss.ticket, ss.S, ss.ctl, out, epi, a0, a1, 0};
  }
  // For launches after the iteration loop (never skipped).
  RedH red_after(short out, short epi) const {
    return RedH{bpart, ss.ticket, ss.S, ss.ctl_free, out, epi, 0, 0, 0};
  }
  double2* blocks(int count) {
    double2* p = zzeros((long long)count * np * s, st);
    owned.push_back(p);
    return p;
  }
  // Passes 2 and 3 of the complex Cholesky-QR of V (pass 1's epilogue ran
  // on the launch that produced V^H V), then V = V R3^-1 (also to `copy`).
  void qr_tail(double2* V, short post, double2* copy, cudaStream_t s_) {
    for (int pass = 2; pass <= 3; ++pass) {
      ZBlk b(np, s);
      const int iv = b.in(V);
      const int ov = b.out(V);
      b.mat(ov, iv, kZBkRinv);
      b.gram(ZBlk::OUTB + ov, ZBlk::OUTB + ov, kZBkG1, true);
      b.launch(red(kD, pass == 2 ? EZ_QR2 : EZ_QR3, pass == 3 ? post : 0), s_);
    }
    ZBlk b(np, s);
    const int iv = b.in(V);
    const int ov = b.out(V);
    b.mat(ov, iv, kZBkRinv);
    if (copy) {
      const int oc = b.out(copy);
      b.mat(oc, iv, kZBkRinv);
    }
    b.launch(red(kD, E_NONE), s_);
  }
};

}  // namespace

// --------------------------------------------------------- zblbicgstabl
SolveOut zblbicgstabl(const ZDevCsr& A, const double2* Bm, int s, int l,
                      double2* X, double tol, int max_iter, SolveState& ss,
                      cudaStream_t st, double* true_res) {
  if (l < 1 || l > kBlMaxL) throw CudaError("zblbicgstabl: l out of range");
  ZBlockCtx bc(A.n, s, ss, st);
  const long long np = bc.np, bs = np * s;
  double2* Vb = bc.blocks(l + 1);
  double2* Pb = bc.blocks(l + 1);
  double2* Rb = bc.blocks(l + 1);
  double2* Rs = bc.blocks(1);
  double2* Tm = bc.blocks(1);
  auto V = [&](int i) { return Vb + i * bs; };
  auto P = [&](int i) { return Pb + i * bs; };
  auto R = [&](int i) { return Rb + i * bs; };
  ss.start(0, max_iter, tol, st);
  ss.set_scalar(kZBkS, (double)s, st);
  ss.set_scalar(kZBkRows, (double)A.n, st);
  ss.set_scalar(kL, (double)l, st);
  set_z(ss, kZOmega + 2 * (l - 1), 1.0, 0.0, st);   // src/blbicgstabl.c:279
  {                                                  // :287-289 gamma0 = I
    std::vector<double> eye(2 * (size_t)s * s, 0.0);
    for (int i = 0; i < s; ++i) eye[2 * (i * s + i)] = 1.0;
    ss.set_scalars(kZBkGam0, eye.data(), 2 * s * s, st);
  }
  // :321-333: V0 = B + A X (the reference's sign), zqreco(V0, xi), P0 = Rs
  // = V0, ||B||_F.
  launch_zspmm(A.h(), zspmm_args(X, V(0), s), bc.red(kD, E_NONE), st);
  {
    ZBlk b(np, s);
    const int iv = b.in(V(0)), ib = b.in(Bm);
    const int ov = b.out(V(0));
    b.scal(ov, iv, zcf_const(1)).scal(ov, ib, zcf_const(1));
    b.gram(ZBlk::OUTB + ov, ZBlk::OUTB + ov, kZBkG1, true).dot(ib, ib);
    b.launch(bc.red(kD, EZ_BB_INIT), st);
  }
  bc.qr_tail(V(0), ZQR_POST_INIT, P(0), st);
  {
    ZBlk b(np, s);
    const int iv = b.in(V(0));
    const int os = b.out(Rs);
    b.scal(os, iv, zcf_const(1));
    b.launch(bc.red(kD, E_NONE), st);
  }
  SolveOut o;
  if (!no_iterations(max_iter, tol, o)) {
    auto body = [&](cudaStream_t sm) {
      for (int j = 0; j < l; ++j) {
        {  // :343-349  gamma1 = Rs^T V_j, beta
          ZBlk b(np, s);
          const int is = b.in(Rs), iv = b.in(V(j));
          b.gram(is, iv, kZBkG1, false);
          b.launch(bc.red(kD, EZ_BB_BETA), sm);
        }
        for (int i = 0; i <= j; ++i) {   // :352-357  P_i = V_i - P_i beta
          ZBlk b(np, s);
          const int ip = b.in(P(i)), iv = b.in(V(i));
          const int op = b.out(P(i));
          b.mat(op, ip, kZBkBeta, -1.0).scal(op, iv, zcf_const(1));
          b.launch(bc.red(kD, E_NONE), sm);
        }
        launch_zspmm(A.h(), zspmm_args(P(j), P(j + 1), s), bc.red(kD, E_NONE), sm);
        {  // :362-365  alpha = (Rs^T P_{j+1})^-1 gamma1
          ZBlk b(np, s);
          const int is = b.in(Rs), ip = b.in(P(j + 1));
          b.gram(is, ip, kZBkG1, false);
          b.launch(bc.red(kD, EZ_BB_ALPHA), sm);
        }
        {  // :370-373  tmp = P_0 alpha, V_0 -= A tmp
          ZBlk b(np, s);
          const int ip = b.in(P(0));
          const int ot = b.out(Tm);
          b.mat(ot, ip, kZBkAlpha);
          b.launch(bc.red(kD, E_NONE), sm);
        }
        launch_zspmm(A.h(), zspmm_args(Tm, V(0), s, -1, V(0)), bc.red(kD, E_NONE), sm);
        {  // :376  zqreco(V_0, t)
          ZBlk b(np, s);
          const int iv = b.in(V(0));
          b.gram(iv, iv, kZBkG1, true);
          b.launch(bc.red(kD, EZ_QR1), sm);
        }
        bc.qr_tail(V(0), ZQR_POST_T, nullptr, sm);   // + :384-390
        {  // :379-381  X += tmp xi (xi before the update)
          ZBlk b(np, s);
          const int ix = b.in(X), it = b.in(Tm);
          const int ox = b.out(X);
          b.scal(ox, ix, zcf_const(1)).mat(ox, it, kZBkXiOld);
          b.launch(bc.red(kD, E_NONE), sm);
        }
        for (int i = 1; i <= j; ++i) {   // :393-397  V_i = (V_i - P_{i+1} alpha) t^-1
          ZBlk b(np, s);
          const int iv = b.in(V(i)), ip = b.in(P(i + 1));
          const int ov = b.out(V(i));
          b.mat(ov, iv, kZBkTinv).mat(ov, ip, kZBkATinv, -1.0);
          b.launch(bc.red(kD, E_NONE), sm);
        }
        launch_zspmm(A.h(), zspmm_args(V(j), V(j + 1), s), bc.red(kD, E_NONE), sm);   // :401
      }
      for (int i = 0; i <= l; ++i) {   // :405-408  R_i = V_i xi
        ZBlk b(np, s);
        const int iv = b.in(V(i));
        const int orr = b.out(R(i));
        b.mat(orr, iv, kZBkXi);
        b.launch(bc.red(kD, E_NONE), sm);
      }
      // MR part, :412-422, on blocks as vectors of n s entries.
      for (int j = 0; j < l; ++j) {
        if (j == 0) {
          ZLc u(bs);
          const int i1 = u.in(R(1)), i0 = u.in(R(0));
          u.dot(i1, i1).dot(i1, i0);
          u.launch(ss.red(kD, EZ_BB_SIG, 0, 0), sm);
          continue;
        }
        {
          ZLc u(bs);
          const int i1 = u.in(R(1)), ij = u.in(R(j + 1));
          u.dot(i1, ij);
          u.launch(ss.red(kD, EZ_BB_TAU, 0, (short)j), sm);
        }
        for (int i = 0; i < j; ++i) {
          ZLc u(bs);
          const int ij = u.in(R(j + 1)), ii = u.in(R(i + 1));
          const int oj = u.out(R(j + 1));
          u.term(oj, ij, zcf_const(1))
              .term(oj, ii, zcf_slot((short)(kZTau + 2 * (j * l + i)), -1));
          if (i + 1 < j) {
            const int in = u.in(R(i + 2));
            u.dot(in, ZLc::OUT + oj);
            u.launch(ss.red(kD, EZ_BB_TAU, (short)(i + 1), (short)j), sm);
          } else {
            const int i0 = u.in(R(0));
            u.dot(ZLc::OUT + oj, ZLc::OUT + oj).dot(ZLc::OUT + oj, i0);
            u.launch(ss.red(kD, EZ_BB_SIG, 0, (short)j), sm);
          }
        }
      }
      {  // :442-448  tmp = sum omega_i V_i, P_0 -= sum omega_i P_{i+1}
        ZLc u(bs);
        int iv[kBlMaxL], ip[kBlMaxL + 1];
        for (int i = 0; i < l; ++i) iv[i] = u.in(V(i));
        for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
        const int ot = u.out(Tm), op = u.out(P(0));
        u.term(op, ip[0], zcf_const(1));
        for (int i = 0; i < l; ++i) {
          u.term(ot, iv[i], zcf_slot((short)(kZOmega + 2 * i)));
          u.term(op, ip[i + 1], zcf_slot((short)(kZOmega + 2 * i), -1));
        }
        u.launch(ss.red(kD, E_NONE), sm);
      }
      launch_zspmm(A.h(), zspmm_args(Tm, V(0), s, -1, V(0)), bc.red(kD, E_NONE), sm);   // :449-450
      {  // :451-457  X += tmp xi, error = ||xi||_F / ||B||_F
        ZBlk b(np, s);
        const int ix = b.in(X), it = b.in(Tm);
        const int ox = b.out(X);
        b.scal(ox, ix, zcf_const(1)).mat(ox, it, kZBkXi);
        b.launch(bc.red(kD, EZ_BB_CHECK), sm);
      }
    };
    o = finish(run_loop(ss, body, st));
  }
  if (true_res) {   // :461-469  ||B - A X||_F / ||B||_F
    launch_zspmm(A.h(), zspmm_args(X, Tm, s, -1, Bm), bc.red_after(kD, E_NONE), st);
    ZLc u(bs);
    const int it = u.in(Tm);
    u.dot(it, it);
    u.launch(ss.red_after(kD, E_NONE), st);
    const double tt = ss.get_scalar(kD, st);
    *true_res = std::sqrt(tt) / ss.get_scalar(kFnb, st);
  }
  return o;
}

// ------------------------------------------------------------- zqreco
bool zthin_qr(int n, int s, double2* V, double* R_host, SolveState& ss,
              cudaStream_t st) {
  ZBlockCtx bc(n, s, ss, st);
  ss.start(0, 1, 0.0, st);
  ss.set_scalar(kZBkS, (double)s, st);
  ss.set_scalar(kZBkRows, (double)n, st);
  ZBlk b(bc.np, s);
  const int iv = b.in(V);
  b.gram(iv, iv, kZBkG1, true);
  b.launch(bc.red(kD, EZ_QR1), st);
  bc.qr_tail(V, ZQR_POST_NONE, nullptr, st);
  const CtlH c = ss.read(st);
  BK_CHECK(cudaMemcpyAsync(R_host, ss.S + kZBkR, sizeof(double) * 2 * s * s,
                           cudaMemcpyDeviceToHost, st));
  BK_CHECK(cudaStreamSynchronize(st));
  return c.ret != kDivergence;
}

}  // namespace bk
