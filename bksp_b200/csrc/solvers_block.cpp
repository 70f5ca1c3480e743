// Host drivers of the block methods and of the thin QR (myqr).  Blocks are
// row-major np x s on the device; each reference statement group becomes
// one SpMM or one fused block kernel (linear combination + Gram products),
// and all s-by-s algebra runs in the device epilogues (epi_block.cuh).
#include "solvers_block.h"

#include <algorithm>
#include <cstdio>

namespace bk {

namespace {

constexpr int OUTB = 100;   // Gram / dot operand code base for outputs

// Builder of one fused block launch (BlkH).
struct Blk {
  BlkH d;
  // prec 1: FP32 blocks (the pointers below then point to floats).
  Blk(long long n, int s, int prec = 0) {
    std::memset(&d, 0, sizeof(d));
    d.n = n;
    d.s = s;
    d.prec = prec;
    for (int o = 0; o < 2; ++o)
      for (int i = 0; i < 4; ++i) d.mslot[o][i] = -1;
  }
  int in(const void* p) {
    if (d.nin >= 4) throw CudaError("block kernel: too many inputs");
    d.in[d.nin] = static_cast<const double*>(p);
    return d.nin++;
  }
  int out(void* p) {
    if (d.nout >= 2) throw CudaError("block kernel: too many outputs");
    d.out[d.nout] = static_cast<double*>(p);
    return d.nout++;
  }
  Blk& scal(int o, int i, CfH c) {
    d.c[o][i] = c;
    return *this;
  }
  Blk& mat(int o, int i, short slot, bool trans = false, CfH c = cf_const(1)) {
    d.c[o][i] = c;
    d.mslot[o][i] = slot;
    d.trans[o][i] = trans ? 1 : 0;
    return *this;
  }
  int code(int x) const { return x >= OUTB ? d.nin + (x - OUTB) : x; }
  Blk& gram(int u, int v, short slot) {
    if (d.ng >= 2) throw CudaError("block kernel: too many Gram products");
    grams_.push_back({u, v});
    d.gslot[d.ng++] = slot;
    return *this;
  }
  Blk& dot(int u, int v) {
    if (d.nd >= 2) throw CudaError("block kernel: too many dots");
    dots_.push_back({u, v});
    d.nd++;
    return *this;
  }
  void launch(const RedH& rd, cudaStream_t st) {
    for (size_t g = 0; g < grams_.size(); ++g) {
      d.gram[g][0] = (unsigned char)code(grams_[g].first);
      d.gram[g][1] = (unsigned char)code(grams_[g].second);
    }
    for (size_t k = 0; k < dots_.size(); ++k) {
      d.dot[k][0] = (unsigned char)code(dots_[k].first);
      d.dot[k][1] = (unsigned char)code(dots_[k].second);
    }
    launch_block(d, rd, st);
  }
 private:
  std::vector<std::pair<int, int>> grams_, dots_;
};

template <typename T> constexpr int prec_of() { return sizeof(T) == 4 ? 1 : 0; }

template <typename T>
SpmmH spmm_args(const T* X, T* Y, int s, double alpha = 1.0, const T* C = nullptr) {
  SpmmH a;
  std::memset(&a, 0, sizeof(a));
  a.X = reinterpret_cast<const double*>(X);
  a.Y = reinterpret_cast<double*>(Y);
  a.C = reinterpret_cast<const double*>(C);
  a.alpha = alpha;
  a.mode = C ? 1 : 0;
  a.s = s;
  a.prec = prec_of<T>();
  return a;
}

void spmm(const DevCsr& A, const SpmmH& a, const RedH& rd, cudaStream_t st) {
  if (a.prec == 1 && !A.v32) throw CudaError("FP32 block product: FP32 values missing");
  const CsrH h = a.prec == 1 ? A.h32() : A.h64();
  // The drivers' first products run before their loops are captured: the
  // autotuner's one-time timing happens there.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (!g_prog_rec && cudaStreamIsCapturing(st, &cs) == cudaSuccess &&
      cs == cudaStreamCaptureStatusNone)
    spmm_autotune(h, a.s, a.prec, st);
  cudaGetLastError();
  launch_spmm(h, a, rd, st);
}

}  // namespace

BlockCtx::BlockCtx(int n_, int s_, SolveState& ss_, cudaStream_t st_)
    : n(n_), s(s_), np(pad64(n_)), ss(ss_), st(st_) {
  if (s < 1 || s > kBlockMaxS) throw CudaError("block width out of range");
  bpart = dalloc_n<double>(red2_doubles(514), st);
  BK_CHECK(cudaMemsetAsync(bpart + red2_ticket_offset(514), 0,
                           kRedGroups * sizeof(double), st));
}

BlockCtx::~BlockCtx() { dfree(bpart, st); }

RedH BlockCtx::red(short out, short epi, short a0, short a1) const {
  return RedH{bpart, ss.ticket, ss.S, ss.ctl, out, epi, a0, a1, 0};
}

void* BlockCtx::block_bytes(int count, size_t esz) {
  void* p = dalloc((size_t)count * np * s * esz, st);
  BK_CHECK(cudaMemsetAsync(p, 0, (size_t)count * np * s * esz, st));
  owned.push_back(p);
  return p;
}

void BlockCtx::release() {
  for (void* p : owned) dfree(p, st);
  owned.clear();
}

void BlockCtx::start(int max_iter, double tol) {
  ss.start(0, max_iter, tol, st);
  ss.set_scalar(kBkS, (double)s, st);
  ss.set_scalar(kBkRows, (double)n, st);
  ss.set_scalar(kBkU, unit, st);
}

// Passes 2 and 3 of the Cholesky-QR of V (pass 1's epilogue ran on the
// kernel that produced V and its Gram), then V = V R3^-1, optionally copied
// to `copy` as well.  `post` runs after pass 3 (QR_POST_*).
template <typename T>
void BlockCtx::qr_tail(T* V, short post, typename Same<T>::type* copy, cudaStream_t s_) {
  const long long rows = np;
  constexpr int PR = prec_of<T>();
  for (int pass = 2; pass <= 3; ++pass) {
    Blk b(rows, s, PR);
    const int iv = b.in(V);
    const int ov = b.out(V);
    b.mat(ov, iv, kBkRinv);
    b.gram(OUTB + ov, OUTB + ov, kBkG1);
    b.launch(red(kD, pass == 2 ? E_QR2 : E_QR3, pass == 3 ? post : 0), s_);
  }
  Blk b(rows, s, PR);
  const int iv = b.in(V);
  const int ov = b.out(V);
  b.mat(ov, iv, kBkRinv);
  if (copy) {
    const int oc = b.out(copy);
    b.mat(oc, iv, kBkRinv);
  }
  b.launch(red(kD, E_NONE), s_);
}
template void BlockCtx::qr_tail<double>(double*, short, double*, cudaStream_t);
template void BlockCtx::qr_tail<float>(float*, short, float*, cudaStream_t);

// ------------------------------------------------------------- Block CG
template <typename T>
SolveOut blcg(BlockCtx& bc, const DevCsr& A, const T* B, T* X, double tol,
              int max_iter) {
  constexpr int PR = prec_of<T>();
  bc.unit = PR ? 5.9604644775390625e-08 : 1.1102230246251565e-16;
  cudaStream_t st = bc.st;
  const int s = bc.s;
  const long long rows = bc.np;
  T* V = bc.block<T>(1);
  T* P = bc.block<T>(1);
  T* AP = bc.block<T>(1);
  bc.start(max_iter, tol);
  // src/blcg.c:54-63: V = B - A X, ||B||_F, myqr(V, C), P = V, beta = I.
  spmm(A, spmm_args(X, V, s, -1.0, B), bc.red(kD, E_NONE), st);
  {
    Blk b(rows, s, PR);
    const int iv = b.in(V), ib = b.in(B);
    b.gram(iv, iv, kBkG1).dot(ib, ib);
    b.launch(bc.red(kD, E_BCG_INIT), st);
  }
  bc.qr_tail(V, QR_POST_BCG_INIT, P, st);
  SolveOut o;
  if (max_iter <= 0) {
    o.ret = tol > 0 ? 0 : kNotConverged;
    return o;
  }
  auto body = [&](cudaStream_t sm) {
    {  // :68-71  P = V + P beta^T
      Blk b(rows, s, PR);
      const int iv = b.in(V), ip = b.in(P);
      const int op = b.out(P);
      b.scal(op, iv, cf_const(1)).mat(op, ip, kBkBeta, true);
      b.launch(bc.red(kD, E_NONE), sm);
    }
    spmm(A, spmm_args(P, AP, s), bc.red(kD, E_NONE), sm);   // :74
    {  // :78-86  alpha = (P^T AP)^-1, alpha C
      Blk b(rows, s, PR);
      const int ip = b.in(P), ia = b.in(AP);
      b.gram(ip, ia, kBkG1);
      b.launch(bc.red(kD, E_BCG_ALPHA), sm);
    }
    {  // :87-92  X += P (alpha C), V -= AP alpha; Gram of V for myqr (:95)
      Blk b(rows, s, PR);
      const int ix = b.in(X), ip = b.in(P), iv = b.in(V), ia = b.in(AP);
      const int ox = b.out(X), ov = b.out(V);
      b.scal(ox, ix, cf_const(1)).mat(ox, ip, kBkTmp);
      b.scal(ov, iv, cf_const(1)).mat(ov, ia, kBkAlpha, false, cf_const(-1));
      b.gram(OUTB + ov, OUTB + ov, kBkG1);
      b.launch(bc.red(kD, E_QR1), sm);
    }
    bc.qr_tail(V, QR_POST_BCG, nullptr, sm);   // :95-105
  };
  const CtlH c = run_loop(bc.ss, body, st);
  o.ret = c.ret;
  o.iters = c.hist_len;
  return o;
}

// ------------------------------------------------------- Block BiCGSTAB
template <typename T>
SolveOut blbicgstab(BlockCtx& bc, const DevCsr& A, const T* B, T* X, double tol,
                    int max_iter) {
  constexpr int PR = prec_of<T>();
  bc.unit = PR ? 5.9604644775390625e-08 : 1.1102230246251565e-16;
  cudaStream_t st = bc.st;
  const int s = bc.s;
  const long long rows = bc.np;
  T* R = bc.block<T>(1);
  T* P = bc.block<T>(1);
  T* Rs = bc.block<T>(1);
  T* V = bc.block<T>(1);
  T* Tb = bc.block<T>(1);
  bc.start(max_iter, tol);
  // src/blbicgstab.c:169-175: R = B - A X, P = Rs = R, ||B||_F.
  spmm(A, spmm_args(X, R, s, -1.0, B), bc.red(kD, E_NONE), st);
  {
    Blk b(rows, s, PR);
    const int ir = b.in(R), ib = b.in(B);
    const int op = b.out(P), os = b.out(Rs);
    b.scal(op, ir, cf_const(1)).scal(os, ir, cf_const(1));
    b.dot(ib, ib);
    b.launch(bc.red(kD, E_BBS_INIT), st);
  }
  SolveOut o;
  if (max_iter <= 0) {
    o.ret = tol > 0 ? 0 : kNotConverged;
    return o;
  }
  auto body = [&](cudaStream_t sm) {
    spmm(A, spmm_args(P, V, s), bc.red(kD, E_NONE), sm);    // :181
    {  // :185-189  alpha = (Rs^T V)^-1 Rs^T R
      Blk b(rows, s, PR);
      const int is = b.in(Rs), iv = b.in(V), ir = b.in(R);
      b.gram(is, iv, kBkG1).gram(is, ir, kBkG2);
      b.launch(bc.red(kD, E_BBS_ALPHA), sm);
    }
    {  // :192-193  R -= V alpha
      Blk b(rows, s, PR);
      const int ir = b.in(R), iv = b.in(V);
      const int orr = b.out(R);
      b.scal(orr, ir, cf_const(1)).mat(orr, iv, kBkAlpha, false, cf_const(-1));
      b.launch(bc.red(kD, E_NONE), sm);
    }
    {  // :196-201  T = A R, omega = (T, R) / (T, T)
      SpmmH a = spmm_args(R, Tb, s);
      a.W = reinterpret_cast<const double*>(R);
      a.nd = 2;
      spmm(A, a, bc.red(kD, E_BBS_OMEGA), sm);
    }
    {  // :204-206  X += P alpha + omega R
      Blk b(rows, s, PR);
      const int ix = b.in(X), ip = b.in(P), ir = b.in(R);
      const int ox = b.out(X);
      b.scal(ox, ix, cf_const(1)).mat(ox, ip, kBkAlpha).scal(ox, ir, cf_slot(kOmega1));
      b.launch(bc.red(kD, E_NONE), sm);
    }
    {  // :209-214, :226-229  R -= omega T, beta = -(Rs^T V)^-1 Rs^T T, error
      Blk b(rows, s, PR);
      const int ir = b.in(R), it = b.in(Tb), is = b.in(Rs);
      const int orr = b.out(R);
      b.scal(orr, ir, cf_const(1)).scal(orr, it, cf_slot(kOmega1, -1));
      b.gram(is, it, kBkG1).dot(OUTB + orr, OUTB + orr);
      b.launch(bc.red(kD, E_BBS_BETA), sm);
    }
    {  // :217-221  P = (P - omega V) beta + R; Gram for myqr (:224)
      Blk b(rows, s, PR);
      const int ip = b.in(P), iv = b.in(V), ir = b.in(R);
      const int op = b.out(P);
      b.mat(op, ip, kBkBeta).mat(op, iv, kBkBeta, false, cf_slot(kOmega1, -1))
          .scal(op, ir, cf_const(1));
      b.gram(OUTB + op, OUTB + op, kBkG1);
      b.launch(bc.red(kD, E_QR1), sm);
    }
    bc.qr_tail(P, QR_POST_NONE, nullptr, sm);
  };
  const CtlH c = run_loop(bc.ss, body, st);
  o.ret = c.ret;
  o.iters = c.hist_len;
  return o;
}

// ---------------------------------------------------- Block BiCGSTAB(l)
template <typename T>
SolveOut blbicgstabl(BlockCtx& bc, const DevCsr& A, const T* B, T* X, int l,
                     double tol, int max_iter, double* true_res_out) {
  constexpr int PR = prec_of<T>();
  bc.unit = PR ? 5.9604644775390625e-08 : 1.1102230246251565e-16;
  if (l < 1 || l > kBlMaxL) throw CudaError("blbicgstabl: l out of range");
  cudaStream_t st = bc.st;
  const int s = bc.s;
  const long long rows = bc.np;
  const long long bs = rows * s;   // elements per block
  T* Vb = bc.block<T>(l + 1);
  T* Pb = bc.block<T>(l + 1);
  T* Rb = bc.block<T>(l + 1);
  T* Rs = bc.block<T>(1);
  T* Tm = bc.block<T>(1);
  auto V = [&](int i) { return Vb + i * bs; };
  auto P = [&](int i) { return Pb + i * bs; };
  auto R = [&](int i) { return Rb + i * bs; };
  bc.start(max_iter, tol);
  bc.ss.set_scalar(kL, (double)l, st);
  // src/blbicgstabl.c:83-93: V0 = B + A X (the reference's sign), myqr(V0,
  // xi), P0 = Rs = V0, ||B||_F.
  spmm(A, spmm_args(X, V(0), s, 1.0, B), bc.red(kD, E_NONE), st);
  {
    Blk b(rows, s, PR);
    const int iv = b.in(V(0)), ib = b.in(B);
    b.gram(iv, iv, kBkG1).dot(ib, ib);
    b.launch(bc.red(kD, E_BBL_INIT), st);
  }
  bc.qr_tail(V(0), QR_POST_BBL_INIT, P(0), st);
  {
    Blk b(rows, s, PR);
    const int iv = b.in(V(0));
    const int os = b.out(Rs);
    b.scal(os, iv, cf_const(1));
    b.launch(bc.red(kD, E_NONE), st);
  }
  SolveOut o;
  if (max_iter <= 0) {
    o.ret = tol > 0 ? 0 : kNotConverged;
    return o;
  }
  auto body = [&](cudaStream_t sm) {
    for (int j = 0; j < l; ++j) {
      {  // :102-108  gamma1 = Rs^T V_j, beta
        Blk b(rows, s, PR);
        const int is = b.in(Rs), iv = b.in(V(j));
        b.gram(is, iv, kBkG1);
        b.launch(bc.red(kD, E_BBL_BETA), sm);
      }
      for (int i = 0; i <= j; ++i) {   // :111-116  P_i = P_i beta + V_i
        Blk b(rows, s, PR);
        const int ip = b.in(P(i)), iv = b.in(V(i));
        const int op = b.out(P(i));
        b.mat(op, ip, kBkBeta).scal(op, iv, cf_const(1));
        b.launch(bc.red(kD, E_NONE), sm);
      }
      spmm(A, spmm_args(P(j), P(j + 1), s), bc.red(kD, E_NONE), sm);   // :117
      {  // :121-124  alpha = (Rs^T P_{j+1})^-1 gamma1
        Blk b(rows, s, PR);
        const int is = b.in(Rs), ip = b.in(P(j + 1));
        b.gram(is, ip, kBkG1);
        b.launch(bc.red(kD, E_BBL_ALPHA), sm);
      }
      {  // :129-132  tmp = P_0 alpha, V_0 -= A tmp
        Blk b(rows, s, PR);
        const int ip = b.in(P(0));
        const int ot = b.out(Tm);
        b.mat(ot, ip, kBkAlpha);
        b.launch(bc.red(kD, E_NONE), sm);
      }
      spmm(A, spmm_args(Tm, V(0), s, -1.0, V(0)), bc.red(kD, E_NONE), sm);
      {  // :135  myqr(V_0, t)
        Blk b(rows, s, PR);
        const int iv = b.in(V(0));
        b.gram(iv, iv, kBkG1);
        b.launch(bc.red(kD, E_QR1), sm);
      }
      bc.qr_tail(V(0), QR_POST_BBL_T, nullptr, sm);   // + :142-148
      {  // :138-139  X += tmp xi (xi before the update)
        Blk b(rows, s, PR);
        const int ix = b.in(X), it = b.in(Tm);
        const int ox = b.out(X);
        b.scal(ox, ix, cf_const(1)).mat(ox, it, kBkXiOld);
        b.launch(bc.red(kD, E_NONE), sm);
      }
      for (int i = 1; i <= j; ++i) {   // :151-155  V_i = (V_i - P_{i+1} alpha) t^-1
        Blk b(rows, s, PR);
        const int iv = b.in(V(i)), ip = b.in(P(i + 1));
        const int ov = b.out(V(i));
        b.mat(ov, iv, kBkTinv).mat(ov, ip, kBkATinv, false, cf_const(-1));
        b.launch(bc.red(kD, E_NONE), sm);
      }
      spmm(A, spmm_args(V(j), V(j + 1), s), bc.red(kD, E_NONE), sm);   // :159
    }
    for (int i = 0; i <= l; ++i) {   // :163-166  R_i = V_i xi
      Blk b(rows, s, PR);
      const int iv = b.in(V(i));
      const int orr = b.out(R(i));
      b.mat(orr, iv, kBkXi);
      b.launch(bc.red(kD, E_NONE), sm);
    }
    // MR part, :170-187: modified Gram-Schmidt on R_1..R_l as vectors of
    // n * s entries (Frobenius inner products).
    for (int j = 1; j <= l; ++j) {
      if (j == 1) {
        Lc<T> u(bs);
        const int i1 = u.in(R(1)), i0 = u.in(R(0));
        u.dot(i1, i1).dot(i0, i1);
        u.launch(bc.red(kD, E_BL_SIG, 0, 1), sm);
        continue;
      }
      {
        Lc<T> u(bs);
        const int ij = u.in(R(j)), i1 = u.in(R(1));
        u.dot(ij, i1);
        u.launch(bc.red(kD, E_BL_TAU, 1, (short)j), sm);
      }
      for (int i = 1; i < j; ++i) {
        Lc<T> u(bs);
        const int ij = u.in(R(j)), ii = u.in(R(i));
        const int oj = u.out(R(j));
        u.term(oj, ij, cf_const(1))
            .term(oj, ii, cf_slot((short)(kBlTau + i * l + j), -1));
        if (i + 1 < j) {
          const int in = u.in(R(i + 1));
          u.dot(Lc<T>::OUT + oj, in);
          u.launch(bc.red(kD, E_BL_TAU, (short)(i + 1), (short)j), sm);
        } else {
          const int i0 = u.in(R(0));
          u.dot(Lc<T>::OUT + oj, Lc<T>::OUT + oj)
              .dot(i0, Lc<T>::OUT + oj);
          u.launch(bc.red(kD, E_BL_SIG, 0, (short)j), sm);
        }
      }
    }
    {  // :198-203  tmp = sum omega_i V_{i-1}, P_0 -= sum omega_i P_i
      Lc<T> u(bs);
      int iv[kBlMaxL], ip[kBlMaxL + 1];
      for (int i = 0; i < l; ++i) iv[i] = u.in(V(i));
      for (int i = 0; i <= l; ++i) ip[i] = u.in(P(i));
      const int ot = u.out(Tm), op = u.out(P(0));
      u.term(op, ip[0], cf_const(1));
      for (int i = 1; i <= l; ++i) {
        u.term(ot, iv[i - 1], cf_slot((short)(kBlOmega + i)));
        u.term(op, ip[i], cf_slot((short)(kBlOmega + i), -1));
      }
      u.launch(bc.red(kD, E_NONE), sm);
    }
    spmm(A, spmm_args(Tm, V(0), s, -1.0, V(0)), bc.red(kD, E_NONE), sm);   // :204-205
    {  // :206-212  X += tmp xi, error = ||xi||_F / ||B||_F
      Blk b(rows, s, PR);
      const int ix = b.in(X), it = b.in(Tm);
      const int ox = b.out(X);
      b.scal(ox, ix, cf_const(1)).mat(ox, it, kBkXi);
      b.launch(bc.red(kD, E_BBL_CHECK), sm);
    }
  };
  const CtlH c = run_loop(bc.ss, body, st);
  o.ret = c.ret;
  o.iters = c.hist_len;
  if (true_res_out) {   // :216-218  ||B - A X||_F / ||B||_F
    SolveState t;
    t.create(0, st);
    t.start(0, 1, 0.0, st);
    SpmmH a = spmm_args(X, Tm, s, -1.0, B);
    a.nd = 2;
    a.W = reinterpret_cast<const double*>(Tm);
    spmm(A, a, RedH{bc.bpart, t.ticket, t.S, t.ctl, kD, E_NONE, 0, 0, 0}, st);
    const double rr = t.get_scalar(kD + 1, st);
    *true_res_out = std::sqrt(rr) / bc.ss.get_scalar(kFnb, st);
    t.release(st);
  }
  return o;
}

template SolveOut blcg<double>(BlockCtx&, const DevCsr&, const double*, double*, double, int);
template SolveOut blcg<float>(BlockCtx&, const DevCsr&, const float*, float*, double, int);
template SolveOut blbicgstab<double>(BlockCtx&, const DevCsr&, const double*, double*, double, int);
template SolveOut blbicgstab<float>(BlockCtx&, const DevCsr&, const float*, float*, double, int);
template SolveOut blbicgstabl<double>(BlockCtx&, const DevCsr&, const double*, double*, int,
                                      double, int, double*);
template SolveOut blbicgstabl<float>(BlockCtx&, const DevCsr&, const float*, float*, int,
                                     double, int, double*);

// ------------------------------------------- mixed-precision block solves
// Outer FP64 iterative refinement around FP32 inner block solves (no
// reference counterpart): R = B - A X with the FP64 operator; stop when
// every column's ||r_j|| / ||b_j|| <= target; else solve A E = fl32(R) in
// FP32 (blocks and operator values in FP32; Gram products, dots and the
// s-by-s algebra in FP64) to a relative Frobenius residual inner_tol, and
// X += E in FP64.
BlockMixedOut block_mixed(int method, const DevCsr& A, const double* B,
                          double* X, int n, int s, int l, double target,
                          int max_iter, double inner_tol, SolveState& ss,
                          cudaStream_t st) {
  if (!A.v32) throw CudaError("mixed block solve: FP32 values missing");
  BlockMixedOut out;
  const long long np = pad64(n);
  const long long ne = np * s;
  double* R64 = dalloc_n<double>(ne, st);
  float* R32 = dalloc_n<float>(ne, st);
  float* E32 = dalloc_n<float>(ne, st);
  BK_CHECK(cudaMemsetAsync(R64, 0, sizeof(double) * ne, st));
  std::vector<double> g(s * s), bn(s);
  // Column norms of a block: the diagonal of its Gram matrix.
  auto col_norms = [&](BlockCtx& bc, const double* V, std::vector<double>& nrm) {
    Blk b(np, s, 0);
    const int iv = b.in(V);
    b.gram(iv, iv, kBkG1);
    b.launch(bc.red(kD, E_NONE), st);
    BK_CHECK(cudaMemcpyAsync(g.data(), ss.S + kBkG1, sizeof(double) * s * s,
                             cudaMemcpyDeviceToHost, st));
    BK_CHECK(cudaStreamSynchronize(st));
    for (int j = 0; j < s; ++j) nrm[j] = std::sqrt(g[j * s + j]);
  };
  int used = 0;
  double prev = 0.0;
  std::vector<double> rn(s);
  for (int sweep = 0;; ++sweep) {
    {
      BlockCtx bc(n, s, ss, st);
      bc.start(1, 0.0);
      if (sweep == 0) col_norms(bc, B, bn);
      spmm(A, spmm_args<double>(X, R64, s, -1.0, B), bc.red(kD, E_NONE), st);
      col_norms(bc, R64, rn);
      bc.release();
    }
    double worst = 0.0;
    for (int j = 0; j < s; ++j) {
      const double q = bn[j] > 0 ? rn[j] / bn[j] : rn[j];
      worst = std::isfinite(q) ? std::max(worst, q) : q;   // a NaN column wins
      if (!std::isfinite(worst)) break;
    }
    out.true_res = worst;
    if (!std::isfinite(worst)) {
      out.ret = kDivergence;
      break;
    }
    if (worst <= target) {
      out.ret = used > 0 ? used - 1 : 0;
      break;
    }
    if (used >= max_iter || (sweep > 0 && worst > 0.5 * prev)) {
      out.ret = kNotConverged;   // budget spent, or refinement stagnates
      break;
    }
    prev = worst;
    launch_convert_d2f(R64, R32, ne, st);
    BK_CHECK(cudaMemsetAsync(E32, 0, sizeof(float) * ne, st));
    SolveOut o;
    {
      BlockCtx bc(n, s, ss, st);
      const int budget = max_iter - used;
      if (method == 0)
        o = blcg<float>(bc, A, R32, E32, inner_tol, budget);
      else
        o = blbicgstabl<float>(bc, A, R32, E32, l, inner_tol, budget, nullptr);
      bc.release();
    }
    used += o.ret >= 0 ? o.ret + 1 : o.iters;
    out.inner_iters = used;
    ++out.sweeps;
    if (o.ret == kDivergence) {
      // The FP32 inner solve broke down (Krylov blocks whose conditioning
      // FP32 cannot represent): this sweep's correction in FP64 instead.
      double* E64 = dalloc_n<double>(ne, st);
      BK_CHECK(cudaMemsetAsync(E64, 0, sizeof(double) * ne, st));
      SolveOut o64;
      {
        BlockCtx bc(n, s, ss, st);
        const int budget = max_iter - used;
        if (method == 0)
          o64 = blcg<double>(bc, A, R64, E64, inner_tol, budget);
        else
          o64 = blbicgstabl<double>(bc, A, R64, E64, l, inner_tol, budget, nullptr);
        bc.release();
      }
      used += o64.ret >= 0 ? o64.ret + 1 : o64.iters;
      out.inner_iters = used;
      ++out.fp64_sweeps;
      if (o64.ret == kDivergence) {
        dfree(E64, st);
        out.ret = kDivergence;
        break;
      }
      Lc<double> u(ne);
      const int ix = u.in(X), ie = u.in(E64);
      const int ox = u.out(X);
      u.term(ox, ix, cf_const(1)).term(ox, ie, cf_const(1));
      u.launch(ss.red_after(kD, E_NONE), st);
      dfree(E64, st);
      continue;
    }
    launch_mx_accum(X, E32, E32, ne, ss.red_after(kD, E_NONE), st);
    BK_CHECK(cudaGetLastError());
  }
  dfree(R64, st);
  dfree(R32, st);
  dfree(E32, st);
  return out;
}

// ------------------------------------------------------------------ QR
void thin_qr(BlockCtx& bc, double* V) {
  cudaStream_t st = bc.st;
  bc.start(1, 0.0);
  Blk b(bc.np, bc.s);
  const int iv = b.in(V);
  b.gram(iv, iv, kBkG1);
  b.launch(bc.red(kD, E_QR1), st);
  bc.qr_tail(V, QR_POST_NONE, nullptr, st);
}

}  // namespace bk
