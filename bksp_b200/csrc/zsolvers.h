// Host drivers of the complex methods (reference zbicg, zbicgstabl,
// zblbicgstabl, zshbicgstabl) and their operator upload.  Vectors are
// device double2 arrays padded to pad64(n); blocks are row-major n-by-s.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "runtime.h"
#include "solvers.h"
#include "zkernel_api.h"

namespace bk {

// Device complex CSR: col and val padded to a multiple of 4 entries (pad:
// column 0, value 0), row blocks of the tile kernel.
struct ZDevCsr {
  int n = 0, nnz = 0, nrb = 0;
  int* rowptr = nullptr;
  int* col = nullptr;
  double2* val = nullptr;
  int* rb = nullptr;
  // Sliced-ELL copy (kernel_api.h: SellH); nslice = 0: none.
  int nslice = 0;
  int* sptr = nullptr;
  int* scol = nullptr;
  double2* sval = nullptr;
  CsrH h() const {
    CsrH c{};
    c.rowptr = rowptr;
    c.col = col;
    c.val = val;
    c.rb = rb;
    c.n = n;
    c.nrb = nrb;
    c.nnz = nnz;
    c.sell = SellH{sptr, scol, sval, nslice};
    return c;
  }
  void release(cudaStream_t st);
};

// Upload a complex CSR whose values are interleaved (re, im) doubles; with
// conj_transpose the operator uploaded is A^H, each row's entries ordered by
// the original row index (the summation order of the reference's 't'
// scatter, src/matvec.c:74-90).  Throws CudaError on a bad structure.
void upload_zcsr(int n, const int* rowptr, const int* col, const double* val,
                 bool conj_transpose, ZDevCsr& out, cudaStream_t st);

// Builder of one complex linear-combination launch (ZLcH).
struct ZLc {
  ZLcH d;
  explicit ZLc(long long n);
  static constexpr int OUT = 100;
  int in(const double2* p, bool rep = false);
  int out(double2* p, bool rep = false);
  ZLc& term(int o, int i, ZCfH c);
  ZLc& dot(int a, int b, bool conj = true);   // zdotc(a, b) = sum conj(a) b
  ZLc& batch(int reps, long long stride);
  void launch(const RedH& rd, cudaStream_t st);
};

SolveOut zbicg(const ZDevCsr& A, const ZDevCsr& AH, const double2* b,
               double2* x, double tol, int max_iter, SolveState& ss,
               cudaStream_t st);
SolveOut zbicgstabl(const ZDevCsr& A, const double2* b, int l, double2* x,
                    double tol, int max_iter, SolveState& ss, cudaStream_t st);
// x: (ns + 1) vectors of pad64(n): the seed's, then each shift's.
SolveOut zshbicgstabl(const ZDevCsr& A, const double2* b, int l,
                      const double* sigma, int ns, double2* x, double tol,
                      int max_iter, SolveState& ss, cudaStream_t st);
// B, X: row-major pad64(n)-by-s blocks.  true_res: ||B - A X||_F / ||B||_F.
SolveOut zblbicgstabl(const ZDevCsr& A, const double2* B, int s, int l,
                      double2* X, double tol, int max_iter, SolveState& ss,
                      cudaStream_t st, double* true_res);
// Thin QR of the row-major n-by-s block V in place (V <- Q) by shifted
// complex Cholesky-QR3; R (s-by-s, row-major pairs) to the host.  False on
// a breakdown.
bool zthin_qr(int n, int s, double2* V, double* R_host, SolveState& ss,
              cudaStream_t st);

}  // namespace bk
