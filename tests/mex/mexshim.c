/* A minimal stand-in for the MATLAB runtime behind tests/mex/mex.h, so the
 * reference's MEX front-ends (matlab/*.c, compiled where they lie by
 * tests/mex/Makefile and linked against libbksp.so) can be called from
 * the tests.  TEST INFRASTRUCTURE ONLY.
 *
 * Arrays are column-major doubles with separate real and imaginary parts;
 * sparse arrays are compressed-column (jc: n + 1 column starts, ir: row
 * indices), as MATLAB stores them.  mexErrMsgIdAndTxt returns to the
 * enclosing shim_call through longjmp.  Arrays are never freed (a test
 * process makes a handful). */
#include <setjmp.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  size_t m, n;
  int sparse;
  double *pr, *pi;
  mwIndex *ir, *jc;
};

static jmp_buf g_err_jmp;
static int g_in_call = 0;
static char g_err_msg[512];

static mxArray *new_array(size_t m, size_t n) {
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  a->m = m;
  a->n = n;
  return a;
}

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
  mxArray *a = new_array(m, n);
  const size_t cnt = m * n > 0 ? m * n : 1;
  a->pr = (double *)calloc(cnt, sizeof(double));
  if (flag == mxCOMPLEX) a->pi = (double *)calloc(cnt, sizeof(double));
  return a;
}

double *mxGetPr(const mxArray *a) { return a->pr; }
double *mxGetPi(const mxArray *a) { return a->pi; }
void mxSetPr(mxArray *a, double *pr) { a->pr = pr; }
void mxSetPi(mxArray *a, double *pi) { a->pi = pi; }
size_t mxGetM(const mxArray *a) { return a->m; }
size_t mxGetN(const mxArray *a) { return a->n; }
void mxSetM(mxArray *a, mwSize m) { a->m = m; }
void mxSetN(mxArray *a, mwSize n) { a->n = n; }
mwIndex *mxGetIr(const mxArray *a) { return a->ir; }
mwIndex *mxGetJc(const mxArray *a) { return a->jc; }
bool mxIsSparse(const mxArray *a) { return a->sparse != 0; }
bool mxIsComplex(const mxArray *a) { return a->pi != NULL; }

/* The only callback the front-ends make: "transpose" of a sparse matrix
 * (plain transpose, no conjugation: MATLAB's transpose / .'). */
int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[],
                  const char *name) {
  if (nlhs != 1 || nrhs != 1 || strcmp(name, "transpose") != 0 ||
      !prhs[0]->sparse)
    mexErrMsgIdAndTxt("shim:call", "unsupported mexCallMATLAB(%s)", name);
  const mxArray *a = prhs[0];
  const size_t nnz = a->jc[a->n];
  mxArray *t = new_array(a->n, a->m);
  t->sparse = 1;
  t->jc = (mwIndex *)calloc(a->m + 1, sizeof(mwIndex));
  t->ir = (mwIndex *)calloc(nnz > 0 ? nnz : 1, sizeof(mwIndex));
  t->pr = (double *)calloc(nnz > 0 ? nnz : 1, sizeof(double));
  if (a->pi) t->pi = (double *)calloc(nnz > 0 ? nnz : 1, sizeof(double));
  for (size_t k = 0; k < nnz; ++k) t->jc[a->ir[k] + 1]++;
  for (size_t i = 0; i < a->m; ++i) t->jc[i + 1] += t->jc[i];
  mwIndex *pos = (mwIndex *)malloc(sizeof(mwIndex) * (a->m + 1));
  memcpy(pos, t->jc, sizeof(mwIndex) * (a->m + 1));
  for (size_t j = 0; j < a->n; ++j)
    for (mwIndex k = a->jc[j]; k < a->jc[j + 1]; ++k) {
      const mwIndex p = pos[a->ir[k]]++;
      t->ir[p] = j;
      t->pr[p] = a->pr[k];
      if (a->pi) t->pi[p] = a->pi[k];
    }
  free(pos);
  plhs[0] = t;
  return 0;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int k = snprintf(g_err_msg, sizeof(g_err_msg), "%s: ", id);
  if (k < 0) k = 0;
  vsnprintf(g_err_msg + k, sizeof(g_err_msg) - (size_t)k, fmt, ap);
  va_end(ap);
  if (g_in_call) longjmp(g_err_jmp, 1);
  abort();
}

/* ---- test-side entry points (ctypes) ---- */

mxArray *shim_dense(size_t m, size_t n, const double *re, const double *im) {
  mxArray *a = mxCreateDoubleMatrix(m, n, im ? mxCOMPLEX : mxREAL);
  if (re) memcpy(a->pr, re, sizeof(double) * m * n);
  if (im) memcpy(a->pi, im, sizeof(double) * m * n);
  return a;
}

mxArray *shim_sparse(size_t m, size_t n, const mwIndex *jc, const mwIndex *ir,
                     const double *re, const double *im) {
  const size_t nnz = jc[n];
  mxArray *a = new_array(m, n);
  a->sparse = 1;
  a->jc = (mwIndex *)malloc(sizeof(mwIndex) * (n + 1));
  a->ir = (mwIndex *)malloc(sizeof(mwIndex) * (nnz > 0 ? nnz : 1));
  a->pr = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
  memcpy(a->jc, jc, sizeof(mwIndex) * (n + 1));
  memcpy(a->ir, ir, sizeof(mwIndex) * nnz);
  memcpy(a->pr, re, sizeof(double) * nnz);
  if (im) {
    a->pi = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    memcpy(a->pi, im, sizeof(double) * nnz);
  }
  return a;
}

typedef void (*mex_fn)(int, mxArray *[], int, const mxArray *[]);

/* Calls a front-end's mexFunction; 0, or 1 after mexErrMsgIdAndTxt (the
 * message then in shim_error()). */
int shim_call(mex_fn fn, int nlhs, mxArray *plhs[], int nrhs,
              const mxArray *prhs[]) {
  g_err_msg[0] = 0;
  g_in_call = 1;
  if (setjmp(g_err_jmp)) {
    g_in_call = 0;
    return 1;
  }
  fn(nlhs, plhs, nrhs, prhs);
  g_in_call = 0;
  return 0;
}

const char *shim_error(void) { return g_err_msg; }
