/* The subset of MATLAB's documented C MEX API (matrix.h / mex.h) that the
 * reference's MATLAB front-ends (matlab/*.c) use, for compiling and running
 * them without MATLAB.  TEST INFRASTRUCTURE: implemented by mexshim.c, which
 * stands in for the MATLAB runtime (dense and sparse double arrays with
 * separate real / imaginary parts, the "transpose" callback, errors that
 * return to the caller).  64-bit indices as under -largeArrayDims. */
#ifndef BKSP_TEST_MEX_H
#define BKSP_TEST_MEX_H

#include <stdbool.h>
#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
double *mxGetPr(const mxArray *a);
double *mxGetPi(const mxArray *a);
void mxSetPr(mxArray *a, double *pr);
void mxSetPi(mxArray *a, double *pi);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
void mxSetM(mxArray *a, mwSize m);
void mxSetN(mxArray *a, mwSize n);
mwIndex *mxGetIr(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
bool mxIsSparse(const mxArray *a);
bool mxIsComplex(const mxArray *a);

int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[],
                  const char *name);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif /* BKSP_TEST_MEX_H */
