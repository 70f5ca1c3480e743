/*
 * bksp_gpu.h -- extensions of the bksp C API specific to this B200 build.
 *
 * Everything here is additive: bksp.h programs need none of it.  It offers
 *   - per-thread statistics of the bksp.h calls (iteration history, device
 *     time), used by the parity tests to compare residual histories;
 *   - device-resident operators and solves (inputs already in GPU memory),
 *     used to time the iteration without host transfers;
 *   - the mixed-precision / learned-preconditioner solve.
 * None of these entry points has a counterpart in the reference.
 */
#ifndef BKSP_GPU_H
#define BKSP_GPU_H

#include "bksp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ statistics */

typedef struct {
    double *hist;        /* in: host array for the convergence-test values  */
    int hist_cap;        /* in: its capacity (0: no history)                */
    int hist_len;        /* out: convergence tests performed                */
    int ret;             /* out: the call's return code                     */
    double solve_ms;     /* out: device time of the solve (CUDA events)     */
    double total_ms;     /* out: wall time of the call incl. transfers      */
    double true_res;     /* out: FP64 ||b - A x|| / ||b|| where computed    */
} bksp_gpu_stats;

/* Route statistics of this thread's subsequent bksp calls into *s (NULL
 * turns recording off).  The caller keeps *s alive while recording. */
void bksp_gpu_record(bksp_gpu_stats *s);

/* Version / build string, for logs. */
const char *bksp_gpu_version(void);

/* Number of CUDA devices visible (0 when none). */
int bksp_gpu_device_count(void);

/* One sparse product on the GPU with host arrays: y = A x for trans 'n',
 * y = A^T x for 't' (the stored entries of A, as the reference's
 * mkl_cspblas_dcsrgemv / dcsrgemm0 compute them), or the mirrored operator
 * of a one-triangle "symmetric" matrix for 's' (mkl_cspblas_dcsrsymv /
 * dcsrsymm0).  Returns 0 or INVALID_PARAMETERS.  For 'n' the FP64 result is
 * bit-identical to the reference's dcsrgemm0 (same summation order, no
 * fused multiply-add). */
int bksp_gpu_dcsrmv(dspmat *A, char trans, const double *x, double *y);

#ifdef __cplusplus
}
#endif

#endif /* BKSP_GPU_H */
