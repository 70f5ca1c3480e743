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
    long long launches;  /* out: GPU kernel launches the call issued        */
    int inner_iters;     /* out: mixed solves: inner iterations, all sweeps */
    int sweeps;          /* out: mixed solves: refinement sweeps            */
    long long alg_bytes; /* out (bksp_gpu_solve, mixed solves): algorithmic
                          * DRAM bytes of the solve's kernels (SpMV in the
                          * stored format, linear combinations, Gram,
                          * precision conversions, preconditioner build),
                          * each operand once per launch                   */
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

/* The block product with host arrays: C = beta C + alpha A B, B and C
 * column-major n x s (s <= 16), trans 'n' (A as stored; the reference's
 * dcsrgemm1 / mkl_dcsrmm) or 's' (the mirrored one-triangle operator,
 * dcsrsymm1).  Runs the block methods' SpMM kernel: diagonal form with
 * 16-byte row segments for stencil operators, CSR otherwise; entries in
 * ascending column order, y += (alpha a_k) x_k, then C added.  Returns 0 or
 * INVALID_PARAMETERS. */
int bksp_gpu_dcsrmm(dspmat *A, char trans, int s, double alpha,
                    const double *B, double beta, double *C);

/* The complex product with host arrays (the reference's zcsrgemm0,
 * src/matvec.c:55-98): y = A x (trans 'n') or y = A^H x ('t', the
 * reference's 't' conjugates).  Each row is summed left to right from zero
 * with the C99 complex multiply and no fused multiply-add, so the result is
 * bit-identical to zcsrgemm0.  Returns 0 or INVALID_PARAMETERS. */
int bksp_gpu_zcsrmv(zspmat *A, char trans, const double _Complex *x,
                    double _Complex *y);

/* ------------------------------------------------ device-resident solves */

typedef struct bksp_gpu_matrix bksp_gpu_matrix;

#define BKSP_GPU_MIRROR 1      /* A holds one triangle: mirror it            */
#define BKSP_GPU_FP32 2        /* also keep FP32 values (mixed precision)    */
#define BKSP_GPU_TRANSPOSE 4   /* also build A^T (BiCG)                      */

/* Upload A (host arrays) once; the handle keeps it in GPU memory. */
int bksp_gpu_matrix_create(dspmat *A, int flags, bksp_gpu_matrix **out);
int bksp_gpu_matrix_destroy(bksp_gpu_matrix *A);
int bksp_gpu_matrix_info(const bksp_gpu_matrix *A, int *n, int *nnz);

enum {
    BKSP_GPU_CG = 1,
    BKSP_GPU_CR = 2,
    BKSP_GPU_BICG = 3,
    BKSP_GPU_BICGSTAB = 4,
    BKSP_GPU_BICGSTABL = 5,
    /* BiCGSTAB(l) whose minimal-residual step is computed from one pass
     * over r_0..r_l (their Gram matrix, LDL^T on the device) instead of
     * the reference's modified Gram-Schmidt sweeps: the same recurrence in
     * exact arithmetic, fewer passes over memory. */
    BKSP_GPU_BICGSTABL_FAST = 6
};

/* The bksp.h methods on device-resident data: b and x are device pointers
 * to n doubles (x in/out); the work is ordered on `stream` (a cudaStream_t,
 * NULL for the library's stream) and complete when the call returns.
 * Returns the bksp code.  stats may be NULL. */
int bksp_gpu_solve(bksp_gpu_matrix *A, int method, int l, const double *b,
                   double *x, double tol, int max_iter, void *stream,
                   bksp_gpu_stats *stats);

/* SpMV kernel variant of the operator: 0 tile, 1 tile with TMA bulk
 * copies, 2..5 vector CSR with 4, 8, 16, 32 lanes per row, 6 warp tile
 * (each warp streams and sums its own 32 rows), 7 diagonal form (operators
 * without one, and calls whose result / operand vectors are not 16-byte
 * aligned, run the tile kernel), 8 sliced ELL (32-row slices, one lane per
 * row; built at upload for operators of >= 65,536 rows without a diagonal
 * form whose padding stays under half the entries; others run the tile
 * kernel).  variant < 0 queries, otherwise sets.
 * Returns the variant set.  The library picks one by timing all of them
 * when it uploads an operator of >= 65,536 rows (below that: the diagonal
 * form when there is one, else by mean row length). */
int bksp_gpu_matrix_variant(bksp_gpu_matrix *A, int variant);

/* A Matrix Market file (coordinate real / integer / pattern, general or
 * symmetric, square) straight into a device-resident operator: the text is
 * parsed on the host by several threads; sorting the entries into rows --
 * file order within a row, as read_matrix_market (and the reference's
 * reader, src/read_matrix.c) leaves them -- and, with BKSP_GPU_MIRROR and a
 * symmetric file, mirroring the stored triangle (rows then in ascending
 * column order, as bksp_gpu_matrix_create builds them) run on the GPU.
 * Flags: BKSP_GPU_FP32, BKSP_GPU_MIRROR (BKSP_GPU_TRANSPOSE is not
 * accepted).  Returns 0 or INVALID_PARAMETERS (unreadable or malformed file,
 * non-square matrix). */
int bksp_gpu_read_matrix_market(const char *path, int flags,
                                bksp_gpu_matrix **out);

/* Copy the operator's CSR (n + 1 row pointers, nnz columns and FP64 values,
 * as stored on the device; any pointer may be NULL) to host arrays. */
int bksp_gpu_matrix_csr(const bksp_gpu_matrix *A, int *rowptr, int *col,
                        double *val);

/* Diagonal form of the operator: an operator whose stored entries lie on at
 * most 8 diagonals, whose rows list their columns in strictly ascending
 * order, and whose diagonal storage is smaller than its CSR storage, is
 * also kept diagonal by diagonal.  Returns the number of diagonals (0: no
 * diagonal form) and writes their column offsets j - i, ascending, to
 * offsets (8 ints, or NULL). */
int bksp_gpu_matrix_diagonals(const bksp_gpu_matrix *A, int *offsets);

/* y = A x on the device, FP64 (fp32 = 0) or FP32 vectors and values
 * (fp32 = 1, needs BKSP_GPU_FP32); x and y hold n elements.  Asynchronous
 * on `stream`.  For kernel timing. */
int bksp_gpu_spmv(bksp_gpu_matrix *A, int fp32, const void *x, void *y,
                  void *stream);

/* Y = A X for row-major device blocks of n x s (s <= 16), FP64 (fp32 = 0)
 * or FP32 (fp32 = 1, needs BKSP_GPU_FP32): the block methods' product.
 * kernel: -1 the autotuned choice, 0 the diagonal form (operators that
 * have one, s a multiple of the 16-byte vector), 1 CSR.  Asynchronous on
 * `stream`.  For kernel timing. */
int bksp_gpu_spmm(bksp_gpu_matrix *A, int fp32, int s, int kernel,
                  const void *X, void *Y, void *stream);

/* FP64 ||b - A x||_2 / ||b||_2 of device vectors (synchronous). */
double bksp_gpu_true_residual(bksp_gpu_matrix *A, const double *b,
                              const double *x, void *stream);

/* ------------------------------------- mixed precision, preconditioners */

#define BKSP_GPU_PRECOND_NONE 0      /* unpreconditioned                     */
#define BKSP_GPU_PRECOND_JACOBI 1    /* M = diag(A)^-1                       */
#define BKSP_GPU_PRECOND_LEARNED 2   /* M = MLP-predicted SPAI on A's pattern */

/* A trained per-row MLP predicting sparse-approximate-inverse values. */
typedef struct bksp_gpu_spai_model bksp_gpu_spai_model;

typedef struct {
    int l;                      /* BiCGSTAB(l) degree (1..8)                 */
    double target;              /* FP64 true relative residual to reach      */
    int max_iter;               /* outer-iteration budget                    */
    int precond;                /* BKSP_GPU_PRECOND_*                        */
    bksp_gpu_spai_model *model; /* for BKSP_GPU_PRECOND_LEARNED              */
    double delta;               /* replacement trigger (0: 1e-3)             */
    int period;                 /* replacement period, outer its (0: 6)      */
    int fallback;               /* 1: retry with Jacobi when the learned
                                   preconditioner stagnates or breaks down   */
} bksp_gpu_mixed_opts;

/* The learned preconditioner: a per-row MLP (8 -> 64 -> 64 -> 8, FP32)
 * maps a row's normalised stencil (its entries on up to 8 diagonals, a_ij /
 * a_ii) to the sparse-approximate-inverse values of that row on A's
 * pattern.  Trained on the GPU by minimising ||(I - M A) Z||_F^2 over random
 * probe blocks Z.  An untrained model is Jacobi.  Operators qualify when
 * created with BKSP_GPU_FP32 and having the diagonal plus at most 3 lower
 * and 4 upper diagonals in use (stencil matrices). */
int bksp_gpu_spai_create(unsigned seed, bksp_gpu_spai_model **out);
int bksp_gpu_spai_destroy(bksp_gpu_spai_model *model);
int bksp_gpu_spai_nparams(void);
/* Copy the parameters out (set = 0) or in (set = 1); nparams floats. */
int bksp_gpu_spai_params(bksp_gpu_spai_model *model, float *host, int set);
/* Adam training over the rows of nsys operators, `probes` Rademacher probe
 * vectors per operator and epoch; *loss_out gets the last epoch's mean
 * loss. */
int bksp_gpu_spai_train(bksp_gpu_spai_model *model,
                        bksp_gpu_matrix *const *systems, int nsys, int epochs,
                        int probes, float lr, unsigned seed, double *loss_out);
/* Loss and gradient for a given probe block (probes x n column-major host
 * floats, or NULL for seeded Rademacher probes); operators of at most
 * 65,536 rows.  grad: nparams floats or NULL. */
int bksp_gpu_spai_loss_grad(bksp_gpu_spai_model *model, bksp_gpu_matrix *A,
                            const float *Z, int probes, unsigned seed,
                            double *loss, float *grad);
/* Checkpoint file: a one-line JSON header then little-endian FP32 params. */
int bksp_gpu_spai_save(bksp_gpu_spai_model *model, const char *path);
int bksp_gpu_spai_load(const char *path, bksp_gpu_spai_model **out);

/* Right-preconditioned BiCGSTAB(l) in mixed precision: FP32 matrix values
 * and Krylov vectors, FP64 dot products, scalars and solution, FP64
 * residual replacement, stopping on the FP64 true relative residual
 * ||b - A x|| / ||b|| <= target.  The matrix needs BKSP_GPU_FP32.  Device
 * vectors b, x (x in/out).  Returns the index of the converging outer
 * iteration, NOT_CONVERGED, DIVERGENCE or INVALID_PARAMETERS. */
int bksp_gpu_solve_mixed(bksp_gpu_matrix *A, const double *b, double *x,
                         const bksp_gpu_mixed_opts *opts, void *stream,
                         bksp_gpu_stats *stats);

/* The same with host arrays in the bksp.h style: uploads A, b, x, solves,
 * downloads x. */
int bksp_dbicgstabl_mixed(dspmat *A, double *b, const bksp_gpu_mixed_opts *opts,
                          double *x);

/* Preconditioned CG in mixed precision, the same split as
 * bksp_gpu_solve_mixed: FP32 values of A and M and FP32 vectors (r, z = M r,
 * p, A p, the correction), FP64 dot products, scalars and solution, FP64
 * reliable replacement of r by b - A x, stopping on the FP64 true relative
 * residual.  A symmetric positive definite, full storage (BKSP_GPU_MIRROR
 * for one triangle) with BKSP_GPU_FP32.  The preconditioner is symmetric:
 * Jacobi, or the learned one symmetrised, (M + M^T) / 2.  opts->l is not
 * used.  Returns the index of the converging iteration, NOT_CONVERGED,
 * DIVERGENCE or INVALID_PARAMETERS. */
int bksp_gpu_cg_mixed(bksp_gpu_matrix *A, const double *b, double *x,
                      const bksp_gpu_mixed_opts *opts, void *stream,
                      bksp_gpu_stats *stats);

/* The same with host arrays, taking bksp_dcg's matrix: type "symmetric",
 * one triangle stored (INVALID_MATRIX_TYPE otherwise). */
int bksp_dcg_mixed(dspmat *A, double *b, const bksp_gpu_mixed_opts *opts,
                   double *x);

/* Block CG and Block BiCGSTAB(l) (l = opts->l) in mixed precision, with
 * dblcg's / dblbicgstabl's host arrays: an outer FP64 iterative refinement
 * (R = B - A X with the FP64 operator) around inner solves of the same
 * method in FP32 (blocks and operator values; Gram products, dots and the
 * s-by-s factorisations in FP64), each to a relative Frobenius residual of
 * opts->delta (0: 1e-4); stops when every column's FP64 true relative
 * residual ||b_j - A x_j|| / ||b_j|| is <= opts->target.  opts->precond and
 * opts->model are not used.  Returns the total inner iterations minus one
 * at convergence, NOT_CONVERGED (budget opts->max_iter spent, or the
 * refinement stagnates), DIVERGENCE, INVALID_MATRIX_TYPE (Block CG with a
 * non-"symmetric" matrix) or INVALID_PARAMETERS. */
int bksp_dblcg_mixed(dspmat *A, dmat *B, const bksp_gpu_mixed_opts *opts,
                     dmat *X);
int bksp_dblbicgstabl_mixed(dspmat *A, dmat *B, const bksp_gpu_mixed_opts *opts,
                            dmat *X);

/* Shifted BiCGSTAB(l) (l = opts->l) in mixed precision, with dshbicgstabl's
 * host arrays (x: n * (sigma_size + 1) values, seed first, shifted parts
 * zero on entry): the shifted solve stores the per-shift direction vectors
 * p_k -- its bulk traffic -- in FP32 (seed vectors, x_k and every scalar in
 * FP64) and runs to the seed tolerance opts->target; then each system
 * (A + sigma_k I) x_k = b, and the seed, whose FP64 true relative residual
 * is above opts->target is polished from its x_k by the mixed-precision
 * BiCGSTAB(l) on the shifted operator, so every solution ends at the FP64
 * target.  (A shift-invariant Krylov space excludes a preconditioner:
 * opts->precond and opts->model are not used.)  Returns the seed's
 * converging iteration, NOT_CONVERGED (a solve or polish missed the
 * target), DIVERGENCE or INVALID_PARAMETERS. */
int bksp_dshbicgstabl_mixed(dspmat *A, double *b, double *sigma, int sigma_size,
                            const bksp_gpu_mixed_opts *opts, double *x);

/* ------------------------------------------------------------ batches */

/* Many independent systems in one call, each solved as bksp_gpu_solve_mixed
 * / bksp_gpu_solve would solve it.
 *   workers >= 0: that many host threads (0: 8; at most count), each with
 *     its own stream, solve the systems in turn, one CUDA-graph loop per
 *     system.
 *   workers < 0: one persistent launch.  Each system's set-up (initial
 *     residual, preconditioner values) runs on a host thread of its own;
 *     then a single cooperative kernel iterates every system in lockstep,
 *     operation by operation, with a per-system convergence mask: a
 *     converged system drops out, the others continue, and each phase's
 *     work is spread over the whole GPU.  Grid barriers are bounded: a
 *     wait that runs out ends the launch and the call returns
 *     INVALID_PARAMETERS (bksp_gpu_persist_status reports it).  Up to
 *     512 systems; a system whose method has no persistent form (block
 *     and shifted methods, Gram steps of more than five vectors) runs as
 *     its own CUDA-graph loop.  On the benchmark batch (64 systems of
 *     32^3..96^3 rows) this mode is about four times slower than the
 *     graph loops: one CTA of eight warps per SM keeps too few loads in
 *     flight for the streaming phases.
 * A[i], b[i], x[i]: system i's operator and device vectors (x in/out); they
 * must be ready when the call is made, and every x[i] holds its result when
 * it returns.  stats: NULL or count entries (stats[i].ret = system i's
 * return code).  Returns 0 when every system converged, NOT_CONVERGED when
 * at least one did not (or diverged), INVALID_PARAMETERS on bad arguments
 * or a failed system. */
int bksp_gpu_solve_mixed_batch(bksp_gpu_matrix *const *A, const double *const *b,
                               double *const *x, int count,
                               const bksp_gpu_mixed_opts *opts, int workers,
                               bksp_gpu_stats *stats);
int bksp_gpu_solve_batch(bksp_gpu_matrix *const *A, int method, int l,
                         const double *const *b, double *const *x, int count,
                         double tol, int max_iter, int workers,
                         bksp_gpu_stats *stats);

/* Iteration loop of the calling thread's subsequent single-system solves:
 * 0 a CUDA-graph while loop (default), 1 a persistent launch (the batch
 * path's kernel with one system: one launch per solve, a grid barrier per
 * operation; pays off for small systems, where a graph's per-kernel cost
 * dominates).  Other values only query.  Returns the previous mode.  The
 * BKSP_GPU_LOOP=persist environment variable sets 1 as the default. */
int bksp_gpu_loop_mode(int mode);

/* Status of the calling thread's last persistent batch: 0 ok, 1 a grid
 * barrier wait ran out of polls, 2 the launch failed; *grid (may be NULL)
 * receives the CTAs it launched. */
int bksp_gpu_persist_status(int *grid);

/* Test hook for the persistent batch's bounded waits (calling thread's
 * subsequent batches): polls per barrier wait before giving up (0: the
 * default, or BKSP_GPU_SPIN_LIMIT), and a CTA that never arrives at a
 * barrier (-1: none), which makes the others' waits run out. */
void bksp_gpu_persist_debug(long long spin_limit, int absent_cta);

/* The FP64 relative true residual of bksp_gpu_true_residual, computed
 * without allocating any memory, for callers that cannot allocate device
 * memory where they need it (a host application whose memory pool already
 * owns the GPU's memory; latency-critical loops that cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree).  No counterpart in
 * the reference.  Its scratch is a static device array of about 8 MiB that
 * every GPU loading the library holds until exit; operators with more than
 * 1,048,576 rows are rejected with INVALID_PARAMETERS and a message on
 * stderr.  The first call on each device looks up that array's device
 * address (make it before any stream capture).  All calls on a device share
 * the array: calls whose GPU work overlaps race and must be serialised by
 * the caller.  The operator's device must be the current device (else
 * INVALID_PARAMETERS).  b, x: device pointers to n doubles; *res receives
 * the residual; returns 0 or INVALID_PARAMETERS; synchronous on `stream`
 * (NULL: library stream).
 */
int bksp_gpu_true_residual_noalloc(bksp_gpu_matrix *A, const double *b,
                                   const double *x, void *stream,
                                   double *res);

#ifdef __cplusplus
}
#endif

#endif /* BKSP_GPU_H */
