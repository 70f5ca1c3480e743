/*
 * bksp.h -- Krylov subspace solvers for sparse linear systems, executed on an
 * NVIDIA B200 (sm_100a).
 *
 * Drop-in replacement for the C API of aldente39/bksp (include/bksp.h of
 * that project).  Every type and entry point below keeps the reference's
 * name, argument order, argument meaning, memory layout and return
 * convention, so a program written against the reference compiles and links
 * against libbksp.so from this project unchanged:
 *
 *   - dspmat: 0-based CSR with POINTER-to-int size fields (reference
 *     include/bksp.h:12-21).  type == "symmetric" means only one triangle is
 *     stored and the other is implied (reference src/matvec.c:100-127).
 *   - dmat: column-major dense block, value[j * row_size + i]
 *     (reference include/bksp.h:23-27).
 *   - All arrays are host memory owned by the caller.  x / X are in/out:
 *     read as the initial guess, overwritten with the solution.
 *   - Return value: >= 0 is the 0-based index of the iteration whose
 *     convergence test passed; NOT_CONVERGED when max_iter iterations did
 *     not reach tol; INVALID_MATRIX_TYPE when a symmetric-only method gets a
 *     matrix whose type is not "symmetric"; INVALID_PARAMETERS for bad
 *     arguments or a CUDA failure; DIVERGENCE when the iteration broke down
 *     (a NaN/Inf scalar).  (The reference defines but never returns the last
 *     two codes.)
 *
 * Differences from the reference header, none of which changes the ABI:
 * an include guard, extern "C" for C++ callers, and error-code macros
 * without the stray trailing semicolons of the reference (so that
 * `code == NOT_CONVERGED` compiles).
 */
#ifndef BKSP_H
#define BKSP_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */

#define NOT_CONVERGED (-1)
#define DIVERGENCE (-2)
#define INVALID_PARAMETERS (-3)
#define INVALID_MATRIX_TYPE (-4)

/* --------------------------------------------------------------- structs */

/* Sparse matrix, 0-based CSR (reference include/bksp.h:12-21). */
typedef struct {
    int *row;        /* row pointer, row_size + 1 entries              */
    int *col;        /* column index of each stored entry, *nnz        */
    int *nnz;        /* number of stored entries                        */
    int *row_size;   /* number of rows                                  */
    int *col_size;   /* number of columns                               */
    double *value;   /* stored values, *nnz                             */
    char *format;    /* "csr"                                           */
    char *type;      /* "symmetric" (one triangle stored) or other      */
} dspmat;

/* Dense column-major block (reference include/bksp.h:23-27). */
typedef struct {
    int row_size;
    int col_size;
    double *value;
} dmat;

/* ------------------------------------------------------------- accessors */

static inline int dspmat_rowsize(dspmat *mat) { return *mat->row_size; }
static inline int dspmat_colsize(dspmat *mat) { return *mat->col_size; }

static inline int dmat_set(dmat *mat, int m, int n, double num)
{
    mat->value[n * mat->row_size + m] = num;
    return 0;
}

static inline double dmat_get(dmat *mat, int m, int n)
{
    return mat->value[n * mat->row_size + m];
}

static inline int dmat_rowsize(dmat *mat) { return mat->row_size; }
static inline int dmat_colsize(dmat *mat) { return mat->col_size; }
static inline double *dmat_value(dmat *mat) { return mat->value; }

/* --------------------------------------------------------------- helpers */

/* Reads a real Matrix Market coordinate file into a newly allocated CSR
 * dspmat (reference src/read_matrix.c:38-120).  Files whose banner says
 * "symmetric" keep their single stored triangle and get type "symmetric";
 * others get "unsymmetric".  Returns NULL on an unreadable file (the
 * reference calls exit(1)).  Release with free() on each member, as the
 * reference never frees it either. */
dspmat *read_matrix_market(char *filename);

/* Thin QR of the m-by-n column-major block `mat` (m >= n): on return `mat`
 * holds Q (orthonormal columns) and `r` the n-by-n upper-triangular R,
 * column-major (reference src/myqr.c:4-39).  Computed on the GPU by shifted
 * Cholesky-QR; R's diagonal is returned non-negative, whereas LAPACK's
 * dgeqrf may return negative entries -- both are valid factorizations and
 * differ only by the signs of matching Q columns / R rows. */
int myqr(int m, int n, double *mat, double *r);

/* Dense-block helpers (reference src/util.c:5-67). */
dmat *dmat_create(int m, int n);            /* zero-filled m-by-n          */
int darray2dmat(double *arr, int row_size, int col_size, dmat *mat);
int dmat_free(dmat *mat);
/* Writes x (length row_size) into column m of mat.  The reference writes
 * mat->value[i * col_size + m], i.e. row-major into a column-major block;
 * that behaviour is kept for drop-in compatibility. */
int dvec2mat(double *x, int m, dmat *mat);

/* ------------------------------------------------ Krylov subspace methods */

/* CG (reference src/cg.c:6-71).  A must have type "symmetric". */
int bksp_dcg(dspmat *A, double *b, double tol, int max_iter, double *x);

/* Conjugate residual (reference src/cr.c:6-80).  A "symmetric".  The
 * iteration index starts at 1, as in the reference. */
int dcr(dspmat *A, double *b, double tol, int max_iter, double *x);

/* BiCG (reference src/bicg.c:7-88); uses A^T for the shadow sequence. */
int dbicg(dspmat *A, double *b, double tol, int max_iter, double *x);

/* BiCGSTAB (reference src/bicgstab.c:5-72). */
int dbicgstab(dspmat *A, double *b, double tol, int max_iter, double *x);

/* BiCGSTAB(l) of Sleijpen and Fokkema (reference src/bicgstabl.c:13-138). */
int dbicgstabl(dspmat *A, double *b, int l, double tol, int max_iter,
               double *x);

/* ------------------------------------------ Block Krylov subspace methods */

/* Block CG with an orthonormalised residual block (reference
 * src/blcg.c:15-119).  A "symmetric".  B, X: n-by-s column-major.  The
 * convergence test is ||C||_F / ||B||_F < tol. */
int dblcg(dspmat *A, dmat *B, double tol, int max_iter, dmat *X);

/* Block BiCGSTAB with an orthonormalised direction block (reference
 * src/blbicgstab.c:13-123). */
int dblbicgstab(dspmat *A, dmat *B, double tol, int max_iter, dmat *X);

/* Block BiCGSTAB(l)-RH (reference src/blbicgstabl.c:16-252).  Like the
 * reference it starts from V0 = B + A X0 (the residual only for X0 = 0),
 * tests ||xi||_F / ||B||_F < tol and prints a convergence summary. */
int dblbicgstabl(dspmat *A, dmat *B, int l, double tol, int max_iter,
                 dmat *X);

/* ------------------------------- Krylov methods for shifted systems */

/* Shifted BiCG (reference src/shbicg.c:5-129).  x holds
 * n * (sigma_size + 1) values: x[0:n] solves A x = b (the seed) and
 * x[(k+1)n:(k+2)n] solves (A + sigma[k] I) x = b.  The shifted parts must
 * start at zero.  Convergence is tested on the seed system only. */
int dshbicg(dspmat *A, double *b, double *sigma, int sigma_size, double tol,
            int max_iter, double *x);

/* Shifted BiCGSTAB(l) (reference src/shbicgstabl.c:7-285); layout and
 * convergence test as dshbicg. */
int dshbicgstabl(dspmat *A, double *b, int l, double *sigma, int sigma_size,
                 double tol, int max_iter, double *x);

/* ----------------------------------------------------- complex variants */

/* Complex-valued structs, helpers and solvers of the reference
 * (include/bksp.h:111-182), run on the GPU like the real methods
 * (capi_z.cpp).  Values are double _Complex, interleaved (re, im). */
typedef struct {
    int *row;
    int *col;
    int *nnz;
    int *row_size;
    int *col_size;
    double _Complex *value;
    char *format;
    char *type;
} zspmat;

typedef struct {
    int row_size;
    int col_size;
    double _Complex *value;
} zmat;

/* Accessors of the reference (include/bksp.h:134-161); zmat_get returns
 * the real part, as the reference's declares a double result. */
static inline int zspmat_rowsize(zspmat *mat) { return *mat->row_size; }
static inline int zspmat_colsize(zspmat *mat) { return *mat->col_size; }
static inline int zmat_set(zmat *mat, int m, int n, double _Complex *num)
{
    mat->value[n * mat->row_size + m] = *num;
    return 0;
}
static inline double zmat_get(zmat *mat, int m, int n)
{
    return __real__ mat->value[n * mat->row_size + m];
}
static inline int zmat_rowsize(zmat *mat) { return mat->row_size; }
static inline int zmat_colsize(zmat *mat) { return mat->col_size; }
static inline double _Complex *zmat_value(zmat *mat) { return mat->value; }

/* A "matrix coordinate complex" Matrix Market file as CSR (entries in file
 * order within each row); NULL if the file cannot be read or is not
 * complex (the reference exits the process). */
zspmat *zread_matrix_market(char *filename);
/* Thin QR of the column-major m-by-n mat (n <= 16): mat <- Q, r <- R
 * (column-major, upper triangular, real positive diagonal); 0 on success. */
int zqreco(int m, int n, double _Complex *mat, double _Complex *r);
zmat *zmat_create(int m, int n);
int zmat_free(zmat *mat);

int zbicg(zspmat *A, double _Complex *b, double tol, int max_iter,
          double _Complex *x);
int zbicgstabl(zspmat *A, double _Complex *b, int ell, double tol,
               int max_iter, double _Complex *x);
int zblbicgstabl(zspmat *A, zmat *b, int ell, double tol, int max_iter,
                 zmat *x);
int zshbicgstabl(zspmat *A, double _Complex *b, int l, double _Complex *sigma,
                 int sigma_size, double tol, int max_iter,
                 double _Complex *x);

#ifdef __cplusplus
}
#endif

#endif /* BKSP_H */
