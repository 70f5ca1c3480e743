/* Prototype-only LAPACKE header (LP64, column-major entry points) for
 * building the reference oracle against the environment's OpenBLAS, which
 * exports LAPACKE_* but installs no header.  Signatures follow the public
 * LAPACKE interface.  Test infrastructure only. */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

lapack_int LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double *a,
                          lapack_int lda, double *tau);
lapack_int LAPACKE_dorgqr(int layout, lapack_int m, lapack_int n,
                          lapack_int k, double *a, lapack_int lda,
                          const double *tau);
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a,
                         lapack_int lda, lapack_int *ipiv, double *b,
                         lapack_int ldb);
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double *a,
                          lapack_int lda, lapack_int *ipiv);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double *a, lapack_int lda,
                          const lapack_int *ipiv);
lapack_int LAPACKE_dgetrs(int layout, char trans, lapack_int n,
                          lapack_int nrhs, const double *a, lapack_int lda,
                          const lapack_int *ipiv, double *b, lapack_int ldb);
lapack_int LAPACKE_dlarnv(lapack_int idist, lapack_int *iseed, lapack_int n,
                          double *x);

lapack_int LAPACKE_zgeqrf(int layout, lapack_int m, lapack_int n,
                          double _Complex *a, lapack_int lda,
                          double _Complex *tau);
lapack_int LAPACKE_zungqr(int layout, lapack_int m, lapack_int n,
                          lapack_int k, double _Complex *a, lapack_int lda,
                          const double _Complex *tau);
lapack_int LAPACKE_zgesv(int layout, lapack_int n, lapack_int nrhs,
                         double _Complex *a, lapack_int lda, lapack_int *ipiv,
                         double _Complex *b, lapack_int ldb);
lapack_int LAPACKE_zgetrf(int layout, lapack_int m, lapack_int n,
                          double _Complex *a, lapack_int lda,
                          lapack_int *ipiv);
lapack_int LAPACKE_zgetri(int layout, lapack_int n, double _Complex *a,
                          lapack_int lda, const lapack_int *ipiv);
lapack_int LAPACKE_zlarnv(lapack_int idist, lapack_int *iseed, lapack_int n,
                          double _Complex *x);
#endif
