/* Prototype-only CBLAS header for building the reference oracle against the
 * LP64 OpenBLAS that ships inside the Python environment (it exports the
 * standard unprefixed cblas_* symbols but installs no header).  Only the
 * routines the reference calls are declared; signatures follow the public
 * CBLAS specification.  Test infrastructure only. */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

double cblas_ddot(const int n, const double *x, const int incx,
                  const double *y, const int incy);
double cblas_dnrm2(const int n, const double *x, const int incx);
void cblas_daxpy(const int n, const double a, const double *x, const int incx,
                 double *y, const int incy);
void cblas_dcopy(const int n, const double *x, const int incx,
                 double *y, const int incy);
void cblas_dscal(const int n, const double a, double *x, const int incx);
void cblas_dgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE ta,
                 const enum CBLAS_TRANSPOSE tb, const int m, const int n,
                 const int k, const double alpha, const double *a,
                 const int lda, const double *b, const int ldb,
                 const double beta, double *c, const int ldc);

double cblas_dznrm2(const int n, const void *x, const int incx);
void cblas_zaxpy(const int n, const void *a, const void *x, const int incx,
                 void *y, const int incy);
void cblas_zcopy(const int n, const void *x, const int incx,
                 void *y, const int incy);
void cblas_zdotc_sub(const int n, const void *x, const int incx,
                     const void *y, const int incy, void *ret);
void cblas_zscal(const int n, const void *a, void *x, const int incx);
void cblas_zdscal(const int n, const double a, void *x, const int incx);
void cblas_zgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE ta,
                 const enum CBLAS_TRANSPOSE tb, const int m, const int n,
                 const int k, const void *alpha, const void *a, const int lda,
                 const void *b, const int ldb, const void *beta, void *c,
                 const int ldc);
#endif
