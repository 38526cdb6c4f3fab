/* Declaration-only CBLAS header for building the reference CPU oracle.
 * Only the enums and routines the reference calls are declared; the
 * implementation comes from the OpenBLAS shared library found at link time.
 * Test infrastructure: never part of the product library. */
#pragma once
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;

void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
void cblas_dsyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 int n, int k, double alpha, const double *a, int lda,
                 double beta, double *c, int ldc);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
double cblas_dnrm2(int n, const double *x, int incx);
void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy);
void cblas_dscal(int n, double alpha, double *x, int incx);
