/* Declaration-only LAPACKE header for building the reference CPU oracle.
 * Test infrastructure: never part of the product library. */
#pragma once
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
int LAPACKE_dsyev(int layout, char jobz, char uplo, int n, double *a, int lda, double *w);
int LAPACKE_dgesdd(int layout, char jobz, int m, int n, double *a, int lda,
                   double *s, double *u, int ldu, double *vt, int ldvt);
int LAPACKE_dgeqrf(int layout, int m, int n, double *a, int lda, double *tau);
int LAPACKE_dorgqr(int layout, int m, int n, int k, double *a, int lda, const double *tau);
