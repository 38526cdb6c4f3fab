/* Reference-ABI drop-in for the dense factorisations of the site-tensor
 * decomposition.
 *
 * The reference's siteTensor_decompose.c keeps its symmetry bookkeeping,
 * singular-value selection and block copies on the host (they are exact
 * integer work and O(D^2) copies) and hands every symmetry sector's dense
 * matrix to LAPACK: LAPACKE_dgesdd('S') per sector in svdblocks
 * (src/siteTensor_decompose.c:1050-1072), LAPACKE_dgesdd('N') in R_svd
 * (:549-572), LAPACKE_dgeqrf + LAPACKE_dorgqr per sector in qrblocks
 * (:270-311).  Those three LAPACKE entry points are the boundary here: this
 * file exports them with LAPACKE's signatures (column-major only) and runs
 * the factorisations on the GPU (t3ns_gesdd_host, t3ns_geqrf_host,
 * t3ns_orgqr_host).  Linked ahead of the BLAS/LAPACK library, they replace
 * the library's versions for the whole reference driver.
 *
 * Return values follow LAPACK: 0 on success, -i for an illegal i-th
 * argument, 1 when the SVD did not converge.  A device failure (out of
 * memory, a CUDA error) prints the engine's message and exits, as the
 * reference does when an allocation fails.
 */
#include <stdio.h>
#include <stdlib.h>

#include "t3ns_b200.h"

#define T3NS_LAPACK_COL_MAJOR 102

static int dense_status(int rc, const char *who)
{
        if (rc == T3NS_OK) return 0;
        if (rc == T3NS_E_EIG) return 1;
        if (rc == T3NS_E_ARG) return -1;
        fprintf(stderr, "t3ns drop-in: %s: %s\n", who, t3ns_last_error());
        exit(EXIT_FAILURE);
}

int LAPACKE_dgesdd(int layout, char jobz, int m, int n, double *a, int lda, double *s, double *u,
                   int ldu, double *vt, int ldvt)
{
        if (layout != T3NS_LAPACK_COL_MAJOR) return -1;
        if (jobz != 'S' && jobz != 'N') return -2;
        return dense_status(t3ns_gesdd_host(jobz, m, n, a, lda, s, u, ldu, vt, ldvt),
                            "LAPACKE_dgesdd");
}

int LAPACKE_dgeqrf(int layout, int m, int n, double *a, int lda, double *tau)
{
        if (layout != T3NS_LAPACK_COL_MAJOR) return -1;
        return dense_status(t3ns_geqrf_host(m, n, a, lda, tau), "LAPACKE_dgeqrf");
}

int LAPACKE_dorgqr(int layout, int m, int n, int k, double *a, int lda, const double *tau)
{
        if (layout != T3NS_LAPACK_COL_MAJOR) return -1;
        return dense_status(t3ns_orgqr_host(m, n, k, a, lda, tau), "LAPACKE_dorgqr");
}
