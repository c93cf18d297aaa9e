/*
 * Test infrastructure only (oracle build).  Forwards the two CBLAS routines the
 * reference ERI code needs to numpy's bundled OpenBLAS, which exports them with an
 * ILP64 interface under the names scipy_cblas_dgemm64_ / scipy_cblas_daxpy64_.
 * With -DORACLE_NAIVE_BLAS a plain triple loop is used instead (enough for parity).
 */
#include <stdint.h>
#include "cblas/cblas.h"

#ifndef ORACLE_NAIVE_BLAS
extern void scipy_cblas_dgemm64_(int order, int ta, int tb, int64_t m, int64_t n, int64_t k,
                                 double alpha, const double *a, int64_t lda, const double *b,
                                 int64_t ldb, double beta, double *c, int64_t ldc);
extern void scipy_cblas_daxpy64_(int64_t n, double alpha, const double *x, int64_t incx,
                                 double *y, int64_t incy);
#endif

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc)
{
#ifndef ORACLE_NAIVE_BLAS
    scipy_cblas_dgemm64_((int)order, (int)ta, (int)tb, m, n, k, alpha, a, lda, b, ldb, beta,
                         c, ldc);
#else
    /* row-major, no transposes: the only form the reference uses */
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int l = 0; l < k; l++)
                s += a[i * lda + l] * b[l * ldb + j];
            c[i * ldc + j] = alpha * s + beta * c[i * ldc + j];
        }
    (void)order; (void)ta; (void)tb;
#endif
}

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy)
{
#ifndef ORACLE_NAIVE_BLAS
    scipy_cblas_daxpy64_(n, alpha, x, incx, y, incy);
#else
    for (int i = 0; i < n; i++)
        y[i * incy] += alpha * x[i * incx];
#endif
}
