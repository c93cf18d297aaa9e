/*
 * Minimal CBLAS interface used when compiling the reference ERI sources for the
 * test oracle.  Only the two routines the reference calls are declared:
 *   cblas_dgemm  (src/lible/ints/twoel/shark_mm_kernels.cpp:14,21)
 *   cblas_daxpy  (src/lible/ints/twoel/eri_kernel_funs.hpp:464-465,487-502,626-637)
 * They are implemented in oracle/cblas_forward.c, which forwards to the OpenBLAS
 * build bundled with numpy (ILP64 symbols).  Test infrastructure only.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy);

#ifdef __cplusplus
}
#endif
