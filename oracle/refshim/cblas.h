/*
 * Minimal CBLAS header for building the reference OzBLAS CPU library
 * (src/cpu of mukunoki/ozblas) against the OpenBLAS 0.3.30 that ships
 * inside scipy (libscipy_openblas-*.so), whose CBLAS symbols carry a
 * "scipy_" prefix and use 32-bit integers.
 *
 * Test infrastructure only: this header is used to compile the reference
 * library into oracle/_ref/, which serves as the bit-parity oracle and as the
 * timed CPU baseline.  Nothing in the product links against it.
 *
 * Only the routines the reference CPU sources call are declared
 * (src/cpu/ozblas_blas_wrapper.cpp: iamax, asum, scal, axpy, gemv, gemm,
 * omatcopy, dot, nrm2).
 */
#ifndef OZB_REFSHIM_CBLAS_H
#define OZB_REFSHIM_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113, CblasConjNoTrans = 114 } CBLAS_TRANSPOSE;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef int blasint;

/* level 1 */
size_t scipy_cblas_isamax(blasint n, const float *x, blasint incx);
size_t scipy_cblas_idamax(blasint n, const double *x, blasint incx);
float scipy_cblas_sasum(blasint n, const float *x, blasint incx);
double scipy_cblas_dasum(blasint n, const double *x, blasint incx);
void scipy_cblas_sscal(blasint n, float alpha, float *x, blasint incx);
void scipy_cblas_dscal(blasint n, double alpha, double *x, blasint incx);
void scipy_cblas_saxpy(blasint n, float alpha, const float *x, blasint incx, float *y, blasint incy);
void scipy_cblas_daxpy(blasint n, double alpha, const double *x, blasint incx, double *y, blasint incy);
float scipy_cblas_sdot(blasint n, const float *x, blasint incx, const float *y, blasint incy);
double scipy_cblas_ddot(blasint n, const double *x, blasint incx, const double *y, blasint incy);
float scipy_cblas_snrm2(blasint n, const float *x, blasint incx);
double scipy_cblas_dnrm2(blasint n, const double *x, blasint incx);

/* level 2 / 3 */
void scipy_cblas_sgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint m, blasint n, float alpha,
                       const float *a, blasint lda, const float *x, blasint incx, float beta, float *y, blasint incy);
void scipy_cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint m, blasint n, double alpha,
                       const double *a, blasint lda, const double *x, blasint incx, double beta, double *y, blasint incy);
void scipy_cblas_sgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, blasint m, blasint n, blasint k,
                       float alpha, const float *a, blasint lda, const float *b, blasint ldb, float beta, float *c, blasint ldc);
void scipy_cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, blasint m, blasint n, blasint k,
                       double alpha, const double *a, blasint lda, const double *b, blasint ldb, double beta, double *c, blasint ldc);

/* OpenBLAS extensions */
void scipy_cblas_somatcopy(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint rows, blasint cols, float alpha,
                           const float *a, blasint lda, float *b, blasint ldb);
void scipy_cblas_domatcopy(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint rows, blasint cols, double alpha,
                           const double *a, blasint lda, double *b, blasint ldb);
void scipy_cblas_zomatcopy(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint rows, blasint cols, const double *alpha,
                           const double *a, blasint lda, double *b, blasint ldb);
void scipy_openblas_set_num_threads(int n);
int scipy_openblas_get_num_threads(void);

#ifdef __cplusplus
}
#endif

#define cblas_isamax scipy_cblas_isamax
#define cblas_idamax scipy_cblas_idamax
#define cblas_sasum scipy_cblas_sasum
#define cblas_dasum scipy_cblas_dasum
#define cblas_sscal scipy_cblas_sscal
#define cblas_dscal scipy_cblas_dscal
#define cblas_saxpy scipy_cblas_saxpy
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_sdot scipy_cblas_sdot
#define cblas_ddot scipy_cblas_ddot
#define cblas_snrm2 scipy_cblas_snrm2
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_sgemv scipy_cblas_sgemv
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_somatcopy scipy_cblas_somatcopy
#define cblas_domatcopy scipy_cblas_domatcopy
#define cblas_zomatcopy scipy_cblas_zomatcopy

#endif
