// cxx_api.cpp — the reference's C++ entry points (include/cuozblas.h:66-80 of
// mukunoki/ozblas) as explicit specializations forwarding to the C ABI, so
// objects compiled against the reference header link against this library.
// Like the reference they return 0 on success; unlike it they report a
// failure through the return value (the status code) instead of exit(1).
#include <stdio.h>

#include <cstdint>

#include "../../include/cuozblas.h"

static int32_t report(const char *fn, int s) {
    if (s != CUOZBLAS_STATUS_SUCCESS) fprintf(stderr, "OzBLAS error: %s failed with status %d\n", fn, s);
    return s;
}

void cuozblasCreate(cuozblasHandle_t *oh, uint64_t WorkSizeBytes) {
    report("cuozblasCreate", cuozblasHandleCreate(oh, WorkSizeBytes));
}

void cuozblasDestroy(cuozblasHandle_t *oh) { report("cuozblasDestroy", cuozblasHandleDestroy(oh)); }

template <>
int32_t cuozblasRnrm2<double, double, double>(cuozblasHandle_t *oh, const int32_t n, const double *devX,
                                              const int32_t incx, double *ret) {
    return report("cuozblasRnrm2", cuozblasDnrm2(oh, n, devX, incx, ret));
}

template <>
int32_t cuozblasRaxpy<double>(cuozblasHandle_t *oh, const int32_t n, const double alpha, const double *devX,
                              const int32_t incx, double *devY, const int32_t incy) {
    return report("cuozblasRaxpy", cuozblasDaxpy(oh, n, alpha, devX, incx, devY, incy));
}

template <>
int32_t cuozblasRdot<double, double, double>(cuozblasHandle_t *oh, const int32_t n, const double *devA,
                                             const int32_t incx, const double *devB, const int32_t incy,
                                             double *ret) {
    return report("cuozblasRdot", cuozblasDdot(oh, n, devA, incx, devB, incy, ret));
}

template <>
int32_t cuozblasRgemv<double, double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t m,
                                              const int32_t n, const double alpha, const double *devA,
                                              const int32_t lda, const double *devB, const int32_t incx,
                                              const double beta, double *devC, const int32_t incy) {
    return report("cuozblasRgemv", cuozblasDgemv(oh, tranA, m, n, alpha, devA, lda, devB, incx, beta, devC, incy));
}

template <>
int32_t cuozblasRgemm<double, double, double>(cuozblasHandle_t *oh, const char tranA, const char tranB,
                                              const int32_t m, const int32_t n, const int32_t k, const double alpha,
                                              const double *devA, const int32_t lda, const double *devB,
                                              const int32_t ldb, const double beta, double *devC,
                                              const int32_t ldc) {
    return report("cuozblasRgemm",
                  cuozblasDgemm(oh, tranA, tranB, m, n, k, alpha, devA, lda, devB, ldb, beta, devC, ldc));
}

template <>
int32_t cuozblasRgemm<double, int8_t, int32_t>(cuozblasHandle_t *oh, const char tranA, const char tranB,
                                               const int32_t m, const int32_t n, const int32_t k, const double alpha,
                                               const double *devA, const int32_t lda, const double *devB,
                                               const int32_t ldb, const double beta, double *devC,
                                               const int32_t ldc) {
    return report("cuozblasRgemm<int8>",
                  cuozblasDgemmI8(oh, tranA, tranB, m, n, k, alpha, devA, lda, devB, ldb, beta, devC, ldc));
}

template <>
int32_t cuozblasRnrm2<double, float, float>(cuozblasHandle_t *oh, const int32_t n, const double *devX,
                                            const int32_t incx, double *ret) {
    return report("cuozblasRnrm2<float>", cuozblasDSnrm2(oh, n, devX, incx, ret));
}

template <>
int32_t cuozblasRdot<double, float, float>(cuozblasHandle_t *oh, const int32_t n, const double *devA,
                                           const int32_t incx, const double *devB, const int32_t incy, double *ret) {
    return report("cuozblasRdot<float>", cuozblasDSdot(oh, n, devA, incx, devB, incy, ret));
}

template <>
int32_t cuozblasRgemv<double, float, float>(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n,
                                            const double alpha, const double *devA, const int32_t lda,
                                            const double *devB, const int32_t incx, const double beta, double *devC,
                                            const int32_t incy) {
    return report("cuozblasRgemv<float>",
                  cuozblasDSgemv(oh, tranA, m, n, alpha, devA, lda, devB, incx, beta, devC, incy));
}

template <>
int32_t cuozblasRgemm<double, float, float>(cuozblasHandle_t *oh, const char tranA, const char tranB, const int32_t m,
                                            const int32_t n, const int32_t k, const double alpha, const double *devA,
                                            const int32_t lda, const double *devB, const int32_t ldb,
                                            const double beta, double *devC, const int32_t ldc) {
    return report("cuozblasRgemm<float>",
                  cuozblasDSgemm(oh, tranA, tranB, m, n, k, alpha, devA, lda, devB, ldb, beta, devC, ldc));
}

template <>
int32_t cuozblasRnrm2<float, double, double>(cuozblasHandle_t *oh, const int32_t n, const float *devX,
                                             const int32_t incx, float *ret) {
    return report("cuozblasRnrm2<float,double>", cuozblasSDnrm2(oh, n, devX, incx, ret));
}

template <>
int32_t cuozblasRdot<float, double, double>(cuozblasHandle_t *oh, const int32_t n, const float *devA,
                                            const int32_t incx, const float *devB, const int32_t incy, float *ret) {
    return report("cuozblasRdot<float,double>", cuozblasSDdot(oh, n, devA, incx, devB, incy, ret));
}

template <>
int32_t cuozblasRgemv<float, double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n,
                                             const float alpha, const float *devA, const int32_t lda,
                                             const float *devB, const int32_t incx, const float beta, float *devC,
                                             const int32_t incy) {
    return report("cuozblasRgemv<float,double>",
                  cuozblasSDgemv(oh, tranA, m, n, alpha, devA, lda, devB, incx, beta, devC, incy));
}

template <>
int32_t cuozblasRgemm<float, double, double>(cuozblasHandle_t *oh, const char tranA, const char tranB,
                                             const int32_t m, const int32_t n, const int32_t k, const float alpha,
                                             const float *devA, const int32_t lda, const float *devB,
                                             const int32_t ldb, const float beta, float *devC, const int32_t ldc) {
    return report("cuozblasRgemm<float,double>",
                  cuozblasSDgemm(oh, tranA, tranB, m, n, k, alpha, devA, lda, devB, ldb, beta, devC, ldc));
}

#if defined(__SIZEOF_FLOAT128__)
// The quad I/O form: not instantiated by the reference's CUDA library (its
// CPU library has it, src/cpu/ozblas_gemm.cpp:316); offered here with the
// same template signature.
template <>
int32_t cuozblasRgemm<__float128, double, double>(cuozblasHandle_t *oh, const char tranA, const char tranB,
                                                  const int32_t m, const int32_t n, const int32_t k,
                                                  const __float128 alpha, const __float128 *devA, const int32_t lda,
                                                  const __float128 *devB, const int32_t ldb, const __float128 beta,
                                                  __float128 *devC, const int32_t ldc) {
    return report("cuozblasRgemm<__float128>",
                  cuozblasQgemm(oh, tranA, tranB, m, n, k, &alpha, devA, lda, devB, ldb, &beta, devC, ldc));
}

template <>
int32_t cuozblasRgemv<__float128, double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t m,
                                                  const int32_t n, const __float128 alpha, const __float128 *devA,
                                                  const int32_t lda, const __float128 *devB, const int32_t incx,
                                                  const __float128 beta, __float128 *devC, const int32_t incy) {
    return report("cuozblasRgemv<__float128>",
                  cuozblasQgemv(oh, tranA, m, n, &alpha, devA, lda, devB, incx, &beta, devC, incy));
}

template <>
int32_t cuozblasRdot<__float128, double, double>(cuozblasHandle_t *oh, const int32_t n, const __float128 *devA,
                                                 const int32_t incx, const __float128 *devB, const int32_t incy,
                                                 __float128 *ret) {
    return report("cuozblasRdot<__float128>", cuozblasQdot(oh, n, devA, incx, devB, incy, ret));
}

template <>
int32_t cuozblasRnrm2<__float128, double, double>(cuozblasHandle_t *oh, const int32_t n, const __float128 *devX,
                                                  const int32_t incx, __float128 *ret) {
    return report("cuozblasRnrm2<__float128>", cuozblasQnrm2(oh, n, devX, incx, ret));
}
#endif

template <>
int32_t cuozblasRcsrmv<double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n,
                                       const int32_t nnz, const double alpha, const cusparseMatDescr_t descrA,
                                       const double *devA, const int32_t *devAcolind, const int32_t *devArowptr,
                                       const double *devB, const double beta, double *devC) {
    return report("cuozblasRcsrmv", cuozblasDcsrmv(oh, tranA, m, n, nnz, alpha, descrA, devA, devAcolind,
                                                   devArowptr, devB, beta, devC));
}

template <>
double *cuozblasRcsrmvSplitA<double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t m,
                                             const int32_t n, const int32_t nnz, const cusparseMatDescr_t descrA,
                                             const double *devA, const int32_t *devArowptr) {
    double *out = nullptr;
    if (report("cuozblasRcsrmvSplitA",
               cuozblasDcsrmvSplitA(oh, tranA, m, n, nnz, descrA, devA, devArowptr, &out)) != 0)
        return nullptr;
    return out;
}

template <>
int32_t cuozblasRcg<double, double>(cuozblasHandle_t *oh, const char tranA, const int32_t dimN, const int32_t dimNNZ,
                                    const cusparseMatDescr_t descrA, const double *matA, const int32_t *matAcolind,
                                    const int32_t *matArowptr, const double *vecB, double *vecX, int32_t maxiter,
                                    double tol) {
    return report("cuozblasRcg", cuozblasDcg(oh, tranA, dimN, dimNNZ, descrA, matA, matAcolind, matArowptr, vecB,
                                             vecX, maxiter, tol));
}
