/*
 * extern "C" entry points into the reference OzBLAS CPU library
 * (mukunoki/ozblas src/cpu, compiled unmodified where it lies).
 *
 * Test infrastructure only.  The parity tests and the CPU-baseline leg of the
 * benchmark call these through ctypes; the product never links them.
 *
 * Every wrapper forwards to the reference's own public template API
 * (include/ozblas.h:60-76) or, for the slice-level checks, to its internal
 * split routines (src/cpu/ozblas_internal.h:28-33), with the handle flags the
 * caller sets through ref_set_flags().
 */
#include <cstring>
#include "ozblas_common.h"

extern "C" {

void *ref_create(uint64_t work_bytes) {
    ozblasHandle_t *h = new ozblasHandle_t;
    memset(h, 0, sizeof(*h));
    ozblasCreate(h, work_bytes);
    return h;
}

void ref_destroy(void *hp) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    ozblasDestroy(h);
    delete h;
}

void ref_set_flags(void *hp, int nSplitMax, int splitMode, int fastMode, int reproMode, int sumMode,
                   int splitEpsMode, int useBatchedGemmFlag, int verbose, int trueresFlag) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    h->nSplitMax = nSplitMax;
    h->splitMode = splitMode;
    h->fastMode = fastMode;
    h->reproMode = reproMode;
    h->sumMode = sumMode;
    h->splitEpsMode = splitEpsMode;
    h->useBatchedGemmFlag = useBatchedGemmFlag;
    h->verbose = verbose;
    h->trueresFlag = trueresFlag;
}

/* exec info: nSplitA, nSplitB, nSplitC, mbk, nbk, splitShift, nSplitA_, cg_numiter */
void ref_get_info(void *hp, float *f3, int *i5) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    f3[0] = h->nSplitA;
    f3[1] = h->nSplitB;
    f3[2] = h->nSplitC;
    i5[0] = h->mbk;
    i5[1] = h->nbk;
    i5[2] = h->splitShift;
    i5[3] = h->nSplitA_;
    i5[4] = h->cg_numiter;
}

void ref_set_threads(int n) {
    omp_set_num_threads(n);
    scipy_openblas_set_num_threads(n);
}

int ref_get_threads(void) { return omp_get_max_threads(); }

int ref_dgemm(void *hp, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
              const double *B, int ldb, double beta, double *C, int ldc) {
    return ozblasRgemm<double, double, double>((ozblasHandle_t *)hp, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta,
                                               C, ldc);
}

/* the mixed form <double, float, float>: double data, FP32 slices and slice products */
int ref_dgemm_f32(void *hp, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                  const double *B, int ldb, double beta, double *C, int ldc) {
    return ozblasRgemm<double, float, float>((ozblasHandle_t *)hp, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                                             ldc);
}

/* the mixed form <float, double, double>: float data, FP64 slices and slice products */
int ref_sgemm_d(void *hp, char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda, const float *B,
                int ldb, float beta, float *C, int ldc) {
    return ozblasRgemm<float, double, double>((ozblasHandle_t *)hp, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                                              ldc);
}

float ref_sdot_d(void *hp, int n, const float *x, const float *y) {
    return ozblasRdot<float, double, double>((ozblasHandle_t *)hp, n, x, 1, y, 1);
}

float ref_snrm2_d(void *hp, int n, const float *x) {
    return ozblasRnrm2<float, double, double>((ozblasHandle_t *)hp, n, x, 1);
}

int ref_sgemv_d(void *hp, char ta, int m, int n, float alpha, const float *A, int lda, const float *x, float beta,
                float *y) {
    return ozblasRgemv<float, double, double>((ozblasHandle_t *)hp, ta, m, n, alpha, A, lda, x, 1, beta, y, 1);
}

/* the quad I/O form <__float128, double, double> (binary128 data as 16-byte values) */
int ref_qgemm_d(void *hp, char ta, char tb, int m, int n, int k, const void *alpha, const void *A, int lda,
                const void *B, int ldb, const void *beta, void *C, int ldc) {
    __float128 al, be;
    memcpy(&al, alpha, 16);
    memcpy(&be, beta, 16);
    return ozblasRgemm<__float128, double, double>((ozblasHandle_t *)hp, ta, tb, m, n, k, al, (const __float128 *)A,
                                                   lda, (const __float128 *)B, ldb, be, (__float128 *)C, ldc);
}

void ref_qdot_d(void *hp, int n, const void *x, const void *y, void *ret) {
    const __float128 r = ozblasRdot<__float128, double, double>((ozblasHandle_t *)hp, n, (const __float128 *)x, 1,
                                                                (const __float128 *)y, 1);
    memcpy(ret, &r, 16);
}

void ref_qnrm2_d(void *hp, int n, const void *x, void *ret) {
    const __float128 r = ozblasRnrm2<__float128, double, double>((ozblasHandle_t *)hp, n, (const __float128 *)x, 1);
    memcpy(ret, &r, 16);
}

/* the reference's tau expression for binary128 data, as its split writes it */
int ref_tau_q(const void *v) {
    __float128 x;
    memcpy(&x, v, 16);
    const short tau = ceil(log21(fabs1(x)));
    return tau;
}

/* log21<float> of the reference (src/cpu/ozblas_aux.cpp:37-42), for the tau rule of float data */
float ref_log21f(float v) { return log21<float>(v); }

double ref_ddot_f32(void *hp, int n, const double *x, const double *y) {
    return ozblasRdot<double, float, float>((ozblasHandle_t *)hp, n, x, 1, y, 1);
}

double ref_dnrm2_f32(void *hp, int n, const double *x) {
    return ozblasRnrm2<double, float, float>((ozblasHandle_t *)hp, n, x, 1);
}

int ref_dgemv_f32(void *hp, char ta, int m, int n, double alpha, const double *A, int lda, const double *x,
                  double beta, double *y) {
    return ozblasRgemv<double, float, float>((ozblasHandle_t *)hp, ta, m, n, alpha, A, lda, x, 1, beta, y, 1);
}

double ref_ddot(void *hp, int n, const double *x, const double *y) {
    return ozblasRdot<double, double, double>((ozblasHandle_t *)hp, n, x, 1, y, 1);
}

double ref_dnrm2(void *hp, int n, const double *x) {
    return ozblasRnrm2<double, double, double>((ozblasHandle_t *)hp, n, x, 1);
}

int ref_dgemv(void *hp, char ta, int m, int n, double alpha, const double *A, int lda, const double *x,
              double beta, double *y) {
    return ozblasRgemv<double, double, double>((ozblasHandle_t *)hp, ta, m, n, alpha, A, lda, x, 1, beta, y, 1);
}

int ref_daxpy(void *hp, int n, double alpha, const double *x, double *y) {
    return ozblasRaxpy<double>((ozblasHandle_t *)hp, n, alpha, x, 1, y, 1);
}

int ref_dcsrmv(void *hp, int m, int n, int nnz, double alpha, const double *val, const int *colind,
               const int *rowptr, const double *x, double beta, double *y) {
    return ozblasRcsrmv<double, double>((ozblasHandle_t *)hp, 'n', m, n, nnz, alpha, "G", val, colind, rowptr, x,
                                        beta, y);
}

/* CG: history arrays must hold maxiter+1 entries when verbose == 1 */
int ref_dcg(void *hp, int n, int nnz, const double *val, const int *colind, const int *rowptr, const double *b,
            double *x, int maxiter, double tol, double *hist1, double *hist2) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    h->cg_verbose1 = hist1;
    h->cg_verbose2 = hist2;
    return ozblasRcg<double, double>(h, 'n', n, nnz, "G", val, colind, rowptr, b, x, maxiter, tol);
}

/*
 * Split of a k x n column panel (each column split independently, as the
 * GEMM driver does for A^T and for B).  `slices` receives nSplit panels of
 * ld x n (ld = 8-aligned k); returns the split count.
 */
int ref_split_panel(void *hp, int k, int n, const double *X, int ldx, double *slices, int *ld_out) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    int maxS = (h->nSplitMax > 0) ? h->nSplitMax : NumSplitDefaultMax;
    int ld = getPitchSize(k);
    double *work = new double[(size_t)ld * (n > 0 ? n : 1)];
    double *mx = new double[n > k ? n : k];
    short *spexp = new short[(size_t)(maxS + 2) * (n > 0 ? n : 1)];
    int s = ozblasSplit<double, double>(h, 'c', k, n, X, ldx, work, ld, slices, ld, spexp, n, mx);
    delete[] work;
    delete[] mx;
    delete[] spexp;
    *ld_out = ld;
    return s;
}

/* Split of one CSR matrix by rows (per-row rho from the row nnz).  slices: nnz x (maxS+1). */
int ref_split_sparse(void *hp, int m, const double *val, const int *rowptr, int nnz, double *slices, int *ld_out) {
    ozblasHandle_t *h = (ozblasHandle_t *)hp;
    int maxS = (h->nSplitMax > 0) ? h->nSplitMax : NumSplitDefaultMax;
    int ld = getPitchSize(nnz);
    double *work = new double[nnz > 0 ? nnz : 1];
    double *mx = new double[m > 0 ? m : 1];
    short *spexp = new short[(size_t)(maxS + 2) * (m > 0 ? m : 1)];
    int s = ozblasSplitSparse<double, double>(h, 'r', m, val, rowptr, work, slices, ld, spexp, m, mx);
    delete[] work;
    delete[] mx;
    delete[] spexp;
    *ld_out = ld;
    return s;
}

/* glibc's ceil(log2(v)) narrowed to short, exactly as the split kernels use it. */
int ref_tau(double v) {
    const short tau = ceil(log21(fabs1(v)));
    return tau;
}

} /* extern "C" */
