/*
 * ozoracle — CPU restatement of the OzBLAS Ozaki-scheme path (FP64 in/out,
 * FP64 slices), plus an exact dot-product accumulator and the seeded input
 * generators used by the parity tests.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * checker.  The product (ozblas_b200) never calls it.
 *
 * The restatement follows the reference CPU library, mukunoki/ozblas
 * src/cpu; each function cites the file:line it restates.  Its output
 * is pinned against the reference library itself (oracle/_ref, built from
 * the reference sources) and against the golden fixtures in tests/golden.
 */
#ifndef OZORACLE_H
#define OZORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* handle flags that change the arithmetic (include/ozblas.h:15-30) */
typedef struct {
    int nSplitMax;    /* 0 = split until exact, capped at 30 */
    int splitMode;    /* only 0/1 (1 prints a warning in the reference) */
    int fastMode;     /* levels dropped from the pair set (CPU meaning) */
    int reproMode;    /* 1 required for the restated paths */
    int sumMode;      /* 0 = ordered FP sum, 1 = NearSum */
    int splitEpsMode; /* 0 (standard), 9 (overflow variant) */
} oz_flags;

/* execution info the reference records in its handle */
typedef struct {
    float nSplitA, nSplitB, nSplitC;
    int splitShift;   /* SplitA's tuned shift (CSRMV/CG) */
    int nSplitA_;
    int cg_numiter;
} oz_info;

/* ---- split helpers ---- */
int oz_rho(int dim, int splitEpsMode);
int oz_rho_f32(int dim, int splitEpsMode);
int oz_rho_sd(int dim, int splitEpsMode);
int oz_rho_q(int dim, int splitEpsMode);
int oz_tau_q_libm(const void *v);
int oz_split_cols_q(const oz_flags *f, int k, int ncol, const void *X, int ldx, double *slices, int lds, short *exps);
int oz_qgemm_d(const oz_flags *f, char ta, char tb, int m, int n, int k, const void *alpha, const void *A, int lda,
               const void *B, int ldb, const void *beta, void *C, int ldc, oz_info *info);
void oz_gen_phi_q(int m, int n, int ld, void *out, double phi, int seed);
void oz_q_scale(void *x, long n, int e);
void oz_q_add(const void *a, const void *b, void *r);
void oz_q_mul(const void *a, const void *b, void *r);
void oz_q_fma(const void *a, const void *b, const void *c, void *r);
void oz_q_from_double(double d, void *r);
double oz_q_to_double(const void *a);
long oz_q128_check(int (*rule)(int, const void *, const void *, const void *, void *), int op, long n,
                   unsigned seed, void *first);
short oz_tau_sd_libm(float v);
long oz_tau_sd_sweep(int (*rule)(float), unsigned stride, unsigned *first);
int oz_split_cols_sd(const oz_flags *f, int k, int ncol, const float *X, int ldx, int shift, double *slices, int lds,
                     short *exps);
int oz_sgemm_d(const oz_flags *f, char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, oz_info *info);
int oz_split_cols_f32(const oz_flags *f, int k, int ncol, const double *X, int ldx, int shift, float *slices,
                      int lds, short *exps);
int oz_dgemm_f32(const oz_flags *f, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc, oz_info *info);
int oz_tau_libm(double v);          /* (short)ceil(log2(v)) as the reference evaluates it */

int oz_split_cols(const oz_flags *f, int k, int ncol, const double *X, int ldx, int shift, double *slices,
                  int lds);
int oz_split_rows_csr(const oz_flags *f, int m, const double *val, const int *rowptr, int shift, double *slices,
                      int lds);

/* ---- summation ---- */
double oz_nearsum(int n, double *vec); /* mutates vec, like the reference */

/* ---- BLAS-level restatements ---- */
int oz_dgemm(const oz_flags *f, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
             const double *B, int ldb, double beta, double *C, int ldc, oz_info *info);
double oz_ddot(const oz_flags *f, int n, const double *x, const double *y, oz_info *info);
double oz_dnrm2(const oz_flags *f, int n, const double *x, oz_info *info);
int oz_dgemv(const oz_flags *f, char ta, int m, int n, double alpha, const double *A, int lda, const double *x,
             double beta, double *y, oz_info *info);
int oz_dcsrmv(const oz_flags *f, int m, int n, int nnz, double alpha, const double *val, const int *colind,
              const int *rowptr, const double *x, double beta, double *y, oz_info *info);
int oz_dcsrmv_presplit(const oz_flags *f, int m, int n, int nnz, double alpha, const double *aslices, int nsa,
                       int lds, const int *colind, const int *rowptr, const double *x, double beta, double *y,
                       oz_info *info);
int oz_dcsrmv_split_a(const oz_flags *f, int m, int nnz, const double *val, const int *rowptr, double *aslices,
                      int lds, int *nsplit_out, int *shift_out);
int oz_dcg(const oz_flags *f, int n, int nnz, const double *val, const int *colind, const int *rowptr,
           const double *b, double *x, int maxiter, double tol, double *hist, oz_info *info);

/* ---- exact arithmetic (error oracle) ---- */
double oz_exact_dot_rn(int n, const double *x, int incx, const double *y, int incy);
void oz_exact_dot_err(int n, const double *x, int incx, const double *y, int incy, double c, double *rn,
                      double *relerr_exact);
void oz_exact_gemm_block(int k, int nr, const double *Arows, int nc, const double *Bcols, const double *Cblk,
                         double *rn, double *relerr);
double oz_exact_sum_rn(int n, const double *v);

/* ---- seeded inputs ---- */
void oz_gen_phi(int m, int n, int ld, double *mat, double phi, int seed);
int64_t oz_stencil7_nnz(int nx, int ny, int nz);
void oz_gen_stencil7(int nx, int ny, int nz, int *rowptr, int *colind);
void oz_gen_poisson_shift(int nx, int ny, int nz, int seed, const int *rowptr, const int *colind, double *val);
void oz_gen_normal(int n, double *x, int seed);
void oz_csrmv_fma(int m, const double *val, const int *colind, const int *rowptr, const double *x, double *y);

#ifdef __cplusplus
}
#endif
#endif
