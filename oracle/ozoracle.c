/*
 * ozoracle.c — CPU restatement of the OzBLAS Ozaki-scheme path (FP64 in/out,
 * FP64 slices, reproMode=1, no batched GEMM), an exact dot-product
 * accumulator, and the seeded input generators.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the parity tests, never the
 * thing measured or shipped.  Parity of this restatement with the reference
 * library itself is pinned by tests/test_oracle.py (live, against oracle/_ref)
 * and by the golden fixtures in tests/golden (generated from oracle/_ref).
 *
 * Citations are to mukunoki/ozblas, paths relative to the project root.
 * Compile with -ffp-contract=off: every a*b+c below is meant to round twice
 * unless it is written as fma().
 */
#define _GNU_SOURCE
#include "ozoracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <quadmath.h>

#define OZ_DEFAULT_MAXSPLIT 30 /* NumSplitDefaultMax, src/cpu/ozblas_common.h:5 */
#define OZ_SPLIT_CONST 0.75    /* CONST, src/cpu/ozblas_split.cpp:9 */

static int oz_max_split(const oz_flags *f) { return f->nSplitMax > 0 ? f->nSplitMax : OZ_DEFAULT_MAXSPLIT; }
static int imax(int a, int b);
static int imin(int a, int b);
static int make_pairs(int nA, int nB, int maxlevel, int *pa, int *pb);

/* std::max(a, b) as the reference uses it: returns a unless a < b. */
static inline double ref_max(double a, double b) { return (a < b) ? b : a; }

/* getRho<double,double>, src/cpu/ozblas_split.cpp:19-34 */
int oz_rho(int dim, int splitEpsMode) {
    switch (splitEpsMode) {
    case 2: return (int)ceil((53 - (106 - log2(1. * dim)) / 2));
    case 9: return (int)ceil((53 - (53 - log2(2. * sqrt(dim))) / 2));
    default: return (int)ceil((53 - (53 - log2(1. * dim)) / 2));
    }
}

/* tau = (short)ceil(log2(|max|)), src/cpu/ozblas_split.cpp:145,801 */
int oz_tau_libm(double v) {
    const short tau = (short)ceil(log2(fabs(v)));
    return tau;
}

/*
 * One split level over ncol columns of length k (mono precision):
 * src/cpu/ozblas_split.cpp:126-178 (column panel) and :62-103 (vector, same
 * arithmetic with one column).  R holds the running remainders; S receives
 * the slice; mx holds the per-column max of R on entry and of the new
 * remainder on exit.  Returns the sum of the new maxima (the termination test).
 */
static double split_level_cols(int k, int ncol, int rho, double *R, int ldr, double *S, int lds, double *mx,
                               int shift) {
    double check = 0.;
    for (int j = 0; j < ncol; j++) {
        const short tau = (short)ceil(log2(fabs(mx[j])));
        const double sigma = OZ_SPLIT_CONST * scalbn(1., rho + tau) * shift;
        double m = 0.;
        for (int i = 0; i < k; i++) {
            double x = R[(size_t)j * ldr + i];
            const double s = (x + sigma) - sigma;
            x = x - s;
            S[(size_t)j * lds + i] = s;
            R[(size_t)j * ldr + i] = x;
            m = ref_max(m, fabs(x));
        }
        mx[j] = m;
        check += m;
    }
    return check;
}

/*
 * Column-panel split driver, src/cpu/ozblas_split.cpp:254-289 (reproMode=1):
 * level 0 always runs, then levels 1.. until one leaves an all-zero
 * remainder (that level is counted) or maxS levels exist.  slices holds
 * maxS panels of lds x ncol.  Returns the split count.
 */
int oz_split_cols(const oz_flags *f, int k, int ncol, const double *X, int ldx, int shift, double *slices,
                  int lds) {
    const int rho = oz_rho(k, f->splitEpsMode);
    const int maxS = oz_max_split(f);
    double *R = (double *)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1) * (ncol > 0 ? ncol : 1));
    double *mx = (double *)malloc(sizeof(double) * (ncol > 0 ? ncol : 1));
    for (int j = 0; j < ncol; j++) {
        double m = 0.;
        for (int i = 0; i < k; i++) {
            R[(size_t)j * k + i] = X[(size_t)j * ldx + i];
            m = ref_max(m, fabs(X[(size_t)j * ldx + i]));
        }
        mx[j] = m;
    }
    split_level_cols(k, ncol, rho, R, k, slices, lds, mx, shift);
    int s = 1;
    while (s < maxS) {
        const double c = split_level_cols(k, ncol, rho, R, k, slices + (size_t)s * lds * ncol, lds, mx, shift);
        s++;
        if (c == 0.) break;
    }
    free(R);
    free(mx);
    return s;
}

/* ------------------------------------------------------------------------ */
/* Mixed form <double, float, float>: FP32 slices of double data             */
/* ------------------------------------------------------------------------ */

/* getRho<double,float>, src/cpu/ozblas_split.cpp:19-34 (epse 53 and 24) */
int oz_rho_f32(int dim, int splitEpsMode) {
    switch (splitEpsMode) {
    case 9: return (int)ceil((53 - (24 - log2(2. * sqrt(dim))) / 2));
    default: return (int)ceil((53 - (24 - log2(1. * dim)) / 2));
    }
}

/* One level, src/cpu/ozblas_split.cpp:181-221 (and the vector form :106-135): the slice is cut in
 * double and stored as scalbn(slice, -tau) in float, tau kept per column and level. */
static double split_level_cols_f32(int k, int ncol, int rho, double *R, int ldr, float *S, int lds, short *E,
                                   double *mx, int shift) {
    double check = 0.;
    for (int j = 0; j < ncol; j++) {
        const short tau = (short)ceil(log2(fabs(mx[j])));
        E[j] = tau;
        const double sigma = OZ_SPLIT_CONST * scalbn(1., rho + tau) * shift;
        double m = 0.;
        for (int i = 0; i < k; i++) {
            double x = R[(size_t)j * ldr + i];
            const double s = (x + sigma) - sigma;
            x = x - s;
            S[(size_t)j * lds + i] = (float)scalbn(s, -tau);
            R[(size_t)j * ldr + i] = x;
            m = ref_max(m, fabs(x));
        }
        mx[j] = m;
        check += m;
    }
    return check;
}

/* Split driver as oz_split_cols (src/cpu/ozblas_split.cpp:254-289); exps holds maxS rows of ncol. */
int oz_split_cols_f32(const oz_flags *f, int k, int ncol, const double *X, int ldx, int shift, float *slices,
                      int lds, short *exps) {
    const int rho = oz_rho_f32(k, f->splitEpsMode);
    const int maxS = oz_max_split(f);
    double *R = (double *)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1) * (ncol > 0 ? ncol : 1));
    double *mx = (double *)malloc(sizeof(double) * (ncol > 0 ? ncol : 1));
    for (int j = 0; j < ncol; j++) {
        double m = 0.;
        for (int i = 0; i < k; i++) {
            R[(size_t)j * k + i] = X[(size_t)j * ldx + i];
            m = ref_max(m, fabs(X[(size_t)j * ldx + i]));
        }
        mx[j] = m;
    }
    split_level_cols_f32(k, ncol, rho, R, k, slices, lds, exps, mx, shift);
    int s = 1;
    while (s < maxS) {
        const double c = split_level_cols_f32(k, ncol, rho, R, k, slices + (size_t)s * lds * ncol, lds,
                                              exps + (size_t)s * ncol, mx, shift);
        s++;
        if (c == 0.) break;
    }
    free(R);
    free(mx);
    return s;
}

/*
 * GEMM <double, float, float>, src/cpu/ozblas_gemm.cpp:3-315 with TYPE2 = TYPE3 = float: the
 * slice products are FP32 GEMMs, exact by the rho rule (so any order gives these bits), and
 * the ordered sum adds scalbn(product, tauA + tauB) in double (ozblas_sum.cpp:382-432).  The
 * reference has no NearSum for mixed types (ozblas_sum.cpp:273-296 exits), nor Dot2.  DOT,
 * NRM2 and GEMV of this form are this GEMM (src/cpu/ozblas_dot.cpp:25, ozblas_gemv.cpp:23-26).
 */
int oz_dgemm_f32(const oz_flags *f, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc, oz_info *info) {
    if (f->reproMode != 1 || f->sumMode != 0 || (f->splitEpsMode != 0 && f->splitEpsMode != 9)) return -1;
    const int is_dot = (m == 1 && n == 1);
    const int fast = is_dot ? 0 : f->fastMode;
    const int maxS = oz_max_split(f);
    const int kk = k > 0 ? k : 1;
    double *Ap = (double *)malloc(sizeof(double) * (size_t)kk * imax(m, 1));
    double *Bp = (double *)malloc(sizeof(double) * (size_t)kk * imax(n, 1));
    const int tA = !(ta == 'n' || ta == 'N'), tB = !(tb == 'n' || tb == 'N');
    for (int i = 0; i < m; i++)
        for (int l = 0; l < k; l++) Ap[(size_t)i * k + l] = tA ? A[(size_t)i * lda + l] : A[(size_t)l * lda + i];
    for (int j = 0; j < n; j++)
        for (int l = 0; l < k; l++) Bp[(size_t)j * k + l] = tB ? B[(size_t)l * ldb + j] : B[(size_t)j * ldb + l];
    float *Sa = (float *)calloc((size_t)(maxS + 1) * kk * imax(m, 1), sizeof(float));
    float *Sb = (float *)calloc((size_t)(maxS + 1) * kk * imax(n, 1), sizeof(float));
    short *Ea = (short *)calloc((size_t)(maxS + 1) * imax(m, 1), sizeof(short));
    short *Eb = (short *)calloc((size_t)(maxS + 1) * imax(n, 1), sizeof(short));
    const int nA = oz_split_cols_f32(f, k, m, Ap, k, 1, Sa, k, Ea);
    const int nB = oz_split_cols_f32(f, k, n, Bp, k, 1, Sb, k, Eb);
    int maxlevel = (nA - 1) + (nB - 1);
    maxlevel = imax(maxlevel - fast, imin(nA - 1, nB - 1));
    int *pa = (int *)malloc(sizeof(int) * nA * nB), *pb = (int *)malloc(sizeof(int) * nA * nB);
    const int np = make_pairs(nA, nB, maxlevel, pa, pb);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            double t = 0.;
            for (int p = 0; p < np; p++) {
                const float *a = Sa + (size_t)pa[p] * k * m + (size_t)i * k;
                const float *b = Sb + (size_t)pb[p] * k * n + (size_t)j * k;
                float c = 0.f;
                for (int l = 0; l < k; l++) c += a[l] * b[l]; /* exact in FP32 */
                t += scalbn((double)c, Ea[(size_t)pa[p] * m + i] + Eb[(size_t)pb[p] * n + j]);
            }
            double *cc = &C[(size_t)j * ldc + i];
            *cc = fma(alpha, t, (beta * *cc));
        }
    if (info) {
        info->nSplitA = (float)nA;
        info->nSplitB = (float)nB;
        if (is_dot)
            info->nSplitC = 1.f;
        else if (n == 1 && fast == 0)
            info->nSplitC = (float)imin(maxlevel + 1, nA);
        else
            info->nSplitC = (float)np;
    }
    free(Ap);
    free(Bp);
    free(Sa);
    free(Sb);
    free(Ea);
    free(Eb);
    free(pa);
    free(pb);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Mixed form <float, double, double>: FP64 slices of float data             */
/* ------------------------------------------------------------------------ */

/* getRho<float,double>, src/cpu/ozblas_split.cpp:19-34 (epse 24 and 53); negative for k < 32 */
int oz_rho_sd(int dim, int splitEpsMode) {
    switch (splitEpsMode) {
    case 9: return (int)ceil((24 - (53 - log2(2. * sqrt(dim))) / 2));
    default: return (int)ceil((24 - (53 - log2(1. * dim)) / 2));
    }
}

/* The reference's float helpers call the double libm functions (src/cpu/ozblas_aux.cpp:3-47 with
 * <cmath>, which declares no float overloads in the global namespace): log21<float> is
 * (float)log2((double)v), scalbn1<float> is (float)scalbn((double)v, n), fma1<float> is
 * (float)fma((double)x, (double)y, (double)z). */
static short tau_sd(float v) { return (short)ceil((float)log2((double)v)); }
short oz_tau_sd_libm(float v) { return tau_sd(v); }

/* Count the positive finite floats (bit patterns from 1, every `stride`-th) where `rule`
 * disagrees with tau_sd; the first disagreement's bits go to *first. */
long oz_tau_sd_sweep(int (*rule)(float), unsigned stride, unsigned *first) {
    long bad = 0;
    for (unsigned long u = 1; u < 0x7f800000ul; u += stride) {
        float v;
        const unsigned b = (unsigned)u;
        memcpy(&v, &b, 4);
        if (rule(v) != tau_sd(v)) {
            if (bad == 0 && first) *first = b;
            bad++;
        }
    }
    return bad;
}
static float scalbn_sd(float v, int e) { return (float)scalbn((double)v, e); }

/* One level, src/cpu/ozblas_split.cpp:181-221 with TYPE1 = float: float arithmetic, the slice
 * stored as the double scalbn(slice, -tau). */
static float split_level_cols_sd(int k, int ncol, int rho, float *R, int ldr, double *S, int lds, short *E,
                                 float *mx, int shift) {
    float check = 0.f;
    for (int j = 0; j < ncol; j++) {
        const short tau = tau_sd(mx[j]);
        E[j] = tau;
        const float sigma = (float)(OZ_SPLIT_CONST * (double)scalbn_sd(1.f, rho + tau) * shift);
        float m = 0.f;
        for (int i = 0; i < k; i++) {
            float x = R[(size_t)j * ldr + i];
            const float s = (x + sigma) - sigma;
            x = x - s;
            S[(size_t)j * lds + i] = (double)scalbn_sd(s, -tau);
            R[(size_t)j * ldr + i] = x;
            const float ax = (float)fabs((double)x);
            m = (m < ax) ? ax : m;
        }
        mx[j] = m;
        check += m;
    }
    return check;
}

int oz_split_cols_sd(const oz_flags *f, int k, int ncol, const float *X, int ldx, int shift, double *slices, int lds,
                     short *exps) {
    const int rho = oz_rho_sd(k, f->splitEpsMode);
    const int maxS = oz_max_split(f);
    float *R = (float *)malloc(sizeof(float) * (size_t)(k > 0 ? k : 1) * (ncol > 0 ? ncol : 1));
    float *mx = (float *)malloc(sizeof(float) * (ncol > 0 ? ncol : 1));
    for (int j = 0; j < ncol; j++) {
        float m = 0.f;
        for (int i = 0; i < k; i++) {
            R[(size_t)j * k + i] = X[(size_t)j * ldx + i];
            const float ax = (float)fabs((double)X[(size_t)j * ldx + i]);
            m = (m < ax) ? ax : m;
        }
        mx[j] = m;
    }
    split_level_cols_sd(k, ncol, rho, R, k, slices, lds, exps, mx, shift);
    int s = 1;
    while (s < maxS) {
        const float c = split_level_cols_sd(k, ncol, rho, R, k, slices + (size_t)s * lds * ncol, lds,
                                            exps + (size_t)s * ncol, mx, shift);
        s++;
        if (c == 0.f) break;
    }
    free(R);
    free(mx);
    return s;
}

/*
 * GEMM <float, double, double>, src/cpu/ozblas_gemm.cpp:3-315 with TYPE1 = float: exact FP64
 * slice products; the ordered sum (src/cpu/ozblas_sum.cpp:382-432) rounds each pair product to
 * float, scales it by 2^(tauA + tauB) in float and adds it to a float t; the output is
 * fma1(alpha, t, beta * C) in float.  FSum only, as for the other mixed form.
 */
int oz_sgemm_d(const oz_flags *f, char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, oz_info *info) {
    if (f->reproMode != 1 || f->sumMode != 0 || (f->splitEpsMode != 0 && f->splitEpsMode != 9)) return -1;
    const int is_dot = (m == 1 && n == 1);
    const int fast = is_dot ? 0 : f->fastMode;
    const int maxS = oz_max_split(f);
    const int kk = k > 0 ? k : 1;
    float *Ap = (float *)malloc(sizeof(float) * (size_t)kk * imax(m, 1));
    float *Bp = (float *)malloc(sizeof(float) * (size_t)kk * imax(n, 1));
    const int tA = !(ta == 'n' || ta == 'N'), tB = !(tb == 'n' || tb == 'N');
    for (int i = 0; i < m; i++)
        for (int l = 0; l < k; l++) Ap[(size_t)i * k + l] = tA ? A[(size_t)i * lda + l] : A[(size_t)l * lda + i];
    for (int j = 0; j < n; j++)
        for (int l = 0; l < k; l++) Bp[(size_t)j * k + l] = tB ? B[(size_t)l * ldb + j] : B[(size_t)j * ldb + l];
    double *Sa = (double *)calloc((size_t)(maxS + 1) * kk * imax(m, 1), sizeof(double));
    double *Sb = (double *)calloc((size_t)(maxS + 1) * kk * imax(n, 1), sizeof(double));
    short *Ea = (short *)calloc((size_t)(maxS + 1) * imax(m, 1), sizeof(short));
    short *Eb = (short *)calloc((size_t)(maxS + 1) * imax(n, 1), sizeof(short));
    const int nA = oz_split_cols_sd(f, k, m, Ap, k, 1, Sa, k, Ea);
    const int nB = oz_split_cols_sd(f, k, n, Bp, k, 1, Sb, k, Eb);
    int maxlevel = (nA - 1) + (nB - 1);
    maxlevel = imax(maxlevel - fast, imin(nA - 1, nB - 1));
    int *pa = (int *)malloc(sizeof(int) * nA * nB), *pb = (int *)malloc(sizeof(int) * nA * nB);
    const int np = make_pairs(nA, nB, maxlevel, pa, pb);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            float t = 0.f;
            for (int p = 0; p < np; p++) {
                const double *a = Sa + (size_t)pa[p] * k * m + (size_t)i * k;
                const double *b = Sb + (size_t)pb[p] * k * n + (size_t)j * k;
                double c = 0.;
                for (int l = 0; l < k; l++) c += a[l] * b[l]; /* exact in FP64 */
                t += scalbn_sd((float)c, Ea[(size_t)pa[p] * m + i] + Eb[(size_t)pb[p] * n + j]);
            }
            float *cc = &C[(size_t)j * ldc + i];
            *cc = (float)fma((double)alpha, (double)t, (double)(beta * *cc));
        }
    if (info) {
        info->nSplitA = (float)nA;
        info->nSplitB = (float)nB;
        if (is_dot)
            info->nSplitC = 1.f;
        else if (n == 1 && fast == 0)
            info->nSplitC = (float)imin(maxlevel + 1, nA);
        else
            info->nSplitC = (float)np;
    }
    free(Ap);
    free(Bp);
    free(Sa);
    free(Sb);
    free(Ea);
    free(Eb);
    free(pa);
    free(pb);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Quad I/O form <__float128, double, double>: FP64 slices of binary128 data */
/* ------------------------------------------------------------------------ */

/* getRho<__float128,double>, src/cpu/ozblas_split.cpp:19-34 (epse 113 and 53) */
int oz_rho_q(int dim, int splitEpsMode) {
    switch (splitEpsMode) {
    case 9: return (int)ceil((113 - (53 - log2(2. * sqrt(dim))) / 2));
    default: return (int)ceil((113 - (53 - log2(1. * dim)) / 2));
    }
}

/* tau of binary128 data: ceil(log21(max)) in the reference resolves to the double ceil of the
 * binary128 log2q converted to double (src/cpu/ozblas_split.cpp:201, ozblas_aux.cpp:43-46) */
static short tau_q(__float128 v) { return (short)ceil((double)log2q(v)); }
int oz_tau_q_libm(const void *v) {
    __float128 x;
    memcpy(&x, v, 16);
    return tau_q(x);
}

static double split_level_cols_q(int k, int ncol, int rho, __float128 *R, int ldr, double *S, int lds, short *E,
                                 __float128 *mx, int shift) {
    __float128 check = 0;
    for (int j = 0; j < ncol; j++) {
        const short tau = tau_q(mx[j]);
        E[j] = tau;
        const __float128 sigma = (__float128)OZ_SPLIT_CONST * scalbnq(1, rho + tau) * shift;
        __float128 m = 0;
        for (int i = 0; i < k; i++) {
            __float128 x = R[(size_t)j * ldr + i];
            const __float128 s = (x + sigma) - sigma;
            x = x - s;
            S[(size_t)j * lds + i] = (double)scalbnq(s, -tau);
            R[(size_t)j * ldr + i] = x;
            const __float128 ax = fabsq(x);
            m = (m < ax) ? ax : m;
        }
        mx[j] = m;
        check += m;
    }
    return check == 0 ? 0. : 1.;
}

int oz_split_cols_q(const oz_flags *f, int k, int ncol, const void *Xv, int ldx, double *slices, int lds,
                    short *exps) {
    const __float128 *X = (const __float128 *)Xv;
    const int rho = oz_rho_q(k, f->splitEpsMode);
    const int maxS = oz_max_split(f);
    __float128 *R = (__float128 *)malloc(sizeof(__float128) * (size_t)(k > 0 ? k : 1) * (ncol > 0 ? ncol : 1));
    __float128 *mx = (__float128 *)malloc(sizeof(__float128) * (ncol > 0 ? ncol : 1));
    for (int j = 0; j < ncol; j++) {
        __float128 m = 0;
        for (int i = 0; i < k; i++) {
            R[(size_t)j * k + i] = X[(size_t)j * ldx + i];
            const __float128 ax = fabsq(X[(size_t)j * ldx + i]);
            m = (m < ax) ? ax : m;
        }
        mx[j] = m;
    }
    split_level_cols_q(k, ncol, rho, R, k, slices, lds, exps, mx, 1);
    int s = 1;
    while (s < maxS) {
        const double c = split_level_cols_q(k, ncol, rho, R, k, slices + (size_t)s * lds * ncol, lds,
                                            exps + (size_t)s * ncol, mx, 1);
        s++;
        if (c == 0.) break;
    }
    free(R);
    free(mx);
    return s;
}

/*
 * GEMM <__float128, double, double>, src/cpu/ozblas_gemm.cpp:3-316 with TYPE1 = __float128:
 * exact FP64 slice products; the ordered sum adds scalbnq(product, tauA + tauB) in binary128
 * (src/cpu/ozblas_sum.cpp:382-432); the output is fmaq(alpha, t, beta * C).  FSum only.
 * A, B, C, alpha and beta are binary128 (16 bytes each, x86-64 layout).
 */
int oz_qgemm_d(const oz_flags *f, char ta, char tb, int m, int n, int k, const void *alphav, const void *Av, int lda,
               const void *Bv, int ldb, const void *betav, void *Cv, int ldc, oz_info *info) {
    if (f->reproMode != 1 || f->sumMode != 0 || (f->splitEpsMode != 0 && f->splitEpsMode != 9)) return -1;
    const __float128 *A = (const __float128 *)Av, *B = (const __float128 *)Bv;
    __float128 *C = (__float128 *)Cv, alpha, beta;
    memcpy(&alpha, alphav, 16);
    memcpy(&beta, betav, 16);
    const int is_dot = (m == 1 && n == 1);
    const int fast = is_dot ? 0 : f->fastMode;
    const int maxS = oz_max_split(f);
    const int kk = k > 0 ? k : 1;
    __float128 *Ap = (__float128 *)malloc(sizeof(__float128) * (size_t)kk * imax(m, 1));
    __float128 *Bp = (__float128 *)malloc(sizeof(__float128) * (size_t)kk * imax(n, 1));
    const int tA = !(ta == 'n' || ta == 'N'), tB = !(tb == 'n' || tb == 'N');
    for (int i = 0; i < m; i++)
        for (int l = 0; l < k; l++) Ap[(size_t)i * k + l] = tA ? A[(size_t)i * lda + l] : A[(size_t)l * lda + i];
    for (int j = 0; j < n; j++)
        for (int l = 0; l < k; l++) Bp[(size_t)j * k + l] = tB ? B[(size_t)l * ldb + j] : B[(size_t)j * ldb + l];
    double *Sa = (double *)calloc((size_t)(maxS + 1) * kk * imax(m, 1), sizeof(double));
    double *Sb = (double *)calloc((size_t)(maxS + 1) * kk * imax(n, 1), sizeof(double));
    short *Ea = (short *)calloc((size_t)(maxS + 1) * imax(m, 1), sizeof(short));
    short *Eb = (short *)calloc((size_t)(maxS + 1) * imax(n, 1), sizeof(short));
    const int nA = oz_split_cols_q(f, k, m, Ap, k, Sa, k, Ea);
    const int nB = oz_split_cols_q(f, k, n, Bp, k, Sb, k, Eb);
    int maxlevel = (nA - 1) + (nB - 1);
    maxlevel = imax(maxlevel - fast, imin(nA - 1, nB - 1));
    int *pa = (int *)malloc(sizeof(int) * nA * nB), *pb = (int *)malloc(sizeof(int) * nA * nB);
    const int np = make_pairs(nA, nB, maxlevel, pa, pb);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            __float128 t = 0;
            for (int p = 0; p < np; p++) {
                const double *a = Sa + (size_t)pa[p] * k * m + (size_t)i * k;
                const double *b = Sb + (size_t)pb[p] * k * n + (size_t)j * k;
                double c = 0.;
                for (int l = 0; l < k; l++) c += a[l] * b[l]; /* exact in FP64 */
                t += scalbnq((__float128)c, Ea[(size_t)pa[p] * m + i] + Eb[(size_t)pb[p] * n + j]);
            }
            __float128 *cc = &C[(size_t)j * ldc + i];
            *cc = fmaq(alpha, t, beta * *cc);
        }
    if (info) {
        info->nSplitA = (float)nA;
        info->nSplitB = (float)nB;
        if (is_dot)
            info->nSplitC = 1.f;
        else if (n == 1 && fast == 0)
            info->nSplitC = (float)imin(maxlevel + 1, nA);
        else
            info->nSplitC = (float)np;
    }
    free(Ap);
    free(Bp);
    free(Sa);
    free(Sb);
    free(Ea);
    free(Eb);
    free(pa);
    free(pb);
    return 0;
}

/* Binary128 test data: the harness's phi distribution in double, widened with a second draw
 * below its last bit so that every value uses about 107 of the 113 bits. */
void oz_gen_phi_q(int m, int n, int ld, void *outv, double phi, int seed) {
    __float128 *out = (__float128 *)outv;
    double *a = (double *)malloc(sizeof(double) * (size_t)(ld > 0 ? ld : 1) * (n > 0 ? n : 1));
    double *b = (double *)malloc(sizeof(double) * (size_t)(ld > 0 ? ld : 1) * (n > 0 ? n : 1));
    oz_gen_phi(m, n, ld, a, phi, seed);
    oz_gen_phi(m, n, ld, b, 1.0, seed + 7919);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            const size_t q = (size_t)j * ld + i;
            out[q] = (__float128)a[q] * (1 + (__float128)b[q] * 0x1p-54Q);
        }
    free(a);
    free(b);
}

/* x[i] = scalbnq(x[i], e) over n binary128 values (test data near the ends of the range) */
void oz_q_scale(void *xv, long n, int e) {
    __float128 *x = (__float128 *)xv;
    for (long i = 0; i < n; i++) x[i] = scalbnq(x[i], e);
}

/* Reference binary128 arithmetic for the tests of the library's software binary128 */
void oz_q_add(const void *a, const void *b, void *r) {
    __float128 x, y, z;
    memcpy(&x, a, 16);
    memcpy(&y, b, 16);
    z = x + y;
    memcpy(r, &z, 16);
}
void oz_q_mul(const void *a, const void *b, void *r) {
    __float128 x, y, z;
    memcpy(&x, a, 16);
    memcpy(&y, b, 16);
    z = x * y;
    memcpy(r, &z, 16);
}
void oz_q_fma(const void *a, const void *b, const void *c, void *r) {
    __float128 x, y, w, z;
    memcpy(&x, a, 16);
    memcpy(&y, b, 16);
    memcpy(&w, c, 16);
    z = fmaq(x, y, w);
    memcpy(r, &z, 16);
}
void oz_q_from_double(double d, void *r) {
    __float128 z = d;
    memcpy(r, &z, 16);
}
double oz_q_to_double(const void *a) {
    __float128 x;
    memcpy(&x, a, 16);
    return (double)x;
}

/* Bulk check of a software binary128 `rule` (the library's cuozblasRuleQ128) against gcc's
 * __float128 and libquadmath on n random cases of operation op (0 add, 1 mul, 2 fma, 3 tau,
 * 4 split); returns the number of mismatches, the first one's inputs and outputs in `first`
 * (a, b, c, got, want: 5 x 16 bytes).  Operands mix random signs and exponents, close
 * exponents (cancellation), short significands (ties), zeros and subnormals. */
static unsigned long long q_rng_state;
static unsigned long long q_rng(void) {
    q_rng_state ^= q_rng_state << 13;
    q_rng_state ^= q_rng_state >> 7;
    q_rng_state ^= q_rng_state << 17;
    return q_rng_state;
}
static __float128 q_rand(int e0, int spread) {
    unsigned long long r = q_rng();
    const int kind = (int)(r % 16);
    if (kind == 0) return (r & 16) ? -0.0Q : 0.0Q;
    unsigned __int128 m = ((unsigned __int128)q_rng() << 64) | q_rng();
    m &= (((unsigned __int128)1) << 112) - 1;
    if (kind <= 3) m &= ~((((unsigned __int128)1) << (int)(q_rng() % 112)) - 1); /* short significand */
    int e = e0 + (spread ? (int)(q_rng() % (unsigned)(2 * spread + 1)) - spread : 0);
    if (kind == 4) e = -16382 - 1 - (int)(q_rng() % 112); /* subnormal */
    if (e < -16494) e = -16494;
    if (e > 16383) e = 16383;
    __float128 v;
    if (e >= -16382) {
        unsigned long long hi = (unsigned long long)(e + 16383) << 48 | (unsigned long long)(m >> 64);
        unsigned long long lo = (unsigned long long)m;
        memcpy(&v, &lo, 8);
        memcpy((char *)&v + 8, &hi, 8);
    } else {
        v = scalbnq(1 + (__float128)(double)(m >> 60) * 0x1p-52Q, e);
    }
    return (r & 32) ? -v : v;
}
long oz_q128_check(int (*rule)(int, const void *, const void *, const void *, void *), int op, long n,
                   unsigned seed, void *first) {
    q_rng_state = 0x9E3779B97F4A7C15ULL ^ seed;
    long bad = 0;
    for (long t = 0; t < n; t++) {
        const int base = (int)(q_rng() % 4) == 0 ? (int)(q_rng() % 32000) - 16000 : (int)(q_rng() % 200) - 100;
        const int spread = (int)(q_rng() % 4) == 0 ? 200 : (int)(q_rng() % 3);
        __float128 a = q_rand(base, spread), b = q_rand(base, spread), c = q_rand(base, spread), want = 0, got = 0;
        int rt[2];
        unsigned char outb[32];
        memset(outb, 0, sizeof outb);
        if (op == 2) c = q_rand(base + (int)(q_rng() % 200) - 100, spread); /* c near a * b's binade or not */
        if (op == 0) want = a + b;
        if (op == 1) want = a * b;
        if (op == 2) want = fmaq(a, b, c);
        if (op == 3) {
            a = fabsq(a);
            if (a == 0) a = 1;
            const int w = tau_q(a);
            memcpy(&want, &w, sizeof w);
        }
        if (op == 4) {
            const __float128 mx = fabsq(a) * (1 + (__float128)(q_rng() % 4));
            rt[0] = 87 + (int)(q_rng() % 20);
            rt[1] = (mx == 0) ? 0 : tau_q(mx);
            const __float128 sigma = (__float128)OZ_SPLIT_CONST * scalbnq(1, rt[0] + rt[1]);
            const __float128 sp = (a + sigma) - sigma;
            const __float128 rem = a - sp;
            const double sl = (double)scalbnq(sp, -rt[1]);
            memcpy(&want, &rem, 16);
            b = 0;
            memcpy(&b, rt, sizeof rt);
            unsigned char wantb[32];
            memcpy(wantb, &rem, 16);
            memcpy(wantb + 16, &sl, 8);
            memset(wantb + 24, 0, 8);
            rule(op, &a, rt, &c, outb);
            if (memcmp(outb, wantb, 24) != 0) {
                if (bad == 0 && first) {
                    memcpy(first, &a, 16);
                    memcpy((char *)first + 16, rt, 8);
                    memcpy((char *)first + 48, outb, 24);
                    memcpy((char *)first + 72, wantb, 8); /* truncated record: inputs + outputs */
                }
                bad++;
            }
            continue;
        }
        if (op == 3) {
            int g = 0;
            rule(op, &a, &b, &c, &g);
            memcpy(&got, &g, sizeof g);
        } else {
            rule(op, &a, &b, &c, &got);
        }
        const int wnan = (op <= 2) && isnanq(want), gnan = (op <= 2) && isnanq(got);
        if (wnan ? !gnan : memcmp(&got, &want, 16) != 0) {
            if (bad == 0 && first) {
                memcpy(first, &a, 16);
                memcpy((char *)first + 16, &b, 16);
                memcpy((char *)first + 32, &c, 16);
                memcpy((char *)first + 48, &got, 16);
                memcpy((char *)first + 64, &want, 16);
            }
            bad++;
        }
    }
    return bad;
}

/*
 * One split level over CSR rows: src/cpu/ozblas_split.cpp:779-815.
 * rho comes from the row's nnz; sigma is divided (not multiplied) by shift.
 */
static double split_level_csr(int m, const int *rowptr, int epsmode, double *R, double *S, double *mx, int shift) {
    double check = 0.;
    for (int r = 0; r < m; r++) {
        const int lo = rowptr[r], hi = rowptr[r + 1];
        if (hi <= lo) { /* an empty row keeps max 0 and writes nothing */
            mx[r] = 0.;
            continue;
        }
        const int rho = oz_rho(hi - lo, epsmode);
        const short tau = (short)ceil(log2(mx[r]));
        const double sigma = OZ_SPLIT_CONST * scalbn(1., rho + tau) / shift;
        double mm = 0.;
        for (int i = lo; i < hi; i++) {
            double x = R[i];
            const double s = (x + sigma) - sigma;
            x = x - s;
            S[i] = s;
            R[i] = x;
            mm = ref_max(mm, fabs(x));
        }
        mx[r] = mm;
        check += mm;
    }
    return check;
}

/* CSR row split driver, src/cpu/ozblas_split.cpp:875-928.  slices: maxS x lds. */
int oz_split_rows_csr(const oz_flags *f, int m, const double *val, const int *rowptr, int shift, double *slices,
                      int lds) {
    const int maxS = oz_max_split(f);
    const int nnz = rowptr[m] - rowptr[0];
    double *R = (double *)malloc(sizeof(double) * (size_t)(rowptr[m] > 0 ? rowptr[m] : 1));
    double *mx = (double *)malloc(sizeof(double) * (m > 0 ? m : 1));
    (void)nnz;
    for (int r = 0; r < m; r++) {
        double mm = 0.;
        for (int i = rowptr[r]; i < rowptr[r + 1]; i++) {
            R[i] = val[i];
            mm = ref_max(mm, fabs(val[i]));
        }
        mx[r] = mm;
    }
    for (int i = 0; i < rowptr[m]; i++) slices[i] = 0.;
    split_level_csr(m, rowptr, f->splitEpsMode, R, slices, mx, shift);
    int s = 1;
    while (s < maxS) {
        const double c = split_level_csr(m, rowptr, f->splitEpsMode, R, slices + (size_t)s * lds, mx, shift);
        s++;
        if (c == 0.) break;
    }
    free(R);
    free(mx);
    return s;
}

/* ------------------------------------------------------------------------ */
/* NearSum (Rump, Ogita, Oishi), src/cpu/ozblas_sum.cpp:10-112               */
/* ------------------------------------------------------------------------ */

static void nearsum_transform(int n, double *v, double rho, double *tau1, double *tau2) {
    const int emin = -1022, epse = 53; /* getEmin/getEpse<double>, src/cpu/ozblas_common.h */
    if (n == 0) {
        *tau1 = rho;
        *tau2 = 0.;
        return;
    }
    double mu = fabs(v[0]);
    for (int i = 1; i < n; i++) mu = (mu > fabs(v[i])) ? mu : fabs(v[i]); /* MAX macro */
    if (mu == 0.) {
        *tau1 = rho;
        *tau2 = 0.;
        return;
    }
    const int M = (int)ceil(log2((double)(n + 2)));
    double sigma = scalbn(1., (int)(M + ceil(log2(mu))));
    double t = rho;
    for (;;) {
        double tau = 0.;
        for (int i = 0; i < n; i++) {
            const double tmp = (sigma + v[i]) - sigma;
            v[i] -= tmp;
            tau += tmp;
        }
        *tau1 = t + tau;
        if ((sigma <= scalbn(1., emin)) || (fabs(*tau1) >= scalbn(1., 2 * M + 1 - epse) * sigma)) {
            *tau2 = tau - (*tau1 - t);
            return;
        }
        sigma = scalbn(1., M - epse) * sigma;
        t = *tau1;
    }
}

static void nearsum_transformk(int n, double *v, double rho, double *res, double *r) {
    double tmp = 0., tau1, tau2;
    nearsum_transform(n, v, rho, &tau1, &tau2);
    for (int i = 0; i < n; i++) tmp += v[i];
    *res = tau1 + (tau2 + tmp);
    *r = tau2 - (*res - tau1);
}

static inline double ref_sign(double v) { return (v < 0) ? -1. : 1.; }

double oz_nearsum(int n, double *vec) {
    const double eps = scalbn(1., -53);
    double res, r, delta, r2, res2, mu, delta2, tmp;
    nearsum_transformk(n, vec, 0., &res, &r);
    nearsum_transformk(n, vec, r, &delta, &r2);
    if (delta == 0) return res;
    res2 = res + ref_sign(delta) * eps * fabs(res);
    if (res2 == res) {
        mu = ref_sign(delta) * eps * fabs(res);
        res2 = res + 2. * ref_sign(delta) * eps * fabs(res);
    } else {
        mu = (res2 - res) / 2.;
    }
    if (fabs(delta) < fabs(mu)) return res;
    if (fabs(delta) > fabs(mu)) return res2;
    nearsum_transformk(n, vec, r2, &delta2, &tmp);
    if (delta2 == 0) return res + mu;
    if (ref_sign(delta2) == ref_sign(mu)) return res2;
    return res;
}

/* ------------------------------------------------------------------------ */
/* GEMM driver, src/cpu/ozblas_gemm.cpp:3-315 (no m/n blocking)              */
/* ------------------------------------------------------------------------ */

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* Pair schedule: ik ascending, ia ascending, ib = ik - ia
 * (src/cpu/ozblas_gemm.cpp:237-243 and the sum loops of ozblas_sum.cpp:340-360). */
static int make_pairs(int nA, int nB, int maxlevel, int *pa, int *pb) {
    int np = 0;
    for (int ik = 0; ik <= maxlevel; ik++)
        for (int ia = 0; ia < nA; ia++)
            for (int ib = 0; ib < nB; ib++)
                if (ia + ib == ik) {
                    pa[np] = ia;
                    pb[np] = ib;
                    np++;
                }
    return np;
}

/* ------------------------------------------------------------------------ */
/* Dot2 (splitEpsMode 2): error-free transformations of src/cpu/eft.h       */
/* ------------------------------------------------------------------------ */

typedef struct {
    double x, y;
} dd_t;

static void eft_two_sum(double a, double b, double *s, double *e) { /* eft.h:11-19 */
    const double ss = a + b;
    const double v = ss - a;
    *e = (a - (ss - v)) + (b - v);
    *s = ss;
}
static void eft_quick_two_sum(double a, double b, double *s, double *e) { /* eft.h:51-57 */
    const double ss = a + b;
    *e = b - (ss - a);
    *s = ss;
}
static void eft_dot2i(double a, double b, dd_t *c) { /* eft.h:99-107 with TwoProdFMA :75-81 */
    const double h = a * b;
    const double r = fma(a, b, -h);
    double q;
    eft_two_sum(c->x, h, &c->x, &q);
    c->y = c->y + (q + r);
}
static dd_t eft_quad_add(dd_t a, dd_t b) { /* eft.h:129-137 */
    dd_t t, c;
    eft_two_sum(a.x, b.x, &t.x, &t.y);
    t.y = t.y + (a.y + b.y);
    eft_quick_two_sum(t.x, t.y, &c.x, &c.y);
    return c;
}
static dd_t eft_quad_mul(double a, dd_t b) { /* eft.h:166-174 */
    dd_t t, c;
    t.x = a * b.x;
    t.y = fma(a, b.x, -t.x);
    t.y = fma(a, b.y, t.y);
    eft_quick_two_sum(t.x, t.y, &c.x, &c.y);
    return c;
}

/* Dot2 DOT: dgemm_tn_skinny_x2 (src/cpu/ozblas_blas_wrapper.cpp:109-152) run by one OpenMP
 * thread (its result depends on the thread count: each thread's Dot2i partial is QuadAdd-ed
 * in critical-section order), then the sum of src/cpu/ozblas_gemm.cpp:281-287 over the hi
 * terms of every pair followed by the lo terms as B indices nB..2nB-1. */
static double dot2_dot(const oz_flags *f, int k, const double *Sa, int nA, const double *Sb, int nB) {
    double *hi = (double *)malloc(sizeof(double) * nA * nB * 2);
    for (int ib = 0; ib < nB; ib++)
        for (int ia = 0; ia < nA; ia++) {
            dd_t L = {0., 0.}, G = {0., 0.};
            const double *a = Sa + (size_t)ia * k, *b = Sb + (size_t)ib * k;
            for (int l = 0; l < k; l++) eft_dot2i(a[l], b[l], &L);
            G = eft_quad_add(G, L);
            G = eft_quad_mul(1., G); /* beta == 0: Gr = QuadMul(alpha, Gr) */
            hi[(size_t)ia * 2 * nB + ib] = G.x;
            hi[(size_t)ia * 2 * nB + nB + ib] = G.y;
        }
    const int nB2 = 2 * nB, maxlevel = (nA - 1) + (nB2 - 1);
    double *terms = (double *)malloc(sizeof(double) * nA * nB2);
    int np = 0;
    for (int ik = 0; ik <= maxlevel; ik++)
        for (int ia = 0; ia < nA; ia++) {
            const int ib = ik - ia;
            if (ib >= 0 && ib < nB2) terms[np++] = hi[(size_t)ia * nB2 + ib];
        }
    double t = 0.;
    if (f->sumMode == 1)
        t = oz_nearsum(np, terms);
    else
        for (int p = 0; p < np; p++) t += terms[p];
    free(hi);
    free(terms);
    return t;
}

int oz_dgemm(const oz_flags *f, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
             const double *B, int ldb, double beta, double *C, int ldc, oz_info *info) {
    if (f->reproMode != 1) return -1;
    const int is_dot = (m == 1 && n == 1);
    const int fast = is_dot ? 0 : f->fastMode; /* src/cpu/ozblas_gemm.cpp:26-29 */
    const int maxS = oz_max_split(f);
    const int kk = k > 0 ? k : 1;
    /* column panels: column i of Ap is row i of op(A); column j of Bp is column j of op(B) */
    double *Ap = (double *)malloc(sizeof(double) * (size_t)kk * imax(m, 1));
    double *Bp = (double *)malloc(sizeof(double) * (size_t)kk * imax(n, 1));
    const int tA = !(ta == 'n' || ta == 'N'), tB = !(tb == 'n' || tb == 'N');
    for (int i = 0; i < m; i++)
        for (int l = 0; l < k; l++) Ap[(size_t)i * k + l] = tA ? A[(size_t)i * lda + l] : A[(size_t)l * lda + i];
    for (int j = 0; j < n; j++)
        for (int l = 0; l < k; l++) Bp[(size_t)j * k + l] = tB ? B[(size_t)l * ldb + j] : B[(size_t)j * ldb + l];
    double *Sa = (double *)calloc((size_t)(maxS + 1) * kk * imax(m, 1), sizeof(double));
    double *Sb = (double *)calloc((size_t)(maxS + 1) * kk * imax(n, 1), sizeof(double));
    const int nA = oz_split_cols(f, k, m, Ap, k, 1, Sa, k);
    const int nB = oz_split_cols(f, k, n, Bp, k, 1, Sb, k);
    if (is_dot && f->splitEpsMode == 2 && f->fastMode == 0 && f->sumMode < 2) { /* ozblas_gemm.cpp:166-172 */
        const double t = dot2_dot(f, k, Sa, nA, Sb, nB);
        C[0] = fma(alpha, t, (beta * C[0]));
        if (info) {
            info->nSplitA = (float)nA;
            info->nSplitB = (float)nB;
            info->nSplitC = 1.f;
        }
        free(Ap);
        free(Bp);
        free(Sa);
        free(Sb);
        return 0;
    }
    if (f->splitEpsMode == 2) { /* Dot2 products exist only for DOT and CSRMV */
        free(Ap);
        free(Bp);
        free(Sa);
        free(Sb);
        return -1;
    }
    int maxlevel = (nA - 1) + (nB - 1);
    maxlevel = imax(maxlevel - fast, imin(nA - 1, nB - 1)); /* src/cpu/ozblas_gemm.cpp:163-164 */
    int *pa = (int *)malloc(sizeof(int) * nA * nB), *pb = (int *)malloc(sizeof(int) * nA * nB);
    const int np = make_pairs(nA, nB, maxlevel, pa, pb);
    double *terms = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < m; i++) {
            for (int p = 0; p < np; p++) {
                const double *a = Sa + (size_t)pa[p] * k * m + (size_t)i * k;
                const double *b = Sb + (size_t)pb[p] * k * n + (size_t)j * k;
                double s = 0.;
                for (int l = 0; l < k; l++) s += a[l] * b[l]; /* exact: any order gives these bits */
                terms[p] = s;
            }
            double t = 0.;
            if (f->sumMode == 1) {
                t = oz_nearsum(np, terms);
            } else {
                for (int p = 0; p < np; p++) t += terms[p];
            }
            double *c = &C[(size_t)j * ldc + i];
            *c = fma(alpha, t, (beta * *c)); /* src/cpu/ozblas_sum.cpp:366 */
        }
    }
    if (info) {
        info->nSplitA = (float)nA;
        info->nSplitB = (float)nB;
        if (is_dot)
            info->nSplitC = 1.f;
        else if (n == 1 && fast == 0)
            info->nSplitC = (float)imin(maxlevel + 1, nA);
        else
            info->nSplitC = (float)np;
    }
    free(Ap);
    free(Bp);
    free(Sa);
    free(Sb);
    free(pa);
    free(pb);
    free(terms);
    return 0;
}

/* DOT = GEMM('t','n',1,1,n) into a zero-initialised result, src/cpu/ozblas_dot.cpp:4-39 */
double oz_ddot(const oz_flags *f, int n, const double *x, const double *y, oz_info *info) {
    double ret = 0.;
    oz_dgemm(f, 't', 'n', 1, 1, n, 1., x, n, y, n, 0., &ret, 1, info);
    return ret;
}

/* NRM2 = sqrt(DOT(x,x)) on the host, src/cpu/ozblas_nrm2.cpp:3-31 */
double oz_dnrm2(const oz_flags *f, int n, const double *x, oz_info *info) { return sqrt(oz_ddot(f, n, x, x, info)); }

/* GEMV through GEMM with n=1, src/cpu/ozblas_gemv.cpp:4-30 */
int oz_dgemv(const oz_flags *f, char ta, int m, int n, double alpha, const double *A, int lda, const double *x,
             double beta, double *y, oz_info *info) {
    if (ta == 'n' || ta == 'N') return oz_dgemm(f, 'n', 'n', m, 1, n, alpha, A, lda, x, n, beta, y, m, info);
    return oz_dgemm(f, 't', 'n', n, 1, m, alpha, A, lda, x, m, beta, y, n, info);
}

/* ------------------------------------------------------------------------ */
/* CSRMV, src/cpu/ozblas_csrmv.cpp:3-181, CSRMM src/cpu/ozblas_blas_wrapper.cpp:231-255 */
/* ------------------------------------------------------------------------ */

int oz_dcsrmv_presplit(const oz_flags *f, int m, int n, int nnz, double alpha, const double *aslices, int nA,
                       int lds, const int *colind, const int *rowptr, const double *x, double beta, double *y,
                       oz_info *info) {
    const int maxS = oz_max_split(f);
    const int nn = n > 0 ? n : 1;
    double *Sx = (double *)calloc((size_t)(maxS + 1) * nn, sizeof(double));
    const int nB = oz_split_cols(f, n, 1, x, n, 1, Sx, n); /* x: vector split, rho from n */
    int maxlevel = (nA - 1) + (nB - 1);
    maxlevel = imax(maxlevel - f->fastMode, imin(nA - 1, nB - 1));
    int *pa = (int *)malloc(sizeof(int) * nA * nB), *pb = (int *)malloc(sizeof(int) * nA * nB);
    const int np = make_pairs(nA, nB, maxlevel, pa, pb);
    const int dot2 = f->splitEpsMode == 2;
    if (dot2 && f->fastMode != 0) { /* the reference's storage and sum disagree there */
        free(Sx);
        free(pa);
        free(pb);
        return -1;
    }
    const int nB2 = 2 * nB;
    double *pv = (double *)malloc(sizeof(double) * (nA * nB2 > 0 ? nA * nB2 : 1));
    double *terms = (double *)malloc(sizeof(double) * (nA * nB2 > np ? nA * nB2 : (np > 0 ? np : 1)));
    for (int r = 0; r < m; r++) {
        if (dot2) {
            /* csrmm_n_x2 (src/cpu/ozblas_blas_wrapper.cpp:262-295): Dot2i along the row, then
             * QuadMul(alpha = 1); hi of pair (ia, ib) at B index ib, lo at nB + ib; summed with
             * maxlevel (nA - 1) + (2 nB - 1) (src/cpu/ozblas_csrmv.cpp:120-162) */
            for (int ia = 0; ia < nA; ia++)
                for (int ib = 0; ib < nB; ib++) {
                    const double *a = aslices + (size_t)ia * lds;
                    const double *xs = Sx + (size_t)ib * n;
                    dd_t T = {0., 0.};
                    for (int i = rowptr[r]; i < rowptr[r + 1]; i++) eft_dot2i(a[i], xs[colind[i]], &T);
                    T = eft_quad_mul(1., T);
                    pv[ia * nB2 + ib] = T.x;
                    pv[ia * nB2 + nB + ib] = T.y;
                }
            int q = 0;
            for (int ik = 0; ik <= (nA - 1) + (nB2 - 1); ik++)
                for (int ia = 0; ia < nA; ia++) {
                    const int ib = ik - ia;
                    if (ib >= 0 && ib < nB2) terms[q++] = pv[ia * nB2 + ib];
                }
            double t = 0.;
            if (f->sumMode == 1)
                t = oz_nearsum(q, terms);
            else
                for (int p = 0; p < q; p++) t += terms[p];
            y[r] = fma(alpha, t, (beta * y[r]));
            continue;
        }
        for (int p = 0; p < np; p++) {
            const double *a = aslices + (size_t)pa[p] * lds;
            const double *xs = Sx + (size_t)pb[p] * n;
            double tr = 0.;
            for (int i = rowptr[r]; i < rowptr[r + 1]; i++) tr = fma(a[i], xs[colind[i]], tr);
            terms[p] = tr; /* alpha = 1, beta = 0 inside the slice CSRMM: C = 1 * tr */
        }
        double t = 0.;
        if (f->sumMode == 1)
            t = oz_nearsum(np, terms);
        else
            for (int p = 0; p < np; p++) t += terms[p];
        y[r] = fma(alpha, t, (beta * y[r]));
    }
    if (info) {
        int ic = 0;
        for (int ia = 0; ia < imin(maxlevel + 1, nA); ia++) ic += imin(nB, maxlevel + 1 - ia);
        info->nSplitA = (float)nA;
        info->nSplitB = (float)nB;
        info->nSplitC = (float)ic;
    }
    free(Sx);
    free(pa);
    free(pb);
    free(pv);
    free(terms);
    (void)nnz;
    return 0;
}

int oz_dcsrmv(const oz_flags *f, int m, int n, int nnz, double alpha, const double *val, const int *colind,
              const int *rowptr, const double *x, double beta, double *y, oz_info *info) {
    const int maxS = oz_max_split(f);
    const int lds = nnz > 0 ? nnz : 1;
    double *Sa = (double *)calloc((size_t)(maxS + 1) * lds, sizeof(double));
    const int nA = oz_split_rows_csr(f, m, val, rowptr, 1, Sa, lds);
    const int rc = oz_dcsrmv_presplit(f, m, n, nnz, alpha, Sa, nA, lds, colind, rowptr, x, beta, y, info);
    free(Sa);
    return rc;
}

/* SplitA with splitShift tuning, src/cpu/ozblas_csrmv.cpp:185-271 */
int oz_dcsrmv_split_a(const oz_flags *f, int m, int nnz, const double *val, const int *rowptr, double *aslices,
                      int lds, int *nsplit_out, int *shift_out) {
    int s = oz_split_rows_csr(f, m, val, rowptr, 1, aslices, lds);
    int shift = 1;
    if (f->nSplitMax == 0) {
        int sold;
        shift = 1;
        do {
            sold = s;
            shift *= 2;
            s = oz_split_rows_csr(f, m, val, rowptr, shift, aslices, lds);
        } while (sold == s && shift < 512);
        if (sold == s) shift = 1;
        s = oz_split_rows_csr(f, m, val, rowptr, shift, aslices, lds);
    }
    (void)nnz;
    *nsplit_out = s;
    *shift_out = shift;
    return 0;
}

/* Unpreconditioned CG, src/cpu/ozblas_cg.cpp:23-128 (verbose=1: history every iteration) */
int oz_dcg(const oz_flags *f, int n, int nnz, const double *val, const int *colind, const int *rowptr,
           const double *b, double *x, int maxiter, double tol, double *hist, oz_info *info) {
    const int maxS = oz_max_split(f);
    const int lds = nnz > 0 ? nnz : 1;
    double *Sa = (double *)calloc((size_t)(maxS + 1) * lds, sizeof(double));
    int nA, shift;
    oz_dcsrmv_split_a(f, n, nnz, val, rowptr, Sa, lds, &nA, &shift);
    double *r = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
    double *q = (double *)calloc(n, sizeof(double));
    const double nrmb = oz_dnrm2(f, n, b, NULL);
    memcpy(r, b, sizeof(double) * n);
    oz_dcsrmv_presplit(f, n, n, nnz, -1., Sa, nA, lds, colind, rowptr, x, 1., r, NULL);
    double dold = oz_ddot(f, n, r, r, NULL);
    double resi = sqrt(dold);
    int cnt = 0;
    if (hist) hist[cnt] = resi / nrmb;
    cnt++;
    memcpy(p, r, sizeof(double) * n);
    int it = 0;
    while (it < maxiter) {
        it++;
        oz_dcsrmv_presplit(f, n, n, nnz, 1., Sa, nA, lds, colind, rowptr, p, 0., q, NULL);
        const double tmp = oz_ddot(f, n, p, q, NULL);
        const double alpha = dold / tmp;
        for (int i = 0; i < n; i++) x[i] = fma(alpha, p[i], x[i]);
        for (int i = 0; i < n; i++) r[i] = fma(-alpha, q[i], r[i]);
        const double dnew = oz_ddot(f, n, r, r, NULL);
        resi = sqrt(dnew);
        const double beta = dnew / dold;
        dold = dnew;
        for (int i = 0; i < n; i++) p[i] = beta * p[i];
        for (int i = 0; i < n; i++) p[i] = fma(1., r[i], p[i]);
        if (hist) hist[cnt] = resi / nrmb;
        cnt++;
        if (resi / nrmb < tol) break;
    }
    if (info) {
        info->cg_numiter = it;
        info->splitShift = shift;
        info->nSplitA_ = nA;
    }
    free(Sa);
    free(r);
    free(p);
    free(q);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exact accumulation (own code; the error oracle)                          */
/* ------------------------------------------------------------------------ */

/* value = sum_i limb[i] * 2^(32 i - ACC_OFF); products of doubles reach 2^-2148 */
#define ACC_OFF 2208
#define ACC_LIMBS 140

typedef struct {
    int64_t d[ACC_LIMBS];
    long adds;
    int special; /* nonzero if an inf/nan term was seen */
} acc_t;

static void acc_init(acc_t *a) {
    memset(a->d, 0, sizeof(a->d));
    a->adds = 0;
    a->special = 0;
}

static void acc_norm(acc_t *a) {
    for (int i = 0; i < ACC_LIMBS - 1; i++) {
        const int64_t c = a->d[i] >> 32; /* arithmetic shift: floor division */
        a->d[i] -= c * ((int64_t)1 << 32);
        a->d[i + 1] += c;
    }
    a->adds = 0;
}

/* add sign * mag * 2^e (mag < 2^112) */
static void acc_add_mag(acc_t *a, int sign, unsigned __int128 mag, int e) {
    if (mag == 0) return;
    int pos = e + ACC_OFF;
    int li = pos >> 5, sh = pos & 31;
    /* spread over up to 5 limbs */
    unsigned __int128 lo = mag << sh; /* mag < 2^112, sh < 32 -> fits 144 bits? keep two parts */
    unsigned __int128 hi = (sh == 0) ? 0 : (mag >> (128 - sh));
    uint32_t parts[8];
    for (int t = 0; t < 4; t++) parts[t] = (uint32_t)(lo >> (32 * t));
    parts[4] = (uint32_t)hi;
    for (int t = 0; t < 5; t++) {
        if (li + t >= ACC_LIMBS) break;
        a->d[li + t] += sign > 0 ? (int64_t)parts[t] : -(int64_t)parts[t];
    }
    if (++a->adds >= (1L << 29)) acc_norm(a);
}

/* split a finite double into sign, 53-bit integer mantissa and exponent of its lsb */
static int dbl_parts(double v, int *sign, uint64_t *mant, int *e) {
    uint64_t b;
    memcpy(&b, &v, 8);
    *sign = (b >> 63) ? -1 : 1;
    const int be = (int)((b >> 52) & 0x7ff);
    const uint64_t fr = b & ((1ULL << 52) - 1);
    if (be == 0x7ff) return -1;
    if (be == 0) {
        *mant = fr;
        *e = -1074;
    } else {
        *mant = fr | (1ULL << 52);
        *e = be - 1075;
    }
    return 0;
}

static void acc_add_prod(acc_t *a, double x, double y) {
    int sx, sy, ex, ey;
    uint64_t mx, my;
    if (dbl_parts(x, &sx, &mx, &ex) || dbl_parts(y, &sy, &my, &ey)) {
        a->special = 1;
        return;
    }
    acc_add_mag(a, sx * sy, (unsigned __int128)mx * my, ex + ey);
}

static void acc_add_dbl(acc_t *a, double x) {
    int s, e;
    uint64_t mt;
    if (dbl_parts(x, &s, &mt, &e)) {
        a->special = 1;
        return;
    }
    acc_add_mag(a, s, (unsigned __int128)mt, e);
}

/* round the exact value to the nearest double, ties to even */
static double acc_round(acc_t *a0) {
    acc_t a = *a0;
    if (a.special) return NAN;
    acc_norm(&a);
    int neg = a.d[ACC_LIMBS - 1] < 0;
    if (neg) { /* two's complement negate of the multi-limb number (limbs are 32-bit digits after norm) */
        int64_t carry = 1;
        for (int i = 0; i < ACC_LIMBS; i++) {
            int64_t v = (~a.d[i] & 0xffffffffLL) + carry;
            carry = v >> 32;
            a.d[i] = v & 0xffffffffLL;
        }
    }
    int h = ACC_LIMBS - 1;
    while (h >= 0 && a.d[h] == 0) h--;
    if (h < 0) return 0.;
    /* 96-bit window from limbs h, h-1, h-2 */
    unsigned __int128 w = 0;
    for (int t = 0; t < 3; t++) {
        w <<= 32;
        if (h - t >= 0) w |= (uint64_t)a.d[h - t];
    }
    int sticky = 0;
    for (int i = h - 3; i >= 0; i--)
        if (a.d[i]) {
            sticky = 1;
            break;
        }
    const int wlsb = 32 * (h - 2) - ACC_OFF; /* exponent of the window's lsb */
    int msb = 127;
    while (!((w >> msb) & 1)) msb--;
    int drop = msb - 52; /* bits below the 53-bit mantissa */
    int elsb = wlsb + drop;
    if (elsb < -1074) { /* subnormal result */
        drop += (-1074 - elsb);
        elsb = -1074;
    }
    unsigned __int128 mant;
    int round = 0, stk = sticky;
    if (drop > 0) {
        if (drop > 127) {
            mant = 0;
            round = 0;
            stk = 1;
        } else {
            mant = w >> drop;
            round = (int)((w >> (drop - 1)) & 1);
            unsigned __int128 below = (drop >= 2) ? (w & (((unsigned __int128)1 << (drop - 1)) - 1)) : 0;
            if (below) stk = 1;
        }
    } else {
        mant = w << (-drop);
    }
    if (round && (stk || (mant & 1))) mant += 1;
    double r = ldexp((double)(uint64_t)mant, elsb);
    return neg ? -r : r;
}

double oz_exact_dot_rn(int n, const double *x, int incx, const double *y, int incy) {
    acc_t *a = (acc_t *)malloc(sizeof(acc_t));
    acc_init(a);
    for (int i = 0; i < n; i++) acc_add_prod(a, x[(size_t)i * incx], y[(size_t)i * incy]);
    const double r = acc_round(a);
    free(a);
    return r;
}

/* rn = RN(exact dot); relerr = |c - exact| / |exact| (0 when both are 0, inf when only exact is 0) */
void oz_exact_dot_err(int n, const double *x, int incx, const double *y, int incy, double c, double *rn,
                      double *relerr_exact) {
    acc_t *a = (acc_t *)malloc(sizeof(acc_t));
    acc_init(a);
    for (int i = 0; i < n; i++) acc_add_prod(a, x[(size_t)i * incx], y[(size_t)i * incy]);
    const double ex = acc_round(a);
    acc_add_dbl(a, -c);
    const double diff = acc_round(a);
    *rn = ex;
    if (ex == 0.)
        *relerr_exact = (diff == 0.) ? 0. : INFINITY;
    else
        *relerr_exact = fabs(diff) / fabs(ex);
    free(a);
}

/* Exact check of a block of GEMM entries: entry (i, j) of the nr x nc block is
 * row i of op(A) (k contiguous values at Arows + i * k) times column j of op(B)
 * (k values at Bcols + j * k).  Cblk holds the computed values (column-major,
 * nr x nc); rn receives RN(exact) and relerr |c - exact| / |exact| per entry
 * (0 when both are 0, inf when only the exact value is 0).  Parallel over
 * entries (OpenMP); each entry is one exact accumulation. */
void oz_exact_gemm_block(int k, int nr, const double *Arows, int nc, const double *Bcols, const double *Cblk,
                         double *rn, double *relerr) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int e = 0; e < nr * nc; e++) {
        const int i = e % nr, j = e / nr;
        oz_exact_dot_err(k, Arows + (size_t)i * k, 1, Bcols + (size_t)j * k, 1, Cblk[e], &rn[e], &relerr[e]);
    }
}

double oz_exact_sum_rn(int n, const double *v) {
    acc_t *a = (acc_t *)malloc(sizeof(acc_t));
    acc_init(a);
    for (int i = 0; i < n; i++) acc_add_dbl(a, v[i]);
    const double r = acc_round(a);
    free(a);
    return r;
}

/* ------------------------------------------------------------------------ */
/* Seeded inputs                                                            */
/* ------------------------------------------------------------------------ */

/* phi mode of mublasInitMat, testing/testing_common.cpp:703-717 (sequential drand48) */
void oz_gen_phi(int m, int n, int ld, double *mat, double phi, int seed) {
    if (ld < m) ld = m;
    srand48(seed);
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < m; i++) {
            const double mu = 0.0, sigma = 1.0;
            const double r1 = drand48();
            const double r2 = drand48();
            const double x1 = mu + (sqrt(-2. * log(r1)) * sin(2. * M_PI * r2)) * sigma;
            const double val = (r1 - 0.5) * exp(phi * x1);
            mat[(size_t)j * ld + i] = val;
        }
    }
}

/* N(0,1) by Box-Muller on drand48, one value per pair of draws */
void oz_gen_normal(int n, double *x, int seed) {
    srand48(seed);
    for (int i = 0; i < n; i++) {
        const double r1 = drand48();
        const double r2 = drand48();
        x[i] = sqrt(-2. * log(r1)) * sin(2. * M_PI * r2);
    }
}

int64_t oz_stencil7_nnz(int nx, int ny, int nz) {
    return 7LL * nx * ny * nz - 2LL * (ny * nz + nx * nz + nx * ny);
}

/* 7-point stencil on an nx*ny*nz grid, natural order (x fastest), ascending columns */
void oz_gen_stencil7(int nx, int ny, int nz, int *rowptr, int *colind) {
    int64_t p = 0;
    int r = 0;
    rowptr[0] = 0;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++, r++) {
                if (z > 0) colind[p++] = r - nx * ny;
                if (y > 0) colind[p++] = r - nx;
                if (x > 0) colind[p++] = r - 1;
                colind[p++] = r;
                if (x < nx - 1) colind[p++] = r + 1;
                if (y < ny - 1) colind[p++] = r + nx;
                if (z < nz - 1) colind[p++] = r + nx * ny;
                rowptr[r + 1] = (int)p;
            }
}

/* Poisson values (6 on the diagonal, -1 off it) plus a 0.01*U(0,1) diagonal shift per row */
void oz_gen_poisson_shift(int nx, int ny, int nz, int seed, const int *rowptr, const int *colind, double *val) {
    const int n = nx * ny * nz;
    srand48(seed);
    for (int r = 0; r < n; r++) {
        const double shift = 0.01 * drand48();
        for (int i = rowptr[r]; i < rowptr[r + 1]; i++) val[i] = (colind[i] == r) ? 6.0 + shift : -1.0;
    }
}

/* y = A x with a row-sequential fma chain (used to build b = A x_true) */
void oz_csrmv_fma(int m, const double *val, const int *colind, const int *rowptr, const double *x, double *y) {
    for (int r = 0; r < m; r++) {
        double t = 0.;
        for (int i = rowptr[r]; i < rowptr[r + 1]; i++) t = fma(val[i], x[colind[i]], t);
        y[r] = t;
    }
}
