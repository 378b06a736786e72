// csrmv.cu — Ozaki CSRMV (src/cuda/cuozblas_csrmv.cu:3-133, CPU
// src/cpu/ozblas_csrmv.cpp:3-181) and the vector updates CG needs.
//
// The slice CSRMM of the reference CPU path accumulates each row with a
// sequential fma chain in storage order (src/cpu/ozblas_blas_wrapper.cpp:231-255
// and the _l2.._l5 variants), then scales by alpha = 1.  One thread per row
// runs the same chain for every slice pair, so the products carry the CPU's
// bits whether or not they are exact (with splitShift > 1 they need not be).
#include "ozb_internal.h"
#include "eft.cuh"
#include "sum.cuh"

namespace ozb {

// y = fma(alpha, t, beta*y) with t the pair sum of the row (FSUM), or the
// pair products written to pbuf[p * m + row] and NearSum-ed (sum_mode 1).
__global__ void __launch_bounds__(256) k_csrmv_pairs(int m, const double *__restrict__ As, int64_t lda_s,
                                                     const int *__restrict__ colind, const int *__restrict__ rowptr,
                                                     const double *__restrict__ xs, int64_t ldx, int nA, int nB,
                                                     int maxlevel, int sum_mode, double alpha, double beta,
                                                     double *__restrict__ y, double *__restrict__ pbuf) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int lo = rowptr[row], hi = rowptr[row + 1];
    double t = 0.0;
    int p = 0;
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) {
        const double *a = As + (size_t)ia * lda_s;
        const double *x = xs + (size_t)ib * ldx;
        double tr = 0.0;
        for (int i = lo; i < hi; i++) tr = fma(a[i], x[colind[i]], tr);
        if (sum_mode == 1)
            pbuf[(size_t)p * m + row] = tr;
        else
            t += tr;
        p++;
    });
    if (sum_mode == 1) t = nearsum(p, pbuf + row, m);
    y[row] = fma(alpha, t, beta * y[row]);
}

// Dot2 CSRMV (splitEpsMode 2, fastMode 0): csrmm_n_x2 of the reference
// (src/cpu/ozblas_blas_wrapper.cpp:262-295) per row and pair, Dot2i along the
// row in storage order then QuadMul(1); pair (ia, ib)'s hi term at B index ib
// and lo term at nB + ib, summed over levels (nA - 1) + (2 nB - 1)
// (src/cpu/ozblas_csrmv.cpp:120-162).  tbuf: 4 nA nB terms per row, stride m.
__global__ void __launch_bounds__(256) k_csrmv_pairs_dot2(int m, const double *__restrict__ As, int64_t lda_s,
                                                          const int *__restrict__ colind,
                                                          const int *__restrict__ rowptr, const double *__restrict__ xs,
                                                          int64_t ldx, int nA, int nB, int sum_mode, double alpha,
                                                          double beta, double *__restrict__ y,
                                                          double *__restrict__ tbuf) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int lo = rowptr[row], hi = rowptr[row + 1], nB2 = 2 * nB;
    double *pv = tbuf + row, *terms = tbuf + (size_t)nA * nB2 * m + row;
    for (int ia = 0; ia < nA; ia++)
        for (int ib = 0; ib < nB; ib++) {
            const double *a = As + (size_t)ia * lda_s;
            const double *x = xs + (size_t)ib * ldx;
            DD t{0.0, 0.0};
            for (int i = lo; i < hi; i++) eft_dot2i(a[i], x[colind[i]], t);
            t = eft_quad_mul(1.0, t);
            pv[(size_t)(ia * nB2 + ib) * m] = t.x;
            pv[(size_t)(ia * nB2 + nB + ib) * m] = t.y;
        }
    int q = 0;
    for (int ik = 0; ik <= (nA - 1) + (nB2 - 1); ik++)
        for (int ia = 0; ia < nA; ia++) {
            const int ib = ik - ia;
            if (ib >= 0 && ib < nB2) terms[(size_t)(q++) * m] = pv[(size_t)(ia * nB2 + ib) * m];
        }
    double t = 0.0;
    if (sum_mode == 1)
        t = nearsum(q, terms, m);
    else
        for (int p = 0; p < q; p++) t += terms[(size_t)p * m];
    y[row] = fma(alpha, t, beta * y[row]);
}

// Plain FP64 CSRMV with a sequential fma chain (the true-residual check of CG).
__global__ void k_csrmv_plain(int m, const double *__restrict__ val, const int *__restrict__ colind,
                              const int *__restrict__ rowptr, const double *__restrict__ x, double alpha,
                              double beta, double *__restrict__ y) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    double tr = 0.0;
    for (int i = rowptr[row]; i < rowptr[row + 1]; i++) tr = fma(val[i], x[colind[i]], tr);
    y[row] = (beta == 0.0) ? alpha * tr : fma(alpha, tr, beta * y[row]);
}

// y = fma(alpha, x, y)  (src/cuda/cuozblas_axpy.cu:5-16)
__global__ void k_axpy(int n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride)
        y[i] = fma(alpha, x[i], y[i]);
}

// x = alpha * x  (the cublasDscal of src/cuda/cuozblas_cg.cu:100)
__global__ void k_scal(int n, double alpha, double *__restrict__ x) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) x[i] = alpha * x[i];
}

// Gather n elements of `esz` bytes spaced `stride` elements apart into a
// contiguous array (a one-row op(A) or one-column op(B) stored with a leading
// dimension above 1, e.g. B^T of a 1 x k B with ldb > 1).
template <typename E>
__global__ void k_gather_strided(int n, const E *__restrict__ src, int64_t stride, E *__restrict__ dst) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += step) dst[i] = src[i * stride];
}

struct Bytes16 {
    uint64_t lo, hi;
};

int gather_strided(cuozblasHandle_t *h, int n, const void *src, int64_t stride, int esz, void *dst) {
    if (n <= 0) return CUOZBLAS_STATUS_SUCCESS;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count() * 8) blocks = sm_count() * 8;
    cudaStream_t s = state(h)->stream;
    counted(h);
    if (esz == 4)
        k_gather_strided<float><<<blocks, 256, 0, s>>>(n, (const float *)src, stride, (float *)dst);
    else if (esz == 8)
        k_gather_strided<double><<<blocks, 256, 0, s>>>(n, (const double *)src, stride, (double *)dst);
    else if (esz == 16)
        k_gather_strided<Bytes16><<<blocks, 256, 0, s>>>(n, (const Bytes16 *)src, stride, (Bytes16 *)dst);
    else
        return CUOZBLAS_STATUS_INVALID_VALUE;
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

// Plain FP64 2-norm in a fixed order (the true residual of CG's diagnostics):
// 256 blocks of strided sums of squares, then one block adds the partials in
// order and writes sqrt to scratch[0] (partials at scratch[1..256]).
__global__ void __launch_bounds__(256) k_sumsq_partials(int n, const double *__restrict__ x,
                                                        double *__restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += (size_t)gridDim.x * blockDim.x)
        s = fma(x[i], x[i], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(256) k_sumsq_final(int nparts, const double *__restrict__ part,
                                                     double *__restrict__ out) {
    __shared__ double red[256];
    red[threadIdx.x] = (int)threadIdx.x < nparts ? part[threadIdx.x] : 0.0;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sqrt(red[0]);
}

int launch_nrm2_plain(cuozblasHandle_t *h, int n, const double *x, double *scratch) {
    constexpr int kParts = 256;
    cudaStream_t s = state(h)->stream;
    counted(h);
    k_sumsq_partials<<<kParts, 256, 0, s>>>(n > 0 ? n : 0, x, scratch + 1);
    counted(h);
    k_sumsq_final<<<1, 256, 0, s>>>(kParts, scratch + 1, scratch);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

int launch_axpy(cuozblasHandle_t *h, int n, double alpha, const double *x, double *y) {
    if (n <= 0) return CUOZBLAS_STATUS_SUCCESS;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count() * 16) blocks = sm_count() * 16;
    counted(h);
    k_axpy<<<blocks, 256, 0, state(h)->stream>>>(n, alpha, x, y);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

int launch_scal(cuozblasHandle_t *h, int n, double alpha, double *x) {
    if (n <= 0) return CUOZBLAS_STATUS_SUCCESS;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count() * 16) blocks = sm_count() * 16;
    counted(h);
    k_scal<<<blocks, 256, 0, state(h)->stream>>>(n, alpha, x);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

int launch_csrmv_plain(cuozblasHandle_t *h, int m, const double *val, const int *colind, const int *rowptr,
                       const double *x, double alpha, double beta, double *y) {
    if (m <= 0) return CUOZBLAS_STATUS_SUCCESS;
    counted(h);
    k_csrmv_plain<<<(m + 255) / 256, 256, 0, state(h)->stream>>>(m, val, colind, rowptr, x, alpha, beta, y);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

// Ozaki CSRMV over given A slices (nA slices of ld_s doubles).
int csrmv_presplit(cuozblasHandle_t *h, int m, int n, double alpha, const double *As, int nA, int64_t ld_s,
                   const int *colind, const int *rowptr, const double *x, double beta, double *y) {
    State *st = state(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    Arena ar(h);
    const int ldx = (n + 31) / 32 * 32;
    double *xs = ar.take<double>((uint64_t)maxS * (ldx > 0 ? ldx : 32));
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    int nB = 0;
    OZB_TRY(split_vector(h, n, x, rho_rule(n, h->splitEpsMode), maxS, xs, ldx, &nB));
    int maxlevel = (nA - 1) + (nB - 1);
    const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
    maxlevel = (maxlevel - h->fastMode) > mn ? (maxlevel - h->fastMode) : mn;
    int np = 0;
    for_each_pair(nA, nB, maxlevel, [&](int, int) { np++; });
    if (h->splitEpsMode == 2) {  // Dot2 (the caller admits fastMode 0 only)
        double *tbuf = ar.take<double>((uint64_t)4 * nA * nB * (m > 0 ? m : 1));
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        if (m > 0) {
            counted(h);
            k_csrmv_pairs_dot2<<<(m + 255) / 256, 256, 0, st->stream>>>(m, As, ld_s, colind, rowptr, xs, ldx, nA, nB,
                                                                       h->sumMode, alpha, beta, y, tbuf);
        }
        OZB_CHECK(cudaGetLastError());
        h->nSplitA = (float)nA;
        h->nSplitB = (float)nB;
        h->nSplitC = (float)(nA * nB);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    double *pbuf = nullptr;
    if (h->sumMode == 1) {
        pbuf = ar.take<double>((uint64_t)np * (m > 0 ? m : 1));
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    }
    if (m > 0) {
        counted(h);
        k_csrmv_pairs<<<(m + 255) / 256, 256, 0, st->stream>>>(m, As, ld_s, colind, rowptr, xs, ldx, nA, nB, maxlevel,
                                                              h->sumMode, alpha, beta, y, pbuf);
    }
    OZB_CHECK(cudaGetLastError());
    int ic = 0;
    for (int ia = 0; ia < (maxlevel + 1 < nA ? maxlevel + 1 : nA); ia++) ic += (nB < maxlevel + 1 - ia ? nB : maxlevel + 1 - ia);
    h->nSplitA = (float)nA;
    h->nSplitB = (float)nB;
    h->nSplitC = (float)ic;
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
