// gemm_f32.cu — the mixed form <double, float, float>: FP64 data, FP32 slices
// and FP32 slice products (src/cuda/cuozblas_gemm.cu:286, src/cpu/ozblas_gemm.cpp:3-315
// with TYPE2 = TYPE3 = float).
//
// The split (src/cpu/ozblas_split.cpp:181-221) cuts each line in FP64 with
// rho = ceil(53 - (24 - log2 k) / 2) and stores scalbn(slice, -tau) as FP32,
// tau = ceil(log2 max) of the level kept per line (src/cpu/ozblas_split.cpp:19-34).
// A slice then has at most 53 - rho significant bits, so a slice product over
// k terms has at most 24 and is exact in FP32 in any order: the FP32 SIMT
// pipe computes it, and the bits are fixed by the split and the order of the
// sum.  The sum is the reference's FSum for mixed types
// (src/cpu/ozblas_sum.cpp:382-432): t += scalbn((double)product, tauA + tauB)
// over the pairs in order (ik ascending, ia ascending).  The reference has no
// NearSum for mixed types (src/cpu/ozblas_sum.cpp:273-296 exits), so neither
// does this form.
#include <math.h>
#include <stdlib.h>

#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "sum.cuh"

namespace ozb {

// getRho<double, float> on the host, with the reference's own expression
// (src/cpu/ozblas_split.cpp:19-34, epse 53 and 24).
int rho_rule_f32(int dim, int splitEpsMode) {
    const double d = dim < 1 ? 1.0 : (double)dim;
    if (splitEpsMode == 9) return (int)ceil((53 - (24 - log2(2. * sqrt(d))) / 2));
    return (int)ceil((53 - (24 - log2(d)) / 2));
}

// ---------------------------------------------------------------------------
// General GEMM: every slice pair of a 128 x 128 output tile, fused with the
// ordered sum.  256 threads, 8 x 8 outputs each (rows ty*4+i and 64+ty*4+i,
// columns tx*4+j and 64+tx*4+j).  Operands are K-major FP32 slices (A slice
// ia: m lines x ldk, B slice ib: n lines x ldk, ldk % 16 == 0, zero padded);
// the (pair, k-tile) sequence is one register-prefetched, double-buffered
// pipeline, transposed into shared memory as [k][line].  At the last k-tile
// of a pair each thread adds its exact FP32 products, scaled by 2^(tauA +
// tauB), to its running FP64 sums, kept in shared memory (64 per thread).
// ---------------------------------------------------------------------------
constexpr int kFM = 128, kFN = 128, kFK = 16, kFLd = kFM + 4, kFThreads = 256;
constexpr size_t kFSumBytes = sizeof(double) * kFM * kFN;                 // 128 KB
constexpr size_t kFSmem = kFSumBytes + sizeof(float) * 2 * 2 * kFK * kFLd;  // + 2 operands x 2 stages

__global__ void __launch_bounds__(kFThreads, 1)
    k_gemm_pairs_f32(int m, int n, int ldk, const float *__restrict__ As, const float *__restrict__ Bs,
                     const short *__restrict__ Ea, const short *__restrict__ Eb, const int2 *__restrict__ pairs,
                     int np, double alpha, double beta, double *__restrict__ C, int ldc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *tsum = reinterpret_cast<double *>(smem_raw);  // [64][256]: element e of thread t at e*256 + t
    float *sA = reinterpret_cast<float *>(smem_raw + kFSumBytes);
    float *sB = sA + 2 * kFK * kFLd;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.x * kFM, n0 = blockIdx.y * kFN;
    const int lrow = tid >> 2, lk = (tid & 3) * 4;  // loader: lines lrow, lrow + 64; k lk..lk+3
    const int nkt = ldk / kFK;
    const int total = np * nkt;

#pragma unroll 8
    for (int e = 0; e < 64; e++) tsum[e * kFThreads + tid] = 0.0;

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

    float4 ra[2], rb[2];
    auto gload = [&](int q) {
        const int p = q / nkt, kt = q - p * nkt;
        const int2 pr = pairs[p];
        const float *a = As + (size_t)pr.x * m * ldk + kt * kFK + lk;
        const float *b = Bs + (size_t)pr.y * n * ldk + kt * kFK + lk;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = m0 + lrow + 64 * h, c = n0 + lrow + 64 * h;
            ra[h] = r < m ? __ldg(reinterpret_cast<const float4 *>(a + (size_t)r * ldk)) : make_float4(0, 0, 0, 0);
            rb[h] = c < n ? __ldg(reinterpret_cast<const float4 *>(b + (size_t)c * ldk)) : make_float4(0, 0, 0, 0);
        }
    };
    auto sstore = [&](int buf) {
        float *a = sA + buf * kFK * kFLd, *b = sB + buf * kFK * kFLd;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int l = lrow + 64 * h;
            a[(lk + 0) * kFLd + l] = ra[h].x;
            a[(lk + 1) * kFLd + l] = ra[h].y;
            a[(lk + 2) * kFLd + l] = ra[h].z;
            a[(lk + 3) * kFLd + l] = ra[h].w;
            b[(lk + 0) * kFLd + l] = rb[h].x;
            b[(lk + 1) * kFLd + l] = rb[h].y;
            b[(lk + 2) * kFLd + l] = rb[h].z;
            b[(lk + 3) * kFLd + l] = rb[h].w;
        }
    };

    gload(0);
    sstore(0);
    __syncthreads();
    for (int q = 0; q < total; q++) {
        const int buf = q & 1;
        if (q + 1 < total) gload(q + 1);
        const float *a = sA + buf * kFK * kFLd, *b = sB + buf * kFK * kFLd;
#pragma unroll
        for (int kk = 0; kk < kFK; kk++) {
            const float4 a0 = *reinterpret_cast<const float4 *>(a + kk * kFLd + ty * 4);
            const float4 a1 = *reinterpret_cast<const float4 *>(a + kk * kFLd + 64 + ty * 4);
            const float4 b0 = *reinterpret_cast<const float4 *>(b + kk * kFLd + tx * 4);
            const float4 b1 = *reinterpret_cast<const float4 *>(b + kk * kFLd + 64 + tx * 4);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (q % nkt == nkt - 1) {  // pair complete: scaled FP64 sum in pair order
            const int2 pr = pairs[q / nkt];
            int ea[8], eb[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
                const int c = n0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + i - 4);
                ea[i] = r < m ? Ea[(size_t)pr.x * m + r] : 0;
                eb[i] = c < n ? Eb[(size_t)pr.y * n + c] : 0;
            }
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    double &ts = tsum[(i * 8 + j) * kFThreads + tid];
                    ts = __dadd_rn(ts, scale2((double)acc[i][j], ea[i] + eb[j]));
                    acc[i][j] = 0.f;
                }
        }
        if (q + 1 < total) sstore(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
            if (c >= n) continue;
            double *cp = &C[(size_t)c * ldc + r];
            *cp = fma(alpha, tsum[(i * 8 + j) * kFThreads + tid], beta * *cp);
        }
    }
}

// ---------------------------------------------------------------------------
// Skinny forms.  Products of at most 8 x 8 slice pairs per launch, in FP32:
// every partial sum is an exact FP32 value, so the reduction order (and the
// atomic accumulation into P) does not change the bits.
// ---------------------------------------------------------------------------
// DOT: P[a * ldp + b] += sum_i xs[a][i] * ys[b][i] (P zeroed by the caller).
__global__ void __launch_bounds__(256) k_pair_dot_f32(int n, int nA, int nB, const float *__restrict__ xs, int ldx,
                                                      const float *__restrict__ ys, int ldy, float *__restrict__ P,
                                                      int ldp) {
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.f;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        float xa[8], yb[8];
#pragma unroll
        for (int a = 0; a < 8; a++) xa[a] = a < nA ? xs[(size_t)a * ldx + i] : 0.f;
#pragma unroll
        for (int b = 0; b < 8; b++) yb[b] = b < nB ? ys[(size_t)b * ldy + i] : 0.f;
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = fmaf(xa[a], yb[b], acc[a][b]);
    }
    __shared__ float red[8][8][8];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            float v = acc[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (l == 0) red[w][a][b] = v;
        }
    __syncthreads();
    if (threadIdx.x < 64) {
        const int a = threadIdx.x >> 3, b = threadIdx.x & 7;
        if (a < nA && b < nB) {
            float v = 0.f;
            for (int i = 0; i < 8; i++) v += red[i][a][b];
            atomicAdd(&P[a * ldp + b], v);
        }
    }
}

// GEMV: one warp per row; P[(ia*nBtot + ib) * ldp + row] = sum_k As[ia][row][k] * xs[ib][k].
__global__ void __launch_bounds__(256) k_pair_gemv_f32(int m, int k, int na, int nb, int ia0, int ib0, int nBtot,
                                                       const float *__restrict__ As, int ldk,
                                                       const float *__restrict__ xs, int ldx, float *__restrict__ P,
                                                       int64_t ldp) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= m) return;
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.f;
    for (int i = lane; i < k; i += 32) {
        float xa[8], yb[8];
#pragma unroll
        for (int a = 0; a < 8; a++) xa[a] = a < na ? As[((size_t)(ia0 + a) * m + row) * ldk + i] : 0.f;
#pragma unroll
        for (int b = 0; b < 8; b++) yb[b] = b < nb ? xs[(size_t)(ib0 + b) * ldx + i] : 0.f;
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = fmaf(xa[a], yb[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            float v = acc[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && a < na && b < nb) P[(size_t)((ia0 + a) * nBtot + (ib0 + b)) * ldp + row] = v;
        }
}

// Ordered sums of the skinny forms: t += scalbn((double)P, tauA + tauB), then
// fma(alpha, t, beta * y) (src/cpu/ozblas_sum.cpp:382-432).  Row exponents of
// A at Ea[ia * ldea + row]; the vector's at Eb[ib].
__global__ void k_sum_rows_f32(int m, int nA, int nB, int maxlevel, const float *__restrict__ P, int64_t ldp,
                               const short *__restrict__ Ea, int ldea, const short *__restrict__ Eb, double alpha,
                               double beta, double *__restrict__ y) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    double t = 0.0;
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) {
        t = __dadd_rn(t, scale2((double)P[(size_t)(ia * nB + ib) * ldp + row], Ea[(size_t)ia * ldea + row] + Eb[ib]));
    });
    y[row] = fma(alpha, t, beta * y[row]);
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
static int ceil_to(int v, int q) { return (v + q - 1) / q * q; }

// Split op(X) by lines of length k into FP32 slices (ns x nl x ldk) and
// exponents (ns x nl); X with strided lines is transposed first.
static int split_operand_f32(cuozblasHandle_t *h, bool lines_strided, int nl, int k, const double *X, int ldx,
                             int rho, int maxS, int ldk, float **slices, short **exps, int *ns, Arena &ar) {
    const double *src = X;
    int lds = ldx;
    if (lines_strided) {  // element (line l, i) at X[i * ldx + l]
        double *tmp = ar.take<double>((uint64_t)nl * (k > 0 ? k : 1));
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(transpose(h, nl, k, X, ldx, tmp, k));
        src = tmp;
        lds = k;
    }
    OZB_TRY(split_lines_count(h, k, nl, src, lds, rho, maxS, ns));
    *slices = ar.take<float>((uint64_t)(*ns) * nl * ldk);
    *exps = ar.take<short>((uint64_t)(*ns) * nl);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    return split_lines_write_f32(h, k, nl, src, lds, rho, *ns, *slices, ldk, *exps);
}

int gemm_f32_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                  const double *B, int ldb, double beta, double *C, int ldc, int fastMode) {
    State *st = state(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule_f32(k, h->splitEpsMode);
    Arena ar(h);
    const bool dot = (m == 1 && n == 1);
    const bool skinny_n = (n == 1);
    const int ldk = dot || skinny_n ? ceil_to(k > 0 ? k : 1, 4) : ceil_to(k > 0 ? k : 1, kFK);

    // rho >= 47 (k > 1024): every slice is an int8 times a power of two, and the
    // exact slice products run on the INT8 tensor cores (same bits)
    if (!dot && !skinny_n && rho >= 47 && !state(h)->env.ds_simt) {
        st->plain_timers = true;
        int nA = 0, nB = 0, np = 0;
        OZB_TRY(gemm_ds_i8_core(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, rho, fastMode, &nA, &nB,
                                &np));
        h->nSplitA = (float)nA;
        h->nSplitB = (float)nB;
        h->nSplitC = (float)np;
        h->mbk = m;
        h->nbk = n;
        return CUOZBLAS_STATUS_SUCCESS;
    }

    // ---- split ----  (phase events 0..4: start, A split, B split, products, sum)
    ev_record(h, 0);
    st->plain_timers = true;
    float *Sa = nullptr, *Sb = nullptr;
    short *Ea = nullptr, *Eb = nullptr;
    int nA = 0, nB = 0;
    if (dot) {
        Sa = ar.take<float>((uint64_t)maxS * ldk);
        Ea = ar.take<short>((uint64_t)maxS + 1);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(split_vector_f32(h, k, A, rho, maxS, Sa, ldk, Ea, &nA));
    } else {
        OZB_TRY(split_operand_f32(h, !is_trans(ta), m, k, A, lda, rho, maxS, ldk, &Sa, &Ea, &nA, ar));
    }
    ev_record(h, 1);
    if (skinny_n) {
        Sb = ar.take<float>((uint64_t)maxS * ldk);
        Eb = ar.take<short>((uint64_t)maxS + 1);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(split_vector_f32(h, k, B, rho, maxS, Sb, ldk, Eb, &nB));
    } else {
        OZB_TRY(split_operand_f32(h, is_trans(tb), n, k, B, ldb, rho, maxS, ldk, &Sb, &Eb, &nB, ar));
    }
    ev_record(h, 2);
    const int fast = dot ? 0 : fastMode;
    int maxlevel = (nA - 1) + (nB - 1);
    {
        const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
        maxlevel = (maxlevel - fast) > mn ? (maxlevel - fast) : mn;  // src/cpu/ozblas_gemm.cpp:163-164
    }
    int np = 0;
    for_each_pair(nA, nB, maxlevel, [&](int, int) { np++; });
    h->nSplitA = (float)nA;
    h->nSplitB = (float)nB;
    h->nSplitC = dot ? 1.f : (skinny_n && fast == 0 ? (float)(maxlevel + 1 < nA ? maxlevel + 1 : nA) : (float)np);
    h->mbk = m;
    h->nbk = n;

    if (dot || skinny_n) {
        const int rows = dot ? 1 : m;
        const int64_t ldp = rows;
        float *P = ar.take<float>((uint64_t)nA * nB * ldp);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        if (dot) OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(float) * nA * nB, st->stream));
        for (int ia0 = 0; ia0 < nA; ia0 += 8)
            for (int ib0 = 0; ib0 < nB; ib0 += 8) {
                const int na = nA - ia0 < 8 ? nA - ia0 : 8, nb = nB - ib0 < 8 ? nB - ib0 : 8;
                counted(h);
                if (dot) {
                    int blocks = (k + 255) / 256;
                    if (blocks > sm_count() * 8) blocks = sm_count() * 8;
                    if (blocks < 1) blocks = 1;
                    k_pair_dot_f32<<<blocks, 256, 0, st->stream>>>(k, na, nb, Sa + (size_t)ia0 * ldk, ldk,
                                                                   Sb + (size_t)ib0 * ldk, ldk, P + ia0 * nB + ib0,
                                                                   nB);
                } else {
                    const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
                    k_pair_gemv_f32<<<blocks, 256, 0, st->stream>>>(m, k, na, nb, ia0, ib0, nB, Sa, ldk, Sb, ldk, P,
                                                                    ldp);
                }
                OZB_CHECK(cudaGetLastError());
            }
        ev_record(h, 3);
        counted(h);
        k_sum_rows_f32<<<(rows + 127) / 128, 128, 0, st->stream>>>(rows, nA, nB, maxlevel, P, ldp, Ea, rows, Eb,
                                                                   alpha, beta, C);
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 4);
        return CUOZBLAS_STATUS_SUCCESS;
    }

    // ---- general GEMM ----
    int2 *hp = new int2[np > 0 ? np : 1];
    int q = 0;
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { hp[q++] = make_int2(ia, ib); });
    int2 *dp = ar.take<int2>(np > 0 ? np : 1);
    if (!ar.ok) {
        delete[] hp;
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    cudaError_t ce = cudaMemcpyAsync(dp, hp, sizeof(int2) * np, cudaMemcpyHostToDevice, st->stream);
    cudaError_t ce2 = cudaStreamSynchronize(st->stream);
    delete[] hp;
    OZB_CHECK(ce);
    OZB_CHECK(ce2);
    OZB_CHECK(cudaFuncSetAttribute(k_gemm_pairs_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFSmem));
    dim3 grid((m + kFM - 1) / kFM, (n + kFN - 1) / kFN);
    counted(h);
    k_gemm_pairs_f32<<<grid, kFThreads, kFSmem, st->stream>>>(m, n, ldk, Sa, Sb, Ea, Eb, dp, np, alpha, beta, C, ldc);
    OZB_CHECK(cudaGetLastError());
    ev_record(h, 3);  // the ordered sum runs inside the product kernel here
    ev_record(h, 4);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
