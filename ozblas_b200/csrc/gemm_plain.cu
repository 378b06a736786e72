// gemm_plain.cu — the plain (FP64-slice) Ozaki GEMM and the skinny forms it
// serves (GEMV, DOT), src/cuda/cuozblas_gemm.cu:7-284 / src/cpu/ozblas_gemm.cpp:3-315.
//
// Slices are exact: a slice of a line of length k carries at most 53 - rho
// significant bits on a common grid, rho = ceil(53 - (53 - log2 k)/2), so
// any sum of k slice products is exact in FP64 (src/cuda/cuozblas_split.cu:51-67).
// The product of one slice pair is therefore the same in any order or
// association, which lets the FP64 tensor pipe (DMMA) compute it.  What
// fixes the bits is (1) the split and (2) the order of the pair sum, which
// the fused epilogue follows exactly.
#include <stdlib.h>

#include <vector>

#include "ozb_internal.h"
#include "eft.cuh"
#include "sum.cuh"

namespace ozb {

// ---------------------------------------------------------------------------
// DMMA tile kernel.  CTA tile 64x64, k-tile 16, 4 warps (2x2), warp tile
// 32x32 = 4x4 mma.m8n8k4.f64 fragments.  Operands are K-major slices:
// A slice ia: m lines x ldk, B slice ib: n lines x ldk (ldk % 16 == 0, zero
// padded).  The (pair, k-tile) sequence is one software pipeline; at each
// pair boundary the exact pair product is added to the running FP64 sum in
// summation order (FSUM) or stored to the pair buffer (STORE).
// ---------------------------------------------------------------------------
constexpr int kBM = 64, kBN = 64, kBK = 16, kLds = kBK + 4;  // row stride 20 doubles: conflict-free fragments

struct PairList {
    const int2 *pairs;  // (ia, ib) in summation order
    int np;
};

__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// SD: the mixed form <float, double, double>.  At each pair boundary the
// exact product is rounded to float, scaled by 2^(tauA + tauB) in float
// ((float)scalbn, one rounding) and added to a float sum; the output is
// (float)fma(alpha, t, beta * C) computed in double, as the reference's float
// helpers do (src/cpu/ozblas_sum.cpp:382-432, src/cpu/ozblas_aux.cpp:3-35).
template <bool STORE, bool SD>
__global__ void __launch_bounds__(128) k_gemm_pairs_dmma(int m, int n, int nlB, int ldk, const double *__restrict__ As,
                                                         const double *__restrict__ Bs, const int2 *__restrict__ pairs,
                                                         int np, double alpha, double beta, double *__restrict__ C,
                                                         int ldc, double *__restrict__ pbuf,
                                                         const short *__restrict__ Ea, const short *__restrict__ Eb,
                                                         float *__restrict__ Cf) {
    __shared__ __align__(16) double sA[2][kBM][kLds];
    __shared__ __align__(16) double sB[2][kBN][kLds];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int nkt = ldk / kBK;
    const int total = np * nkt;

    double acc[4][4][2], t[4][4][2];
    float tf[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            acc[i][j][0] = acc[i][j][1] = 0.0;
            t[i][j][0] = t[i][j][1] = 0.0;
            tf[i][j][0] = tf[i][j][1] = 0.f;
        }

    // each thread copies 4 x 16B of A and of B per k-tile (64 lines x 8 chunks)
    auto load_tile = [&](int step, int buf) {
        const int p = step / nkt, kt = step - p * nkt;
        const int2 pr = pairs[p];
        const double *a = As + ((size_t)pr.x * m) * ldk + (size_t)kt * kBK;
        const double *b = Bs + ((size_t)pr.y * nlB) * ldk + (size_t)kt * kBK;  // nlB: lines per B slice
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int idx = tid + c * 128;  // 0..511
            const int row = idx >> 3, ch = idx & 7;
            const int gr = m0 + row, gc = n0 + row;
            cp_async16(&sA[buf][row][ch * 2], a + (size_t)(gr < m ? gr : 0) * ldk + ch * 2, gr < m);
            cp_async16(&sB[buf][row][ch * 2], b + (size_t)(gc < n ? gc : 0) * ldk + ch * 2, gc < n);
        }
    };

    if (total > 0) load_tile(0, 0);
    cp_async_commit();
    for (int step = 0; step < total; step++) {
        const int buf = step & 1;
        if (step + 1 < total) load_tile(step + 1, buf ^ 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; i++) af[i] = sA[buf][wm * 32 + i * 8 + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
            for (int j = 0; j < 4; j++) bf[j] = sB[buf][wn * 32 + j * 8 + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
        const int p = step / nkt;
        if (step - p * nkt == nkt - 1) {  // pair complete: acc is the exact product of pair p
            if (SD) {
                const int2 pr = pairs[p];
                int ea[4], eb[8];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
                    ea[i] = r < m ? Ea[(size_t)pr.x * m + r] : 0;
                }
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int c = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + h;
                        eb[j * 2 + h] = c < n ? Eb[(size_t)pr.y * nlB + c] : 0;
                    }
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const float c32 = __double2float_rn(acc[i][j][h]);
                            tf[i][j][h] = __fadd_rn(tf[i][j][h],
                                                    __double2float_rn(scale2((double)c32, ea[i] + eb[j * 2 + h])));
                            acc[i][j][h] = 0.0;
                        }
            } else if (STORE) {
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
                            const int c = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + h;
                            if (r < m && c < n) pbuf[((size_t)p * n + c) * m + r] = acc[i][j][h];
                            acc[i][j][h] = 0.0;
                        }
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            t[i][j][h] += acc[i][j][h];
                            acc[i][j][h] = 0.0;
                        }
            }
        }
    }
    if (SD) {
        const float af = (float)alpha, bf = (float)beta;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
                    const int c = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + h;
                    if (r < m && c < n) {
                        float *cp = &Cf[(size_t)c * ldc + r];
                        *cp = __double2float_rn(fma((double)af, (double)tf[i][j][h], (double)__fmul_rn(bf, *cp)));
                    }
                }
    } else if (!STORE) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
                    const int c = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + h;
                    if (r < m && c < n) {
                        double *cp = &C[(size_t)c * ldc + r];
                        *cp = fma(alpha, t[i][j][h], beta * *cp);
                    }
                }
    }
}

// Sum a pair buffer (pair p of np at pbuf + p*ld_pair, element e at + e) in
// summation order; output element e (row e % m, column e / m) of C.
__global__ void k_sum_pairs(int m, int64_t count, int np, const double *__restrict__ pbuf_c, int64_t ld_pair,
                            int sum_mode, double alpha, double beta, double *__restrict__ C, int ldc) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    double *pbuf = const_cast<double *>(pbuf_c);
    double t = 0.0;
    if (sum_mode == 1) {
        t = nearsum(np, pbuf + e, ld_pair);
    } else {
        for (int p = 0; p < np; p++) t += pbuf[p * ld_pair + e];
    }
    const int64_t r = e % m, c = e / m;
    double *cp = &C[c * ldc + r];
    *cp = fma(alpha, t, beta * *cp);
}

// ---------------------------------------------------------------------------
// Skinny products: P[ia][ib] over n elements for slice vectors (DOT) —
// at most 8 x 8 pairs per launch, exact, so atomic accumulation order does
// not change the bits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_pair_dot(int n, int nA, int nB, const double *__restrict__ xs, int ldx,
                                                  const double *__restrict__ ys, int ldy, double *__restrict__ P,
                                                  int ldp) {
    double acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        double xa[8], yb[8];
#pragma unroll
        for (int a = 0; a < 8; a++) xa[a] = a < nA ? xs[(size_t)a * ldx + i] : 0.0;
#pragma unroll
        for (int b = 0; b < 8; b++) yb[b] = b < nB ? ys[(size_t)b * ldy + i] : 0.0;
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
    }
    __shared__ double red[8][8][8];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            double v = acc[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (l == 0) red[w][a][b] = v;
        }
    __syncthreads();
    if (threadIdx.x < 64) {
        const int a = threadIdx.x >> 3, b = threadIdx.x & 7;
        if (a < nA && b < nB) {
            double v = 0.0;
            for (int i = 0; i < 8; i++) v += red[i][a][b];
            atomicAdd(&P[a * ldp + b], v);
        }
    }
}

// Dot2 DOT (splitEpsMode 2): the reference forms each pair with Dot2i over
// all k and combines per-thread partials with QuadAdd in OpenMP
// critical-section order (src/cpu/ozblas_blas_wrapper.cpp:109-152), so its bits
// depend on its thread count.  Here the order is fixed: every thread runs
// Dot2i over a strided share, a block combines its threads with QuadAdd in a
// fixed tree, and one thread per pair combines the blocks in block order;
// then QuadAdd onto (0, 0) and QuadMul(1), as the reference finishes.
// Grid (blocks, nA * nB); partials[pair * gridDim.x + block].
__global__ void __launch_bounds__(256) k_pair_dot2(int k, int nB, const double *__restrict__ xs, int ldx,
                                                   const double *__restrict__ ys, int ldy, DD *__restrict__ partials) {
    __shared__ DD red[256];
    const int pair = blockIdx.y, ia = pair / nB, ib = pair % nB;
    const double *x = xs + (size_t)ia * ldx, *y = ys + (size_t)ib * ldy;
    DD c{0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < k; i += (int64_t)gridDim.x * 256)
        eft_dot2i(x[i], y[i], c);
    red[threadIdx.x] = c;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = eft_quad_add(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[(size_t)pair * gridDim.x + blockIdx.x] = red[0];
}

// The pairs' hi terms at B index ib and lo terms at nB + ib, summed over
// levels (nA - 1) + (2 nB - 1) (src/cpu/ozblas_gemm.cpp:281-287); one block.
__global__ void k_dot2_finish(int nA, int nB, int blocks, const DD *__restrict__ partials, int sum_mode,
                              double alpha, double beta, double *__restrict__ out, double *__restrict__ tmp) {
    const int nB2 = 2 * nB, np = nA * nB;
    for (int pair = threadIdx.x; pair < np; pair += blockDim.x) {
        DD g{0.0, 0.0};
        for (int b = 0; b < blocks; b++) g = eft_quad_add(g, partials[(size_t)pair * blocks + b]);
        g = eft_quad_add(DD{0.0, 0.0}, g);
        g = eft_quad_mul(1.0, g);
        const int ia = pair / nB, ib = pair % nB;
        tmp[ia * nB2 + ib] = g.x;
        tmp[ia * nB2 + nB + ib] = g.y;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double *terms = tmp + nA * nB2;
    int q = 0;
    for (int ik = 0; ik <= (nA - 1) + (nB2 - 1); ik++)
        for (int ia = 0; ia < nA; ia++) {
            const int ib = ik - ia;
            if (ib >= 0 && ib < nB2) terms[q++] = tmp[ia * nB2 + ib];
        }
    double t = 0.0;
    if (sum_mode == 1)
        t = nearsum(q, terms, 1);
    else
        for (int p = 0; p < q; p++) t += terms[p];
    *out = fma(alpha, t, beta * *out);
}

// One scalar result from a pair matrix P[ia * ldp + ib] (DOT): FSum or NearSum.
__global__ void k_sum_pair_matrix(int nA, int nB, int maxlevel, const double *__restrict__ P, int ldp, int sum_mode,
                                  double alpha, double beta, double *__restrict__ out, double *__restrict__ tmp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    if (sum_mode == 1) {
        int np = 0;
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { tmp[np++] = P[ia * ldp + ib]; });
        t = nearsum(np, tmp, 1);
    } else {
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { t += P[ia * ldp + ib]; });
    }
    *out = fma(alpha, t, beta * *out);
}

// GEMV pairs: one warp per row i; P[p][i] = sum_k As[ia][i][k] * xs[ib][k]
// for the pairs given (at most 8 x 8 block per launch).  Exact.
__global__ void __launch_bounds__(256) k_pair_gemv(int m, int k, int na, int nb, int ia0, int ib0, int nBtot,
                                                   const double *__restrict__ As, int ldk,
                                                   const double *__restrict__ xs, int ldx, double *__restrict__ P,
                                                   int64_t ldp) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= m) return;
    double acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.0;
    for (int i = lane; i < k; i += 32) {
        double xa[8], yb[8];
#pragma unroll
        for (int a = 0; a < 8; a++) xa[a] = a < na ? As[((size_t)(ia0 + a) * m + row) * ldk + i] : 0.0;
#pragma unroll
        for (int b = 0; b < 8; b++) yb[b] = b < nb ? xs[(size_t)(ib0 + b) * ldx + i] : 0.0;
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) {
            double v = acc[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && a < na && b < nb) P[(size_t)((ia0 + a) * nBtot + (ib0 + b)) * ldp + row] = v;
        }
}

// Sum a per-row pair buffer P[(ia*nB+ib)*ldp + row] in order; y = fma(alpha, t, beta*y).
// NearSum gathers the terms in summation order into `scratch` (np x ldp).
__global__ void k_sum_rows(int m, int nA, int nB, int maxlevel, double *__restrict__ P, int64_t ldp, int sum_mode,
                           double alpha, double beta, double *__restrict__ y, double *__restrict__ scratch) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    double t = 0.0;
    if (sum_mode == 1) {
        int np = 0;
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) {
            scratch[(size_t)np * ldp + row] = P[(size_t)(ia * nB + ib) * ldp + row];
            np++;
        });
        t = nearsum(np, scratch + row, ldp);
    } else {
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { t += P[(size_t)(ia * nB + ib) * ldp + row]; });
    }
    y[row] = fma(alpha, t, beta * y[row]);
}

// The ordered sum of a per-row pair buffer (the skinny forms), with the handle's sum mode.
int sum_rows_launch(cuozblasHandle_t *h, int m, int nA, int nB, int maxlevel, double *P, int64_t ldp, double alpha,
                    double beta, double *y, double *scratch) {
    counted(h);
    k_sum_rows<<<(m + 127) / 128, 128, 0, state(h)->stream>>>(m, nA, nB, maxlevel, P, ldp, h->sumMode, alpha, beta, y,
                                                               scratch);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Host drivers
// ---------------------------------------------------------------------------
static int ceil_to(int v, int q) { return (v + q - 1) / q * q; }

// Split op(A) by rows (lines of length k) into ns slices of m x ldk.  If A is
// 'n' (m x k, column-major) it is first transposed so every line is contiguous.
static int split_operand(cuozblasHandle_t *h, bool lines_strided, int nl, int k, const double *X, int ldx, int rho,
                         int maxS, int ldk, double **slices, int *ns, Arena &ar, short **exps = nullptr) {
    const double *src = X;
    int lds = ldx;
    double *tmp = nullptr;
    const uint64_t mk = ar.mark();
    if (lines_strided) {  // element (line l, i) at X[i * ldx + l]
        tmp = ar.take<double>((uint64_t)nl * (k > 0 ? k : 1));
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(transpose(h, nl, k, X, ldx, tmp, k));
        src = tmp;
        lds = k;
    }
    OZB_TRY(split_lines_count(h, k, nl, src, lds, rho, maxS, ns));
    // slices go below the temporary so the temporary can be released after
    double *out;
    if (tmp) {
        // place the slices after the transposed copy, then compact is unnecessary:
        out = ar.take<double>((uint64_t)(*ns) * nl * ldk);
    } else {
        out = ar.take<double>((uint64_t)(*ns) * nl * ldk);
    }
    if (exps) *exps = ar.take<short>((uint64_t)(*ns) * (nl > 0 ? nl : 1));
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    if (exps)
        OZB_TRY(split_lines_write_e(h, k, nl, src, lds, rho, *ns, out, ldk, *exps));
    else
        OZB_TRY(split_lines_write(h, k, nl, src, lds, rho, *ns, out, ldk));
    (void)mk;
    *slices = out;
    return CUOZBLAS_STATUS_SUCCESS;
}

__global__ void k_slices_to_digits(int ns, int nl, int k, int ldk, const double *__restrict__ S, int scale,
                                   const short *__restrict__ exps, int D, int lines_pad, int k_pad,
                                   int8_t *__restrict__ dig);  // below

int gemm_plain_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta, double *C, int ldc, int fastMode) {
    State *st = state(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(k, h->splitEpsMode);
    Arena ar(h);
    const bool dot = (m == 1 && n == 1);
    const bool skinny_n = (n == 1);
    const int ldk = dot || skinny_n ? ceil_to(k > 0 ? k : 1, 2) : ceil_to(k > 0 ? k : 1, kBK);

    // ---- split ----  (phase events 0..4: start, A split, B split, products, sum)
    ev_record(h, 0);
    st->plain_timers = true;
    // GEMV 'n' with NearSum: correctly rounded exact row dots, A read once
    if (skinny_n && !dot && !is_trans(ta) && h->sumMode == 1 && fastMode == 0 && h->splitEpsMode == 0 &&
        !state(h)->env.gemv_split && !state(h)->env.gemv_slices) {
        bool done = false;
        int nAv = 0, nBv = 0;
        OZB_TRY(gemv_rn_n(h, m, k, A, lda, B, alpha, beta, C, &done, &nAv, &nBv));
        if (done) {
            const int ml = (nAv - 1) + (nBv - 1);
            h->nSplitA = (float)nAv;
            h->nSplitB = (float)nBv;
            h->nSplitC = (float)(ml + 1 < nAv ? ml + 1 : nAv);
            h->mbk = m;
            h->nbk = n;
            return CUOZBLAS_STATUS_SUCCESS;  // gemv_rn_n recorded the span of its kernels (t_comp)
        }
        ev_record(h, 0);
    }
    // GEMV 'n' (rows of A strided): fused split and products, A read nA + 2 times
    if (skinny_n && !dot && !is_trans(ta) && !state(h)->env.gemv_split) {
        const uint64_t mk0 = ar.mark();
        double *xs = ar.take<double>((uint64_t)maxS * ldk);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        int nBv = 0, nAv = 0;
        span_begin(h);  // t_comp: the device span of the vector split and the fused kernels
        OZB_TRY(split_vector(h, k, B, rho, maxS, xs, ldk, &nBv));
        const int fr = gemv_fused_n(h, m, k, A, lda, xs, ldk, nBv, rho, maxS, fastMode, alpha, beta, C, &nAv);
        if (fr == CUOZBLAS_STATUS_SUCCESS) {
            int ml = (nAv - 1) + (nBv - 1);
            const int mn = nAv - 1 < nBv - 1 ? nAv - 1 : nBv - 1;
            ml = (ml - fastMode) > mn ? (ml - fastMode) : mn;
            h->nSplitA = (float)nAv;
            h->nSplitB = (float)nBv;
            h->nSplitC = fastMode == 0 ? (float)(ml + 1 < nAv ? ml + 1 : nAv) : 0.f;
            if (fastMode != 0) {
                int np = 0;
                for_each_pair(nAv, nBv, ml, [&](int, int) { np++; });
                h->nSplitC = (float)np;
            }
            h->mbk = m;
            h->nbk = n;
            span_end(h);
            return CUOZBLAS_STATUS_SUCCESS;
        }
        if (fr != CUOZBLAS_STATUS_NOT_SUPPORTED) return fr;
        ar.release(mk0);  // more levels than the fused kernel holds: the materialised path
        ev_record(h, 0);
    }
    double *Sa = nullptr, *Sb = nullptr;
    short *Ea = nullptr, *Eb = nullptr;  // taus per line and level (general GEMM: the INT8 product path)
    int nA = 0, nB = 0;
    if (dot) {
        Sa = ar.take<double>((uint64_t)maxS * ldk);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(split_vector(h, k, A, rho, maxS, Sa, ldk, &nA));
    } else {
        // lines of op(A): 'n' -> row i of A is strided by lda
        OZB_TRY(split_operand(h, !is_trans(ta), m, k, A, lda, rho, maxS, ldk, &Sa, &nA, ar, skinny_n ? nullptr : &Ea));
    }
    ev_record(h, 1);
    if (skinny_n) {
        Sb = ar.take<double>((uint64_t)maxS * ldk);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(split_vector(h, k, B, rho, maxS, Sb, ldk, &nB));
    } else {
        OZB_TRY(split_operand(h, is_trans(tb), n, k, B, ldb, rho, maxS, ldk, &Sb, &nB, ar, &Eb));
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

    if (dot && h->splitEpsMode == 2) {  // Dot2 DOT (the caller admits fastMode 0 only)
        int blocks = (k + 255) / 256;
        if (blocks > sm_count() * 4) blocks = sm_count() * 4;
        if (blocks < 1) blocks = 1;
        DD *partials = ar.take<DD>((uint64_t)nA * nB * blocks);
        double *tmp = ar.take<double>((uint64_t)4 * nA * nB + 1);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        counted(h);
        k_pair_dot2<<<dim3(blocks, nA * nB), 256, 0, st->stream>>>(k, nB, Sa, ldk, Sb, ldk, partials);
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 3);
        counted(h);
        k_dot2_finish<<<1, 64, 0, st->stream>>>(nA, nB, blocks, partials, h->sumMode, alpha, beta, C, tmp);
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 4);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    if (dot || skinny_n) {
        // pair products into P[(ia*nB+ib)][row]
        const int rows = dot ? 1 : m;
        const int64_t ldp = rows;
        double *P = ar.take<double>((uint64_t)nA * nB * ldp);
        double *scr = ar.take<double>((uint64_t)nA * nB * ldp + 1);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(double) * nA * nB * ldp, st->stream));
        for (int ia0 = 0; ia0 < nA; ia0 += 8)
            for (int ib0 = 0; ib0 < nB; ib0 += 8) {
                const int na = nA - ia0 < 8 ? nA - ia0 : 8, nb = nB - ib0 < 8 ? nB - ib0 : 8;
                if (dot) {
                    // P block at (ia0, ib0) with row stride nB
                    int blocks = (k + 255) / 256;
                    if (blocks > sm_count() * 8) blocks = sm_count() * 8;
                    if (blocks < 1) blocks = 1;
                    counted(h);
                    k_pair_dot<<<blocks, 256, 0, st->stream>>>(k, na, nb, Sa + (size_t)ia0 * ldk, ldk,
                                                               Sb + (size_t)ib0 * ldk, ldk, P + ia0 * nB + ib0, nB);
                } else {
                    const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
                    counted(h);
                    k_pair_gemv<<<blocks, 256, 0, st->stream>>>(m, k, na, nb, ia0, ib0, nB, Sa, ldk, Sb, ldk, P,
                                                                ldp);
                }
                OZB_CHECK(cudaGetLastError());
            }
        ev_record(h, 3);
        if (dot) {
            counted(h);
            k_sum_pair_matrix<<<1, 32, 0, st->stream>>>(nA, nB, maxlevel, P, nB, h->sumMode, alpha, beta, C, scr);
        } else {
            counted(h);
            k_sum_rows<<<(m + 127) / 128, 128, 0, st->stream>>>(m, nA, nB, maxlevel, P, ldp, h->sumMode, alpha, beta,
                                                              C, scr);
        }
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 4);
        return CUOZBLAS_STATUS_SUCCESS;
    }

    // ---- general GEMM ----
    // Pair products on the INT8 tensor cores: a slice is q 2^(rho + tau - 53)
    // with an integer |q| <= 2^(53 - rho) < 2^(7 D), cut into D <= 4 int8 digits;
    // the kernel stores the exact FP64 pair products (the DMMA kernel's values)
    // and the ordered sum (FSum or NearSum) reads them as before.
    {
        const int D = (53 - rho + 1 + 6) / 7;
        const int k_pad = (k + 127) / 128 * 128;
        const int lpadA = (m + 127) / 128 * 128, lpadB = (n + 127) / 128 * 128;
        const uint64_t need = (uint64_t)nA * D * lpadA * k_pad + (uint64_t)nB * D * lpadB * k_pad +
                              sizeof(double) * (uint64_t)np * m * n + (1u << 20);
        const uint64_t avail = h->workSizeBytes - ((ar.mark() + 255) / 256 * 256);
        if (Ea && Eb && D <= 4 && (double)D * k * 127.0 * 127.0 < 2147483647.0 && need < avail &&
            !state(h)->env.plain_dmma) {
            std::vector<int2> pl;
            for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { pl.push_back(make_int2(ia, ib)); });
            int8_t *dg[2];
            for (int o = 0; o < 2; o++) {
                const int nl = o == 0 ? m : n, ns = o == 0 ? nA : nB, lpad = o == 0 ? lpadA : lpadB;
                dg[o] = ar.take<int8_t>((uint64_t)ns * D * lpad * k_pad);
                if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
                OZB_CHECK(cudaMemsetAsync(dg[o], 0, (size_t)ns * D * lpad * k_pad, st->stream));
                const int64_t total = (int64_t)ns * nl * k;
                int blocks = (int)((total + 255) / 256);
                if (blocks > sm_count() * 16) blocks = sm_count() * 16;
                if (blocks < 1) blocks = 1;
                counted(h);
                k_slices_to_digits<<<blocks, 256, 0, st->stream>>>(ns, nl, k, ldk, o == 0 ? Sa : Sb, 53 - rho,
                                                                  o == 0 ? Ea : Eb, D, lpad, k_pad, dg[o]);
                OZB_CHECK(cudaGetLastError());
            }
            double *pbuf = ar.take<double>((uint64_t)np * m * n);
            if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
            OZB_TRY(i8_exact_pairs(h, m, n, k_pad, dg[0], lpadA, nA * D, dg[1], lpadB, nB * D, D, pl, 2 * (rho - 53),
                                   Ea, Eb, pbuf));
            ev_record(h, 3);
            const int64_t count = (int64_t)m * n;
            counted(h);
            k_sum_pairs<<<(unsigned)((count + 255) / 256), 256, 0, st->stream>>>(m, count, np, pbuf, count,
                                                                                h->sumMode, alpha, beta, C, ldc);
            OZB_CHECK(cudaGetLastError());
            ev_record(h, 4);
            return CUOZBLAS_STATUS_SUCCESS;
        }
    }
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
    dim3 grid((m + kBM - 1) / kBM, (n + kBN - 1) / kBN);
    if (h->sumMode == 1) {
        // pair products to a buffer, blocked over columns if the arena is short
        const uint64_t avail = h->workSizeBytes - ((ar.mark() + 255) / 256 * 256);
        int64_t ncols = (int64_t)(avail / (sizeof(double) * (uint64_t)np * (uint64_t)m));
        if (ncols >= n) {
            ncols = n;
        } else {
            ncols = ncols / kBN * kBN;
            if (ncols == 0) return CUOZBLAS_STATUS_WORKSPACE;
        }
        double *pbuf = ar.take<double>((uint64_t)np * m * ncols);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        for (int64_t c0 = 0; c0 < n; c0 += ncols) {
            const int nc = (int)((n - c0) < ncols ? (n - c0) : ncols);
            dim3 g((m + kBM - 1) / kBM, (nc + kBN - 1) / kBN);
            counted(h);
            k_gemm_pairs_dmma<true, false><<<g, 128, 0, st->stream>>>(m, nc, n, ldk, Sa, Sb + (size_t)c0 * ldk, dp,
                                                                      np, alpha, beta, C, ldc, pbuf, nullptr,
                                                                      nullptr, nullptr);
            OZB_CHECK(cudaGetLastError());
            const int64_t count = (int64_t)m * nc;
            counted(h);
            k_sum_pairs<<<(unsigned)((count + 255) / 256), 256, 0, st->stream>>>(
                m, count, np, pbuf, count, 1, alpha, beta, C + (size_t)c0 * ldc, ldc);
            OZB_CHECK(cudaGetLastError());
        }
    } else {
        counted(h);
        k_gemm_pairs_dmma<false, false><<<grid, 128, 0, st->stream>>>(m, n, n, ldk, Sa, Sb, dp, np, alpha, beta, C,
                                                                      ldc, nullptr, nullptr, nullptr, nullptr);
        OZB_CHECK(cudaGetLastError());
    }
    ev_record(h, 3);  // the ordered sum runs inside the product kernels here
    ev_record(h, 4);
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Exact FP64 pair products for other sums (the quad form): every pair of the
// list to pbuf[p][col][row] for columns c0 .. c0 + nc of B's n lines, and the
// skinny forms' pair matrices P[(ia * nB + ib) * ldp + row].
// ---------------------------------------------------------------------------
int gemm_pairs_store(cuozblasHandle_t *h, int m, int nc, int nlB, int ldk, const double *Sa, const double *Sb,
                     const int2 *dp, int np, double *pbuf) {
    State *st = state(h);
    dim3 g((m + kBM - 1) / kBM, (nc + kBN - 1) / kBN);
    counted(h);
    k_gemm_pairs_dmma<true, false><<<g, 128, 0, st->stream>>>(m, nc, nlB, ldk, Sa, Sb, dp, np, 0.0, 0.0, nullptr,
                                                              1, pbuf, nullptr, nullptr, nullptr);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

int pair_products_skinny(cuozblasHandle_t *h, bool dot, int m, int k, int nA, int nB, const double *Sa,
                         const double *Sb, int ldk, double *P) {
    State *st = state(h);
    const int64_t ldp = dot ? 1 : m;
    if (dot) OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(double) * nA * nB, st->stream));
    for (int ia0 = 0; ia0 < nA; ia0 += 8)
        for (int ib0 = 0; ib0 < nB; ib0 += 8) {
            const int na = nA - ia0 < 8 ? nA - ia0 : 8, nb = nB - ib0 < 8 ? nB - ib0 : 8;
            counted(h);
            if (dot) {
                int blocks = (k + 255) / 256;
                if (blocks > sm_count() * 8) blocks = sm_count() * 8;
                if (blocks < 1) blocks = 1;
                k_pair_dot<<<blocks, 256, 0, st->stream>>>(k, na, nb, Sa + (size_t)ia0 * ldk, ldk,
                                                           Sb + (size_t)ib0 * ldk, ldk, P + ia0 * nB + ib0, nB);
            } else {
                const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
                k_pair_gemv<<<blocks, 256, 0, st->stream>>>(m, k, na, nb, ia0, ib0, nB, Sa, ldk, Sb, ldk, P, ldp);
            }
            OZB_CHECK(cudaGetLastError());
        }
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Mixed form <float, double, double> (src/cpu/ozblas_gemm.cpp:3-315 with
// TYPE1 = float): float data split in float arithmetic into FP64 slices
// (split_lines_*_sd), exact FP64 slice products on the DMMA / skinny kernels
// above, and the float-scaled ordered sum.
// ---------------------------------------------------------------------------
// getRho<float, double> on the host with the reference's own expression
// (src/cpu/ozblas_split.cpp:19-34, epse 24 and 53); negative below k = 32.
int rho_rule_sd(int dim, int splitEpsMode) {
    const double d = dim < 1 ? 1.0 : (double)dim;
    if (splitEpsMode == 9) return (int)ceil((24 - (53 - log2(2. * sqrt(d))) / 2));
    return (int)ceil((24 - (53 - log2(d)) / 2));
}

// Ordered float sum of the skinny forms: P[(ia*nB+ib)*ldp + row] exact in FP64;
// t += (float)scalbn((float)P, tauA + tauB); y = (float)fma(alpha, t, beta*y).
__global__ void k_sum_rows_sd(int m, int nA, int nB, int maxlevel, const double *__restrict__ P, int64_t ldp,
                              const short *__restrict__ Ea, int ldea, const short *__restrict__ Eb, float alpha,
                              float beta, float *__restrict__ y) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    float t = 0.f;
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) {
        const float c32 = __double2float_rn(P[(size_t)(ia * nB + ib) * ldp + row]);
        t = __fadd_rn(t, __double2float_rn(scale2((double)c32, Ea[(size_t)ia * ldea + row] + Eb[ib])));
    });
    y[row] = __double2float_rn(fma((double)alpha, (double)t, (double)__fmul_rn(beta, y[row])));
}

// FP64 slices q 2^-(scale - tau) (slices [ns][nl][ldk], tau = exps[s * nl + line] or
// 0, q an integer below 2^(7 D))
// cut into D int8 digit planes, most significant first:
// dig[((s D + d) lines_pad + line) k_pad + i] = sign(q) ((|q| >> 7 (D-1-d)) & 127).
// The buffer is zeroed before (padding lines and columns stay zero).
__global__ void k_slices_to_digits(int ns, int nl, int k, int ldk, const double *__restrict__ S, int scale,
                                   const short *__restrict__ exps, int D, int lines_pad, int k_pad,
                                   int8_t *__restrict__ dig) {
    const int64_t total = (int64_t)ns * nl * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % k);
        const int64_t sl = e / k;  // s * nl + line
        const int line = (int)(sl % nl), s = (int)(sl / nl);
        const int sc = exps ? scale - (int)exps[sl] : scale;  // plain slices: q 2^(rho + tau - 53)
        const long long q = (long long)scale2(S[(size_t)sl * ldk + i], sc);
        const unsigned long long aq = (unsigned long long)(q < 0 ? -q : q);
        for (int d = 0; d < D; d++) {
            const int dv = (int)((aq >> (7 * (D - 1 - d))) & 127);
            dig[(((size_t)s * D + d) * lines_pad + line) * k_pad + i] = (int8_t)(q < 0 ? -dv : dv);
        }
    }
}

// The <float,double,double> ordered sum over a buffer of exact pair products
// pbuf[p][col][row]: t(float) += (float)scalbn((float)P, tauA + tauB), then
// C = (float)fma((double)alpha, t, (double)(beta * C)).
__global__ void k_sum_pairs_sd(int m, int n, int np, const double *__restrict__ pbuf, const int2 *__restrict__ dp,
                               const short *__restrict__ Ea, const short *__restrict__ Eb, float alpha, float beta,
                               float *__restrict__ C, int ldc) {
    const int64_t count = (int64_t)m * n;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const int row = (int)(e % m), col = (int)(e / m);
    float t = 0.f;
    for (int p = 0; p < np; p++) {
        const int2 pr = dp[p];
        const float c32 = __double2float_rn(pbuf[(size_t)p * count + e]);
        t = __fadd_rn(t, __double2float_rn(scale2((double)c32, Ea[(size_t)pr.x * m + row] + Eb[(size_t)pr.y * n + col])));
    }
    float *cp = C + (size_t)col * ldc + row;
    *cp = __double2float_rn(fma((double)alpha, (double)t, (double)__fmul_rn(beta, *cp)));
}

// Split op(X) (float, nl lines of length k) into FP64 slices ns x nl x ldk
// and exponents ns x nl; X with strided lines is transposed first.
static int split_operand_sd(cuozblasHandle_t *h, bool lines_strided, int nl, int k, const float *X, int ldx, int rho,
                            int maxS, int ldk, double **slices, short **exps, int *ns, Arena &ar) {
    const float *src = X;
    int lds = ldx;
    if (lines_strided) {
        float *tmp = ar.take<float>((uint64_t)nl * (k > 0 ? k : 1));
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(transpose_f32(h, nl, k, X, ldx, tmp, k));
        src = tmp;
        lds = k;
    }
    OZB_TRY(split_lines_count_sd(h, k, nl, src, lds, rho, maxS, ns));
    *slices = ar.take<double>((uint64_t)(*ns) * nl * ldk);
    *exps = ar.take<short>((uint64_t)(*ns) * nl);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    return split_lines_write_sd(h, k, nl, src, lds, rho, *ns, *slices, ldk, *exps);
}

int gemm_sd_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int fastMode) {
    State *st = state(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule_sd(k, h->splitEpsMode);
    Arena ar(h);
    const bool dot = (m == 1 && n == 1);
    const bool skinny_n = (n == 1);
    const int ldk = dot || skinny_n ? ceil_to(k > 0 ? k : 1, 2) : ceil_to(k > 0 ? k : 1, kBK);

    ev_record(h, 0);
    st->plain_timers = true;
    double *Sa = nullptr, *Sb = nullptr;
    short *Ea = nullptr, *Eb = nullptr;
    int nA = 0, nB = 0;
    // lines of op(A): 'n' -> row i of A is strided by lda; a vector is one line
    OZB_TRY(split_operand_sd(h, dot ? false : !is_trans(ta), m, k, A, dot ? k : lda, rho, maxS, ldk, &Sa, &Ea, &nA,
                             ar));
    ev_record(h, 1);
    OZB_TRY(split_operand_sd(h, skinny_n ? false : is_trans(tb), n, k, B, skinny_n ? k : ldb, rho, maxS, ldk, &Sb,
                             &Eb, &nB, ar));
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
        double *P = ar.take<double>((uint64_t)nA * nB * ldp);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        if (dot) OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(double) * nA * nB, st->stream));
        for (int ia0 = 0; ia0 < nA; ia0 += 8)
            for (int ib0 = 0; ib0 < nB; ib0 += 8) {
                const int na = nA - ia0 < 8 ? nA - ia0 : 8, nb = nB - ib0 < 8 ? nB - ib0 : 8;
                counted(h);
                if (dot) {
                    int blocks = (k + 255) / 256;
                    if (blocks > sm_count() * 8) blocks = sm_count() * 8;
                    if (blocks < 1) blocks = 1;
                    k_pair_dot<<<blocks, 256, 0, st->stream>>>(k, na, nb, Sa + (size_t)ia0 * ldk, ldk,
                                                               Sb + (size_t)ib0 * ldk, ldk, P + ia0 * nB + ib0, nB);
                } else {
                    const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
                    k_pair_gemv<<<blocks, 256, 0, st->stream>>>(m, k, na, nb, ia0, ib0, nB, Sa, ldk, Sb, ldk, P,
                                                                ldp);
                }
                OZB_CHECK(cudaGetLastError());
            }
        ev_record(h, 3);
        counted(h);
        k_sum_rows_sd<<<(rows + 127) / 128, 128, 0, st->stream>>>(rows, nA, nB, maxlevel, P, ldp, Ea, rows, Eb, alpha,
                                                                  beta, C);
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 4);
        return CUOZBLAS_STATUS_SUCCESS;
    }

    // Pair products on the INT8 tensor cores: for rho >= 2 (k > 128) x + sigma
    // stays in sigma's binade, so a slice is q 2^(rho - 24) with an integer
    // |q| <= 2^(24 - rho) < 2^(7 D), cut into D <= 4 int8 digits; D k 127^2 must
    // keep an INT32 group exact and the products of all pairs must fit.
    {
        const int D = (24 - rho + 1 + 6) / 7;
        const int k_pad = (k + 127) / 128 * 128;
        const int lpadA = (m + 127) / 128 * 128, lpadB = (n + 127) / 128 * 128;
        const uint64_t need = (uint64_t)nA * D * lpadA * k_pad + (uint64_t)nB * D * lpadB * k_pad +
                              sizeof(double) * (uint64_t)np * m * n + (1u << 20);
        const uint64_t avail = h->workSizeBytes - ((ar.mark() + 255) / 256 * 256);
        if (rho >= 2 && D <= 4 && (double)D * k * 127.0 * 127.0 < 2147483647.0 && need < avail &&
            !state(h)->env.sd_dmma) {
            std::vector<int2> pl;
            for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { pl.push_back(make_int2(ia, ib)); });
            int8_t *dg[2];
            for (int o = 0; o < 2; o++) {
                const int nl = o == 0 ? m : n, ns = o == 0 ? nA : nB, lpad = o == 0 ? lpadA : lpadB;
                dg[o] = ar.take<int8_t>((uint64_t)ns * D * lpad * k_pad);
                if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
                OZB_CHECK(cudaMemsetAsync(dg[o], 0, (size_t)ns * D * lpad * k_pad, st->stream));
                const int64_t total = (int64_t)ns * nl * k;
                int blocks = (int)((total + 255) / 256);
                if (blocks > sm_count() * 16) blocks = sm_count() * 16;
                if (blocks < 1) blocks = 1;
                counted(h);
                k_slices_to_digits<<<blocks, 256, 0, st->stream>>>(ns, nl, k, ldk, o == 0 ? Sa : Sb, 24 - rho, nullptr,
                                                                  D, lpad, k_pad, dg[o]);
                OZB_CHECK(cudaGetLastError());
            }
            double *pbuf = ar.take<double>((uint64_t)np * m * n);
            int2 *dp = ar.take<int2>(np > 0 ? np : 1);
            if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
            OZB_CHECK(cudaMemcpyAsync(dp, pl.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, st->stream));
            OZB_TRY(i8_exact_pairs(h, m, n, k_pad, dg[0], lpadA, nA * D, dg[1], lpadB, nB * D, D, pl, 2 * (rho - 24),
                                   nullptr, nullptr, pbuf));
            const int64_t count = (int64_t)m * n;
            counted(h);
            k_sum_pairs_sd<<<(unsigned)((count + 255) / 256), 256, 0, st->stream>>>(m, n, np, pbuf, dp, Ea, Eb, alpha,
                                                                                   beta, C, ldc);
            OZB_CHECK(cudaGetLastError());
            ev_record(h, 3);
            ev_record(h, 4);
            return CUOZBLAS_STATUS_SUCCESS;
        }
    }

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
    dim3 grid((m + kBM - 1) / kBM, (n + kBN - 1) / kBN);
    counted(h);
    k_gemm_pairs_dmma<false, true><<<grid, 128, 0, st->stream>>>(m, n, n, ldk, Sa, Sb, dp, np, (double)alpha,
                                                                 (double)beta, nullptr, ldc, nullptr, Ea, Eb, C);
    OZB_CHECK(cudaGetLastError());
    ev_record(h, 3);
    ev_record(h, 4);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
