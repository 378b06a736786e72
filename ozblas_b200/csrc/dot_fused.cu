// dot_fused.cu — the plain-form DOT in two passes over x and y.
//
// The reference splits each vector level by level with one global tau chain
// (src/cpu/ozblas_split.cpp:62-103), one pass per level, and then forms the
// nA x nB exact slice products (src/cpu/ozblas_gemm.cpp:209-215).  Here:
//
//  pass 1  max|x| and max|y|, hence tau_0 of each chain;
//  pass 2  the chain is predicted as tau_{s+1} = tau_s + rho - 54 (the
//          remainder after level s is at most 2^(tau_s + rho - 54), and with
//          many elements its maximum is almost surely in the top binade); every
//          element's slices are cut in registers with those sigmas, all slice
//          products are accumulated (exact, so any order gives the same sums),
//          and two bits per level record whether some remainder is nonzero and
//          whether some remainder is large enough to have that predicted tau;
//  finish  one thread checks the bits: the prediction holds iff every level
//          that leaves a nonzero remainder also leaves one whose tau is the
//          predicted one.  It then applies the reference's count rule and the
//          FSum / NearSum over the pairs.  If the prediction fails (or more than
//          kDotLevels levels are needed) the host runs the general level-by-
//          level path instead, so the result is always the reference's.
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "sum.cuh"

namespace ozb {

constexpr int kDotLevels = 8;
constexpr int kDotThreads = 256;

struct DotScratch {
    double mx[2];                            // max|x|, max|y| (bit-pattern atomics)
    double P[kDotLevels * kDotLevels];       // exact slice products P[ia * 8 + ib]
    unsigned int nz[2], hi[2];               // per-level flags (bit s: after level s)
    double tmp[kDotLevels * kDotLevels];     // NearSum workspace
    int status;                              // 1: valid
    int ns[2];
};

__global__ void __launch_bounds__(kDotThreads) k_dot_max(int n, const double *__restrict__ x,
                                                         const double *__restrict__ y, DotScratch *sc) {
    __shared__ double red[kDotThreads / 32];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double mx = 0.0, my = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        mx = ref_max(mx, fabs(x[i]));
        my = ref_max(my, fabs(y[i]));
    }
    mx = block_max_nonneg(mx, red);
    my = block_max_nonneg(my, red);
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&sc->mx[0], mx);
        atomic_max_nonneg(&sc->mx[1], my);
    }
}

// Largest double whose tau_rule is t - 1 (so v > it  <=>  tau_rule(v) >= t),
// for normal binades; returns a negative value when t - 1 is subnormal (the
// prediction is then not checked and the general path runs).
__device__ __forceinline__ double tau_floor_threshold(int t) {
    const int e = t - 1;
    if (e < -1022 || e > 1023) return -1.0;
    const int ae = e < 0 ? -e : e;
    int p = (ae == 0) ? -1 : (31 - clz32((uint32_t)ae));
    if (e < 0 && (ae & (ae - 1)) == 0) p -= 1;
    int J;
    switch (p) {
        case 2: J = 1; break;
        case 3: J = 2; break;
        case 4: J = 5; break;
        case 5: J = 11; break;
        case 6: J = 22; break;
        case 7: J = 44; break;
        case 8: J = 88; break;
        case 9: J = 177; break;
        case 10: J = 354; break;
        default: J = 0; break;
    }
    return from_bits(dbits(pow2(e)) + (uint64_t)J);
}

struct Chain {
    double sigma[kDotLevels];
    double thr[kDotLevels];  // remainder after level s must exceed thr[s] somewhere
};

__device__ __forceinline__ void make_chain(double mx, int rho, Chain &c) {
    int tau = tau_rule(mx);
#pragma unroll
    for (int s = 0; s < kDotLevels; s++) {
        c.sigma[s] = 0.75 * pow2(rho + tau);
        tau = tau + rho - 54;
        c.thr[s] = tau_floor_threshold(tau);
    }
}

template <bool SAME>
__global__ void __launch_bounds__(kDotThreads) k_dot_fused(int n, const double *__restrict__ x,
                                                           const double *__restrict__ y, int rho,
                                                           DotScratch *__restrict__ sc) {
    __shared__ Chain cx, cy;  // predicted sigmas and tau thresholds, shared by the block
    if (threadIdx.x == 0) {
        make_chain(sc->mx[0], rho, cx);
        if (!SAME) make_chain(sc->mx[1], rho, cy);
    }
    __syncthreads();
    double P[kDotLevels][kDotLevels];
#pragma unroll
    for (int a = 0; a < kDotLevels; a++)
#pragma unroll
        for (int b = 0; b < kDotLevels; b++) P[a][b] = 0.0;
    unsigned int nzx = 0, hix = 0, nzy = 0, hiy = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        double sx[kDotLevels], sy[kDotLevels];
        double r = x[i];
#pragma unroll
        for (int s = 0; s < kDotLevels; s++) {
            const double sl = (r + cx.sigma[s]) - cx.sigma[s];
            r = r - sl;
            sx[s] = sl;
            const uint64_t rb = dbits(r) & 0x7fffffffffffffffULL;
            nzx |= (rb != 0) ? (1u << s) : 0u;
            hix |= (rb > dbits(cx.thr[s])) ? (1u << s) : 0u;
        }
        if (SAME) {
#pragma unroll
            for (int s = 0; s < kDotLevels; s++) sy[s] = sx[s];
        } else {
            r = y[i];
#pragma unroll
            for (int s = 0; s < kDotLevels; s++) {
                const double sl = (r + cy.sigma[s]) - cy.sigma[s];
                r = r - sl;
                sy[s] = sl;
                const uint64_t rb = dbits(r) & 0x7fffffffffffffffULL;
                nzy |= (rb != 0) ? (1u << s) : 0u;
                hiy |= (rb > dbits(cy.thr[s])) ? (1u << s) : 0u;
            }
        }
#pragma unroll
        for (int a = 0; a < kDotLevels; a++)
#pragma unroll
            for (int b = 0; b < kDotLevels; b++) P[a][b] = fma(sx[a], sy[b], P[a][b]);
    }
    // reduce: exact sums, so the order is free
    __shared__ double red[kDotThreads / 32][kDotLevels * kDotLevels];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int a = 0; a < kDotLevels; a++)
#pragma unroll
        for (int b = 0; b < kDotLevels; b++) {
            double v = P[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (l == 0) red[w][a * kDotLevels + b] = v;
        }
    for (int o = 16; o > 0; o >>= 1) {
        nzx |= __shfl_xor_sync(0xffffffffu, nzx, o);
        hix |= __shfl_xor_sync(0xffffffffu, hix, o);
        nzy |= __shfl_xor_sync(0xffffffffu, nzy, o);
        hiy |= __shfl_xor_sync(0xffffffffu, hiy, o);
    }
    if (l == 0) {
        atomicOr(&sc->nz[0], nzx);
        atomicOr(&sc->hi[0], hix);
        if (!SAME) {
            atomicOr(&sc->nz[1], nzy);
            atomicOr(&sc->hi[1], hiy);
        }
    }
    __syncthreads();
    if (threadIdx.x < kDotLevels * kDotLevels) {
        double v = 0.0;
        for (int i = 0; i < kDotThreads / 32; i++) v += red[i][threadIdx.x];
        atomicAdd(&sc->P[threadIdx.x], v);
    }
}

// Count rule of the reference (src/cpu/ozblas_split.cpp:272-289) from the
// per-level nonzero bits; -1 when the prediction is not proven or more
// levels than computed are needed.
__device__ __forceinline__ int chain_count(unsigned nz, unsigned hi, int maxS, const double thr_valid) {
    (void)thr_valid;
    int z = kDotLevels;
    for (int s = 0; s < kDotLevels; s++)
        if (!(nz & (1u << s))) {
            z = s;
            break;
        }
    int ns;
    if (z >= kDotLevels) {
        if (maxS > kDotLevels) return -1;
        ns = maxS;
    } else {
        ns = (z < 1 ? 1 : z) + 1;
        if (ns > maxS) ns = maxS;
    }
    // levels 1..ns-1 were cut with predicted sigmas: valid iff every nonzero
    // remainder feeding them has the predicted tau
    for (int s = 0; s + 1 < ns; s++)
        if ((nz & (1u << s)) && !(hi & (1u << s))) return -1;
    return ns;
}

__global__ void k_dot_finish(DotScratch *sc, int maxS, int rho, int same, int sum_mode, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    // thresholds below the normal range cannot be checked: general path
    Chain cx, cy;
    make_chain(sc->mx[0], rho, cx);
    make_chain(sc->mx[1], rho, cy);
    const int nA = chain_count(sc->nz[0], sc->hi[0], maxS, 0.0);
    const int nB = same ? nA : chain_count(sc->nz[1], sc->hi[1], maxS, 0.0);
    bool ok = nA > 0 && nB > 0;
    for (int s = 0; ok && s + 1 < nA; s++)
        if (cx.thr[s] < 0.0 && (sc->nz[0] & (1u << s))) ok = false;
    for (int s = 0; ok && s + 1 < nB; s++)
        if ((same ? cx.thr[s] : cy.thr[s]) < 0.0 && (sc->nz[same ? 0 : 1] & (1u << s))) ok = false;
    sc->status = ok ? 1 : 0;
    sc->ns[0] = nA;
    sc->ns[1] = nB;
    if (!ok) return;
    const int maxlevel = nA + nB - 2;  // DOT: fastMode is ignored (src/cpu/ozblas_gemm.cpp:26-29)
    double t = 0.0;
    if (sum_mode == 1) {
        int np = 0;
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { sc->tmp[np++] = sc->P[ia * kDotLevels + ib]; });
        t = nearsum(np, sc->tmp, 1);
    } else {
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { t += sc->P[ia * kDotLevels + ib]; });
    }
    *out = fma(1.0, t, 0.0 * *out);  // alpha = 1, beta = 0 as the DOT driver passes them
}

// Returns SUCCESS with *done = true and the result in *out_dev when the fused
// path proves its chain; *done = false means the caller must use the general
// path (nothing was written to out_dev).
int dot_fused(cuozblasHandle_t *h, int n, const double *x, const double *y, double *out_dev, bool *done, int *nA,
              int *nB) {
    State *st = state(h);
    *done = false;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    DotScratch *sc = ar.take<DotScratch>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    const bool same = (x == y);
    OZB_CHECK(cudaMemsetAsync(sc, 0, sizeof(DotScratch), st->stream));
    int dev = 0, nsm = 0;
    OZB_CHECK(cudaGetDevice(&dev));
    OZB_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int blocks = (int)(((int64_t)n + kDotThreads - 1) / kDotThreads);
    int cap = nsm * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    counted(h);
    k_dot_max<<<blocks, kDotThreads, 0, st->stream>>>(n, x, y, sc);
    int fblocks = (int)(((int64_t)n + kDotThreads - 1) / kDotThreads);
    const int fcap = nsm;  // ~240 registers per thread: one 256-thread block per SM
    if (fblocks > fcap) fblocks = fcap;
    if (fblocks < 1) fblocks = 1;
    counted(h);
    if (same)
        k_dot_fused<true><<<fblocks, kDotThreads, 0, st->stream>>>(n, x, y, rho, sc);
    else
        k_dot_fused<false><<<fblocks, kDotThreads, 0, st->stream>>>(n, x, y, rho, sc);
    counted(h);
    k_dot_finish<<<1, 32, 0, st->stream>>>(sc, maxS, rho, same ? 1 : 0, h->sumMode, out_dev);
    OZB_CHECK(cudaGetLastError());
    int res[3];
    OZB_CHECK(cudaMemcpyAsync(res, &sc->status, sizeof(res), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    ar.release(mk);
    if (res[0] == 1) {
        *done = true;
        *nA = res[1];
        *nB = res[2];
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
