// dot_fused.cu — the plain-form DOT in two passes over x and y.
//
// The reference splits each vector level by level with one global tau chain
// (src/cpu/ozblas_split.cpp:62-103), one pass per level, and then forms the
// nA x nB exact slice products (src/cpu/ozblas_gemm.cpp:209-215).  Here:
//
//  pass 1  (k_dot_scan) max|v|, hence tau_0, and the lowest set bit of any
//          nonzero element, for x and y.
//  pass 2  (k_dot_tree) the chain is predicted as tau_{s+1} = tau_s + rho - 54
//          (the remainder after level s is at most 2^(tau_s + rho - 54); with
//          many elements its maximum is almost surely in the top binade).
//          Under that chain level s rounds to the grid g_s = 2^(rho+tau_s-53),
//          the partial sum of slices 0..s is RN_{g_s}(v) and the remainder
//          after level s is zero exactly when v is a multiple of g_s, so the
//          lowest set bit gives the first all-zero level (and with it the
//          reference's count rule) before pass 2 starts.  Each element is cut
//          in registers; slice products are accumulated (exact, so any order
//          gives the same sums); per level the largest next slice is kept,
//          which bounds the remainder from below and proves that its tau is
//          the predicted one.  The last block to finish checks the proof and
//          applies the FSum / NearSum over the pairs.  If the prediction is
//          not proven (or more than kDotLevels levels are needed, or an element
//          is Inf/NaN) the host runs the general level-by-level path instead,
//          so the result is always the reference's.
//
// Cutting: RN_g(v) = (v + sigma) - sigma is exact while |v| <= sigma / 3, so
// within a group of G levels (G - 1 <= (rho - 3) / d, d = 54 - rho) all
// roundings come from one base value at once and slice s is RN_s - RN_{s-1};
// the base of the next group is the remainder.  This is the same arithmetic
// as the level-by-level chain with a dependency depth of ~3 per group.
#include <cstring>

#include "fused.h"
#include "ozb_internal.h"
#include "sum.cuh"

namespace ozb {

// ---- pass 1 ---------------------------------------------------------------

template <bool ALIGNED, bool SAME>
__global__ void __launch_bounds__(256) k_dot_scan(int n, const double *__restrict__ x, const double *__restrict__ y,
                                                  DotScratch *sc) {
    __shared__ double red[8];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double mx = 0.0, my = 0.0;
    int lx = 0, ly = 0, bx = 0, by = 0;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ALIGNED) {
        const int64_t np = (int64_t)n >> 1;
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        for (; i + 3 * stride < np; i += 4 * stride) {
            double2 a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                a[u] = x2[i + u * stride];
                if (!SAME) b[u] = y2[i + u * stride];
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                scan_elem(a[u].x, mx, lx, bx);
                scan_elem(a[u].y, mx, lx, bx);
                if (!SAME) {
                    scan_elem(b[u].x, my, ly, by);
                    scan_elem(b[u].y, my, ly, by);
                }
            }
        }
        for (; i < np; i += stride) {
            const double2 a = x2[i];
            scan_elem(a.x, mx, lx, bx);
            scan_elem(a.y, mx, lx, bx);
            if (!SAME) {
                const double2 b = y2[i];
                scan_elem(b.x, my, ly, by);
                scan_elem(b.y, my, ly, by);
            }
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
            scan_elem(x[n - 1], mx, lx, bx);
            if (!SAME) scan_elem(y[n - 1], my, ly, by);
        }
    } else {
        for (; i < n; i += stride) {
            scan_elem(x[i], mx, lx, bx);
            if (!SAME) scan_elem(y[i], my, ly, by);
        }
    }
    scan_commit(&sc->vs, 0, mx, lx, bx, red);
    if (!SAME) scan_commit(&sc->vs, 1, my, ly, by, red);
}

// ---- pass 2 -----------------------------------------------------------------

// Two elements of x (and y) per lane, cut to levels 0..T; while levels of a
// vector wait for their proof the warp votes on them; then all products.
template <int G, int T, bool SAME>
__device__ __forceinline__ void dot_body(double x0, double y0, double x1, double y1, const TreePlan &pl,
                                         double (&P)[kDotLevels][kDotLevels], unsigned (&prov)[2]) {
    double a0[T + 1], a1[T + 1], b0[T + 1], b1[T + 1];
    cut_tree<G, T>(x0, pl.sig[0], a0);
    cut_tree<G, T>(x1, pl.sig[0], a1);
    if (!SAME) {
        cut_tree<G, T>(y0, pl.sig[1], b0);
        cut_tree<G, T>(y1, pl.sig[1], b1);
    }
    const unsigned px = pl.need[0] & ~prov[0];
    if (px) {  // uniform
        unsigned hw[kDotLevels];
#pragma unroll
        for (int s = 0; s < T; s++) hw[s] = max(abs_hiword(a0[s + 1]), abs_hiword(a1[s + 1]));
        prov[0] |= prove_levels<T>(hw, pl.hb[0], px);
    }
    if (!SAME) {
        const unsigned py = pl.need[1] & ~prov[1];
        if (py) {
            unsigned hw[kDotLevels];
#pragma unroll
            for (int s = 0; s < T; s++) hw[s] = max(abs_hiword(b0[s + 1]), abs_hiword(b1[s + 1]));
            prov[1] |= prove_levels<T>(hw, pl.hb[1], py);
        }
    }
#pragma unroll
    for (int a = 0; a <= T; a++)
#pragma unroll
        for (int b = 0; b <= T; b++) {
            if (SAME) {
                if (b >= a) P[a][b] = fma(a1[a], a1[b], fma(a0[a], a0[b], P[a][b]));
            } else {
                P[a][b] = fma(a1[a], b1[b], fma(a0[a], b0[b], P[a][b]));
            }
        }
}

template <int G, bool SAME>
__device__ __forceinline__ void dot_element(double x0, double y0, double x1, double y1, const TreePlan &pl,
                                            double (&P)[kDotLevels][kDotLevels], unsigned (&prov)[2]) {
    // the deepest level any lane of this warp needs (every lane calls this)
    int T = plan_depth(pl, 0, __reduce_min_sync(0xffffffffu, min(exp_key(x0), exp_key(x1))));
    if (!SAME) {
        const int ty = plan_depth(pl, 1, __reduce_min_sync(0xffffffffu, min(exp_key(y0), exp_key(y1))));
        T = ty > T ? ty : T;
    }
    if (T > pl.L - 1) T = pl.L - 1;
    switch (T) {
        case 0: dot_body<G, 0, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 1: dot_body<G, 1, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 2: dot_body<G, 2, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 3: dot_body<G, 3, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 4: dot_body<G, 4, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 5: dot_body<G, 5, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        case 6: dot_body<G, 6, SAME>(x0, y0, x1, y1, pl, P, prov); break;
        default: dot_body<G, 7, SAME>(x0, y0, x1, y1, pl, P, prov); break;
    }
}

// Proof of the chain, count rule and the FSum / NearSum over the pairs; one
// thread of the last block.  `Pv` and `tmp` are shared arrays.
__device__ void dot_finish(DotScratch *sc, const TreePlan &pl, int rho, bool same, int sum_mode, double *Pv,
                           double *tmp) {
    int valid = pl.valid;
    for (int v = 0; v < (same ? 1 : 2); v++)
        if ((__ldcg(&sc->proven[v]) & pl.need[v]) != pl.need[v]) valid = 0;
    const int nA = pl.ns[0], nB = same ? pl.ns[0] : pl.ns[1];
    sc->out.ns0 = nA;
    sc->out.ns1 = nB;
    sc->out.status = valid;
    if (!valid) return;
    const int maxlevel = nA + nB - 2;  // DOT: fastMode is ignored (src/cpu/ozblas_gemm.cpp:26-29)
    double t = 0.0;
    if (sum_mode == 1) {
        int np = 0;
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { tmp[np++] = Pv[ia * kDotLevels + ib]; });
        t = nearsum(np, tmp, 1);
    } else {
        for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { t += Pv[ia * kDotLevels + ib]; });
    }
    sc->out.result = fma(1.0, t, 0.0 * 0.0);  // alpha = 1, beta = 0 as the DOT driver passes them
}

template <int G, bool SAME, bool ALIGNED>
__global__ void __launch_bounds__(kDotThreads, 1) k_dot_tree(int n, const double *__restrict__ x,
                                                             const double *__restrict__ y, int rho, int maxS,
                                                             int sum_mode, DotScratch *__restrict__ sc,
                                                             const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    __shared__ TreePlan pl;
    extern __shared__ __align__(16) double2 ring_raw[];  // [kDotStages][SAME ? 1 : 2][kDotThreads]
    auto ring = reinterpret_cast<double2(*)[SAME ? 1 : 2][kDotThreads]>(ring_raw);
    __shared__ double red[kDotThreads / 32][kDotLevels * kDotLevels];
    __shared__ int last;
    const int t = threadIdx.x;
    plan_in_block(&sc->vs, rho, maxS, SAME, pl);
    __syncthreads();
    double P[kDotLevels][kDotLevels];
#pragma unroll
    for (int a = 0; a < kDotLevels; a++)
#pragma unroll
        for (int b = 0; b < kDotLevels; b++) P[a][b] = 0.0;
    unsigned prov[2] = {0u, 0u};  // per warp (uniform)

    if (pl.valid) {  // uniform
        if (ALIGNED) {
            const int64_t npairs = (int64_t)n >> 1;
            const int64_t stride = (int64_t)gridDim.x * kDotThreads;
            const int64_t i0 = (int64_t)blockIdx.x * kDotThreads + t;
            const int64_t iw = (int64_t)blockIdx.x * kDotThreads + (t & ~31);  // the warp's first pair
            const int64_t K = iw < npairs ? (npairs - iw + stride - 1) / stride : 0;
            const double2 *x2 = reinterpret_cast<const double2 *>(x);
            const double2 *y2 = reinterpret_cast<const double2 *>(y);
#pragma unroll
            for (int s = 0; s < kDotStages - 1; s++) {
                const int64_t i = i0 + s * stride;
                const bool ok = i < npairs;
                cp_async16(&ring[s][0][t], x2 + (ok ? i : 0), ok);
                if (!SAME) cp_async16(&ring[s][SAME ? 0 : 1][t], y2 + (ok ? i : 0), ok);
                cp_async_commit();
            }
            int slot = 0, fill = kDotStages - 1;
            for (int64_t k = 0; k < K; k++) {
                cp_async_wait<kDotStages - 2>();
                const double2 xv = ring[slot][0][t];
                const double2 yv = SAME ? xv : ring[slot][SAME ? 0 : 1][t];
                {
                    const int64_t i = i0 + (k + kDotStages - 1) * stride;
                    const bool ok = i < npairs;
                    cp_async16(&ring[fill][0][t], x2 + (ok ? i : 0), ok);
                    if (!SAME) cp_async16(&ring[fill][SAME ? 0 : 1][t], y2 + (ok ? i : 0), ok);
                    cp_async_commit();
                }
                slot = slot + 1 == kDotStages ? 0 : slot + 1;
                fill = fill + 1 == kDotStages ? 0 : fill + 1;
                dot_element<G, SAME>(xv.x, yv.x, xv.y, yv.y, pl, P, prov);
            }
            cp_async_wait<0>();
            if ((n & 1) && blockIdx.x == 0 && t < 32) {  // the odd last element, one warp
                const double xe = t == 0 ? x[n - 1] : 0.0;
                const double ye = t == 0 ? y[n - 1] : 0.0;
                dot_element<G, SAME>(xe, ye, 0.0, 0.0, pl, P, prov);
            }
        } else {
            const int64_t stride = (int64_t)gridDim.x * kDotThreads;
            const int64_t iw = (int64_t)blockIdx.x * kDotThreads + (t & ~31);
            const int64_t K = iw < n ? ((int64_t)n - iw + stride - 1) / stride : 0;
            int64_t i = (int64_t)blockIdx.x * kDotThreads + t;
            for (int64_t k = 0; k < K; k++, i += stride) {
                const double xe = i < n ? x[i] : 0.0;
                const double ye = SAME ? xe : (i < n ? y[i] : 0.0);
                dot_element<G, SAME>(xe, ye, 0.0, 0.0, pl, P, prov);
            }
        }
    }
    // block reduction: exact sums, so the order is free
    const int w = t >> 5, l = t & 31;
#pragma unroll
    for (int a = 0; a < kDotLevels; a++)
#pragma unroll
        for (int b = 0; b < kDotLevels; b++) {
            double v = SAME ? (b >= a ? P[a][b] : P[b][a]) : P[a][b];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (l == 0) red[w][a * kDotLevels + b] = v;
        }
    if (l == 0) {
        if (prov[0]) atomicOr(&sc->proven[0], prov[0]);
        if (!SAME && prov[1]) atomicOr(&sc->proven[1], prov[1]);
    }
    __syncthreads();
    if (t < kDotLevels * kDotLevels) {
        double v = 0.0;
        for (int i = 0; i < kDotThreads / 32; i++) v += red[i][t];
        if (v != 0.0) atomicAdd(&sc->P[t], v);
    }
    // the last block checks the chain and sums the pairs
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double *Pv = &red[0][0], *tmp = &red[1][0];
    if (t < kDotLevels * kDotLevels) Pv[t] = __ldcg(&sc->P[t]);
    __syncthreads();
    if (t == 0) dot_finish(sc, pl, rho, SAME, sum_mode, Pv, tmp);
    __syncthreads();
    // leave the accumulators zeroed for the next use (replayed graphs skip the memset)
    if (t < kDotLevels * kDotLevels) sc->P[t] = 0.0;
    if (t == 0) {
        sc->proven[0] = sc->proven[1] = 0u;
        sc->ticket = 0u;
        sc->vs = VecStats{};  // every CTA has read the statistics (the ticket comes after)
    }
}

template <int G, bool SAME>
static int launch_tree(bool aligned, int grid, cudaStream_t s, int n, const double *x, const double *y, int rho,
                       int maxS, int sum_mode, DotScratch *sc, const int *gate) {
    if (aligned) {
        const int smem = kDotStages * (SAME ? 1 : 2) * kDotThreads * (int)sizeof(double2);
        static std::atomic<uint64_t> attr{0};  // devices already opted in, per instantiation
        if (smem_optin((const void *)k_dot_tree<G, SAME, true>, smem, attr) != cudaSuccess)
            return CUOZBLAS_STATUS_CUDA_ERROR;
        k_dot_tree<G, SAME, true><<<grid, kDotThreads, smem, s>>>(n, x, y, rho, maxS, sum_mode, sc, gate);
    } else {
        k_dot_tree<G, SAME, false><<<grid, kDotThreads, 0, s>>>(n, x, y, rho, maxS, sum_mode, sc, gate);
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

template <int G, bool SAME>
static int prepare_tree() {
    const int smem = kDotStages * (SAME ? 1 : 2) * kDotThreads * (int)sizeof(double2);
    return cudaFuncSetAttribute(k_dot_tree<G, SAME, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
                   cudaSuccess
               ? CUOZBLAS_STATUS_SUCCESS
               : CUOZBLAS_STATUS_CUDA_ERROR;
}

int dot_tree_prepare() {
    int r = dot_i8_prepare();
    r |= prepare_tree<1, true>() | prepare_tree<1, false>() | prepare_tree<2, true>() | prepare_tree<2, false>();
    r |= prepare_tree<3, true>() | prepare_tree<3, false>() | prepare_tree<4, true>() | prepare_tree<4, false>();
    return r ? CUOZBLAS_STATUS_CUDA_ERROR : CUOZBLAS_STATUS_SUCCESS;
}

int dot_scan_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, DotScratch *sc) {
    const bool same = (x == y);
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15u) == 0;
    int blocks = (int)(((int64_t)n + 2 * kDotThreads - 1) / (2 * kDotThreads));
    if (blocks > nsm * 8) blocks = nsm * 8;
    if (blocks < 1) blocks = 1;
    if (aligned) {
        if (same)
            k_dot_scan<true, true><<<blocks, 256, 0, s>>>(n, x, y, sc);
        else
            k_dot_scan<true, false><<<blocks, 256, 0, s>>>(n, x, y, sc);
    } else {
        if (same)
            k_dot_scan<false, true><<<blocks, 256, 0, s>>>(n, x, y, sc);
        else
            k_dot_scan<false, false><<<blocks, 256, 0, s>>>(n, x, y, sc);
    }
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

int dot_tree_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, int rho, int maxS,
                    int sum_mode, DotScratch *sc, const int *gate, bool tree_only) {
    const int G = chain_group(rho, 4);  // levels cut from one base value
    const bool same = (x == y);
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15u) == 0;
    // 16-byte aligned vectors of at least 2^22 elements with 2 or 3 digits per
    // level take the tensor-core pass (it holds every valid plan; below that
    // length its fixed costs outweigh the FP64 tree pass, which takes the rest)
    if (aligned && n >= (1 << 22) && dot_i8_digits(rho) > 0 && !tree_only)
        return dot_i8_launch(s, nsm, n, x, y, rho, maxS, sum_mode, sc, gate);
    int fblocks = (int)(((int64_t)n + 2 * kDotThreads - 1) / (2 * kDotThreads));
    if (fblocks > nsm) fblocks = nsm;  // ~250 registers per thread: one 256-thread block per SM
    if (fblocks < 1) fblocks = 1;
    int ls;
    switch (G) {
        case 1:
            ls = same ? launch_tree<1, true>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate)
                      : launch_tree<1, false>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate);
            break;
        case 2:
            ls = same ? launch_tree<2, true>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate)
                      : launch_tree<2, false>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate);
            break;
        case 3:
            ls = same ? launch_tree<3, true>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate)
                      : launch_tree<3, false>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate);
            break;
        default:
            ls = same ? launch_tree<4, true>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate)
                      : launch_tree<4, false>(aligned, fblocks, s, n, x, y, rho, maxS, sum_mode, sc, gate);
            break;
    }
    if (ls) return ls;
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

// Returns SUCCESS with *done = true and the result in *ret when the fused
// path proves its chain; *done = false means the caller must use the general
// path.
int dot_fused(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret, bool *done, int *nA,
              int *nB) {
    State *st = state(h);
    *done = false;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    DotScratch *sc = ar.take<DotScratch>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    OZB_CHECK(cudaMemsetAsync(sc, 0, sizeof(DotScratch), st->stream));
    const int nsm = sm_count();
    span_begin(h);
    counted(h);
    OZB_TRY(dot_scan_launch(st->stream, nsm, n, x, y, sc));
    counted(h);
    OZB_TRY(dot_tree_launch(st->stream, nsm, n, x, y, rho, maxS, h->sumMode, sc, nullptr, st->env.dot_tree));
    span_end(h);
    static_assert(sizeof(DotStatus) == 24, "status block layout");
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, &sc->out, sizeof(DotStatus), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    ar.release(mk);
    DotStatus res;
    memcpy(&res, st->h_dbl, sizeof(res));
    if (res.status != 1 && state(h)->env.dot_trace)
        fprintf(stderr, "cuozblas: dot fused not used (n=%d, reason bits %d)\n", n, res.pad);
    if (res.status == 1) {
        *done = true;
        *nA = res.ns0;
        *nB = res.ns1;
        *ret = res.result;
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
