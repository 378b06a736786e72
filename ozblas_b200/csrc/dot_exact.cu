// dot_exact.cu — the NearSum DOT / NRM2 in one pass over x and y.
//
// With sumMode 1 and a complete split the reference's DOT is RN of the exact
// dot product: its nA x nB slice-pair products are exact, their sum over the
// full pair set is sum_k x_k y_k exactly, NearSum rounds that once
// (src/cpu/ozblas_sum.cpp:10-112) and the driver's fma(1, t, 0 * 0)
// (src/cpu/ozblas_dot.cpp:25-27, src/cpu/ozblas_sum.cpp:366) keeps it.  So
//
//  k_dot_exact  streams x and y once: the first-pass statistics of the split
//               (max, lowest set bit, Inf/NaN: the split counts) and the exact
//               dot in fixed-grid bins (xbins.cuh); its last block rounds the
//               exact sum (certified) into the scratch.
//  k_dot_prove  the split counts of the exec info rest on the predicted tau
//               chain (chain.cuh): this kernel proves it like the two-pass
//               DOT's second pass, cutting elements only until every level has
//               its witness (blocks stop as soon as the proof is complete, so
//               on ordinary data it reads a few thousand elements), and
//               publishes the result only when the chain is proven, the split
//               is complete (first all-zero level below the cap) and the
//               rounding was certified.  Otherwise the host runs the two-pass
//               DOT, which handles every case.
// The result is the reference's bits whenever it is published; the exec-info
// counts are those of the proven chain.
#include <cstring>

#include "fused.h"
#include "ozb_internal.h"
#include "sum.cuh"
#include "xbins.cuh"

namespace ozb {

constexpr int kXThreads = 256;

// Witness candidates of one block of the ring kernel: its largest |x| and the
// x element with the lowest set bit (the same for y).  Large elements carry
// the bits of the first levels, the lowest-bit ones those of the deepest.
struct DotCand {
    double mx, cx, my, cy;
};

struct DotExactScratch {
    XReduce xr;                // the blocks' bins of k_dot_exact
    unsigned ticket2;          // blocks of k_dot_prove that are done
    int certified;
    double result;             // certified RN(x . y)
    unsigned proven[2];        // levels whose predicted tau some element proved
    DotCand cand[kXMaxBlocks];
};

// ---- one pass: statistics and exact bins ----------------------------------

template <bool SAME, bool ALIGNED>
__global__ void __launch_bounds__(kXThreads) k_dot_exact(int n, const double *__restrict__ x,
                                                         const double *__restrict__ y, DotScratch *__restrict__ sc,
                                                         DotExactScratch *__restrict__ xs) {
    __shared__ double red[kXThreads / 32];
    __shared__ double res_sh;
    __shared__ int cert_sh;
    XAcc acc;
    xacc_init(acc);
    double mx = 0.0, my = 0.0;
    int lx = 0, ly = 0, bx = 0, by = 0;
    const int64_t stride = (int64_t)gridDim.x * kXThreads;
    constexpr int U = 2;  // double2 loads per vector per step
    if (ALIGNED) {
        const int64_t np = (int64_t)n >> 1;
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        // every lane of a warp runs the same number of steps (the bins' B is warp-uniform)
        const int64_t iw = (int64_t)blockIdx.x * kXThreads + (threadIdx.x & ~31);
        const int64_t steps = iw < np ? (np - iw + U * stride - 1) / (U * stride) : 0;
        int64_t i = (int64_t)blockIdx.x * kXThreads + threadIdx.x;
        for (int64_t s = 0; s < steps; s++, i += U * stride) {
            double2 a[U], b[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int64_t k = i + u * stride;
                a[u] = k < np ? x2[k] : make_double2(0.0, 0.0);
                if (!SAME) b[u] = k < np ? y2[k] : make_double2(0.0, 0.0);
            }
            unsigned hi = 0u;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const double2 bb = SAME ? a[u] : b[u];
                hi = max(hi, abs_hiword(__dmul_rn(a[u].x, bb.x)));
                hi = max(hi, abs_hiword(__dmul_rn(a[u].y, bb.y)));
                scan_elem(a[u].x, mx, lx, bx);
                scan_elem(a[u].y, mx, lx, bx);
                if (!SAME) {
                    scan_elem(b[u].x, my, ly, by);
                    scan_elem(b[u].y, my, ly, by);
                }
            }
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, hi));
#pragma unroll
            for (int u = 0; u < U; u++) {
                const double2 bb = SAME ? a[u] : b[u];
                xacc_product(acc, a[u].x, bb.x);
                xacc_product(acc, a[u].y, bb.y);
            }
            if ((s & 15) == 15) xacc_normalize(acc);  // every 64 products per lane
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x < 32) {  // the odd last element, one warp
            const double xe = threadIdx.x == 0 ? x[n - 1] : 0.0;
            const double ye = threadIdx.x == 0 ? y[n - 1] : 0.0;
            scan_elem(xe, mx, lx, bx);
            if (!SAME) scan_elem(ye, my, ly, by);
            xacc_normalize(acc);
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(xe, ye))));
            xacc_product(acc, xe, ye);
        }
    } else {
        const int64_t iw = (int64_t)blockIdx.x * kXThreads + (threadIdx.x & ~31);
        const int64_t steps = iw < n ? ((int64_t)n - iw + stride - 1) / stride : 0;
        int64_t i = (int64_t)blockIdx.x * kXThreads + threadIdx.x;
        for (int64_t s = 0; s < steps; s++, i += stride) {
            const double xe = i < n ? x[i] : 0.0;
            const double ye = SAME ? xe : (i < n ? y[i] : 0.0);
            scan_elem(xe, mx, lx, bx);
            if (!SAME) scan_elem(ye, my, ly, by);
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(xe, ye))));
            xacc_product(acc, xe, ye);
            if ((s & 63) == 63) xacc_normalize(acc);
        }
    }
    scan_commit(&sc->vs, 0, mx, lx, bx, red);
    if (!SAME) scan_commit(&sc->vs, 1, my, ly, by, red);
    if (!xreduce_finish(acc, &xs->xr, &res_sh, &cert_sh)) return;
    if (threadIdx.x == 0) {
        xs->result = res_sh;
        xs->certified = cert_sh;
    }
}

// ---- the chain proof, with early exit -------------------------------------

template <int G, int T, bool SAME>
__device__ __forceinline__ void prove_body(double x0, double y0, double x1, double y1, const TreePlan &pl,
                                           unsigned (&prov)[2]) {
    double a0[T + 1], a1[T + 1];
    cut_tree<G, T>(x0, pl.sig[0], a0);
    cut_tree<G, T>(x1, pl.sig[0], a1);
    const unsigned px = pl.need[0] & ~prov[0];
    if (px) {  // uniform
        unsigned hw[kChainLevels];
#pragma unroll
        for (int s = 0; s < T; s++) hw[s] = max(abs_hiword(a0[s + 1]), abs_hiword(a1[s + 1]));
        prov[0] |= prove_levels<T>(hw, pl.hb[0], px);
    }
    if (!SAME) {
        const unsigned py = pl.need[1] & ~prov[1];
        if (py) {
            double b0[T + 1], b1[T + 1];
            cut_tree<G, T>(y0, pl.sig[1], b0);
            cut_tree<G, T>(y1, pl.sig[1], b1);
            unsigned hw[kChainLevels];
#pragma unroll
            for (int s = 0; s < T; s++) hw[s] = max(abs_hiword(b0[s + 1]), abs_hiword(b1[s + 1]));
            prov[1] |= prove_levels<T>(hw, pl.hb[1], py);
        }
    }
}

template <int G, bool SAME>
__device__ __forceinline__ void prove_element(double x0, double y0, double x1, double y1, const TreePlan &pl,
                                              unsigned (&prov)[2]) {
    int T = plan_depth(pl, 0, __reduce_min_sync(0xffffffffu, min(exp_key(x0), exp_key(x1))));
    if (!SAME) {
        const int ty = plan_depth(pl, 1, __reduce_min_sync(0xffffffffu, min(exp_key(y0), exp_key(y1))));
        T = ty > T ? ty : T;
    }
    if (T > pl.L - 1) T = pl.L - 1;
    switch (T) {
        case 0: break;  // level 0 alone proves nothing
        case 1: prove_body<G, 1, SAME>(x0, y0, x1, y1, pl, prov); break;
        case 2: prove_body<G, 2, SAME>(x0, y0, x1, y1, pl, prov); break;
        case 3: prove_body<G, 3, SAME>(x0, y0, x1, y1, pl, prov); break;
        case 4: prove_body<G, 4, SAME>(x0, y0, x1, y1, pl, prov); break;
        case 5: prove_body<G, 5, SAME>(x0, y0, x1, y1, pl, prov); break;
        case 6: prove_body<G, 6, SAME>(x0, y0, x1, y1, pl, prov); break;
        default: prove_body<G, 7, SAME>(x0, y0, x1, y1, pl, prov); break;
    }
}

// The ring kernel's last block: the proof from every block's witness
// candidates (largest and lowest-bit elements), which on ordinary data proves
// every level.  Then status 1: the result is published and the scratch left
// zeroed, as k_dot_prove's last block does; 2: some level still needs a
// witness (k_dot_prove goes on from the levels proven here); 0: the one-pass
// result cannot be used (invalid plan, incomplete split or uncertified
// rounding; scratch left zeroed, the two-pass DOT runs).
template <int G, bool SAME>
__device__ void dot_ring_publish(DotScratch *sc, DotExactScratch *xs, int rho, int maxS, double res, int cert) {
    __shared__ TreePlan pl;
    const int t = threadIdx.x;
    plan_in_block(&sc->vs, rho, maxS, SAME, pl);
    __syncthreads();
    const unsigned need0 = pl.need[0], need1 = SAME ? 0u : pl.need[1];
    const int nA = pl.ns[0], nB = SAME ? pl.ns[0] : pl.ns[1];
    const int zA = pl.z[0], zB = SAME ? pl.z[0] : pl.z[1];
    const bool usable = pl.valid && cert && zA <= nA - 1 && zB <= nB - 1;
    if (usable && (need0 | need1)) {
        unsigned prov[2] = {0u, 0u};
        const int ncand = (int)gridDim.x;
        for (int base = 0; base < ncand; base += kXThreads) {  // uniform trip count
            const int i = base + t;
            DotCand c{0.0, 0.0, 0.0, 0.0};
            if (i < ncand)
                c = DotCand{__ldcg(&xs->cand[i].mx), __ldcg(&xs->cand[i].cx), __ldcg(&xs->cand[i].my),
                            __ldcg(&xs->cand[i].cy)};
            prove_element<G, SAME>(c.mx, c.my, c.cx, c.cy, pl, prov);
        }
        if ((t & 31) == 0) {
            if (prov[0]) atomicOr(&xs->proven[0], prov[0]);
            if (!SAME && prov[1]) atomicOr(&xs->proven[1], prov[1]);
        }
    }
    __threadfence();
    __syncthreads();
    if (t != 0) return;
    const bool proven =
        (__ldcg(&xs->proven[0]) & need0) == need0 && (__ldcg(&xs->proven[1]) & need1) == need1;
    if (usable && !proven) {
        sc->out.status = 2;
        return;
    }
    sc->out.ns0 = nA;
    sc->out.ns1 = nB;
    sc->out.status = usable ? 1 : 0;
    sc->out.pad = 0;
    sc->out.result = fma(1.0, res, 0.0 * 0.0);  // alpha = 1, beta = 0 as the DOT driver passes them
    xs->proven[0] = xs->proven[1] = 0u;
    xs->ticket2 = 0u;
    xs->certified = 0;
    sc->vs = VecStats{};
}

// The aligned form: each thread streams its double2 pairs of x and y through
// a private cp.async ring (kXStages groups of kXU pairs per vector; a thread
// reads back only its own copies, so no barrier), four products per group
// with one warp-wide fit and lean deposits (bounds per group).  The ring is
// reused as the last block's scratch.
constexpr int kXU = 2;
constexpr int kXStages = 4;
constexpr int kXLeanKD = 4;

template <bool SAME>
__host__ __device__ constexpr int dot_ring_bytes() {
    return kXStages * (SAME ? 1 : 2) * kXU * kXThreads * (int)sizeof(double2);
}

template <int G, bool SAME>
__device__ void dot_ring_publish(DotScratch *sc, DotExactScratch *xs, int rho, int maxS, double res, int cert);

template <int G, bool SAME>
__global__ void __launch_bounds__(kXThreads) k_dot_exact_ring(int n, const double *__restrict__ x,
                                                              const double *__restrict__ y, DotScratch *__restrict__ sc,
                                                              DotExactScratch *__restrict__ xs, int rho, int maxS) {
    constexpr int V = SAME ? 1 : 2;
    static_assert(dot_ring_bytes<SAME>() >= 256 * (kXK2 + 3) * (int)sizeof(double), "ring too small for the scratch");
    extern __shared__ __align__(16) double2 dring[];
    auto ring = reinterpret_cast<double2(*)[V][kXU][kXThreads]>(dring);
    __shared__ double red[kXThreads / 32];
    __shared__ double res_sh;
    __shared__ int cert_sh;
    const int t = threadIdx.x;
    XAcc acc;
    xacc_init(acc);
    LazyStats sx, sy;
    const int64_t np = (int64_t)n >> 1;
    const int64_t stride = (int64_t)gridDim.x * kXThreads;
    const double2 *x2 = reinterpret_cast<const double2 *>(x);
    const double2 *y2 = reinterpret_cast<const double2 *>(y);
    // every lane of a warp runs the same number of steps (the bins' B is warp-uniform)
    const int64_t iw = (int64_t)blockIdx.x * kXThreads + (t & ~31);
    const int64_t steps = iw < np ? (np - iw + kXU * stride - 1) / (kXU * stride) : 0;
    const int64_t i0 = (int64_t)blockIdx.x * kXThreads + t;
    auto issue = [&](int64_t s) {
        if (s < steps) {
#pragma unroll
            for (int u = 0; u < kXU; u++) {
                const int64_t k = i0 + (s * kXU + u) * stride;
                const bool ok = k < np;
                cp_async16(&ring[s % kXStages][0][u][t], x2 + (ok ? k : 0), ok);
                if (!SAME) cp_async16(&ring[s % kXStages][V - 1][u][t], y2 + (ok ? k : 0), ok);
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int s = 0; s < kXStages - 1; s++) issue(s);
    for (int64_t s = 0; s < steps; s++) {
        cp_async_wait<kXStages - 2>();
        double2 a[kXU], b[kXU];
#pragma unroll
        for (int u = 0; u < kXU; u++) {
            a[u] = ring[s % kXStages][0][u][t];
            b[u] = SAME ? a[u] : ring[s % kXStages][V - 1][u][t];
        }
        issue(s + kXStages - 1);  // into the slot read in the previous step (this thread's own)
        unsigned hi = 0u;
#pragma unroll
        for (int u = 0; u < kXU; u++) {
            hi = max(hi, abs_hiword(__dmul_rn(a[u].x, b[u].x)));
            hi = max(hi, abs_hiword(__dmul_rn(a[u].y, b[u].y)));
            lazy_elem(sx, a[u].x);
            lazy_elem(sx, a[u].y);
            if (!SAME) {
                lazy_elem(sy, b[u].x);
                lazy_elem(sy, b[u].y);
            }
        }
        lazy_sync(sx);
        if (!SAME) lazy_sync(sy);
        xacc_fit(acc, __reduce_max_sync(0xffffffffu, hi));
#pragma unroll
        for (int u = 0; u < kXU; u++) {
            xacc_product_lean<kXLeanKD>(acc, a[u].x, b[u].x);
            xacc_product_lean<kXLeanKD>(acc, a[u].y, b[u].y);
        }
        xacc_lean_bounds<kXLeanKD>(acc, hi, 2 * kXU);
        if ((s & 15) == 15) xacc_normalize(acc);  // every 64 products per lane
    }
    cp_async_wait<0>();
    if ((n & 1) && blockIdx.x == 0 && t < 32) {  // the odd last element, one warp
        const double xe = t == 0 ? x[n - 1] : 0.0;
        const double ye = t == 0 ? y[n - 1] : 0.0;
        lazy_elem(sx, xe);
        if (!SAME) lazy_elem(sy, ye);
        xacc_normalize(acc);
        xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(xe, ye))));
        xacc_product(acc, xe, ye);
    }
    {  // the block's candidates: per warp, then warp 0 over the warps
        __shared__ double cw[kXThreads / 32][4];
        __shared__ int kw[kXThreads / 32][2];
        double m0 = sx.mx, m1 = sy.mx;
        for (int o = 16; o > 0; o >>= 1) {
            m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
            if (!SAME) m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        }
        const int lk0 = lazy_key(sx), lk1 = lazy_key(sy);
        const int k0 = __reduce_max_sync(0xffffffffu, lk0), k1 = SAME ? 0 : __reduce_max_sync(0xffffffffu, lk1);
        const double c0 = __shfl_sync(0xffffffffu, sx.cand, __ffs(__ballot_sync(0xffffffffu, lk0 == k0)) - 1);
        const double c1 =
            SAME ? 0.0 : __shfl_sync(0xffffffffu, sy.cand, __ffs(__ballot_sync(0xffffffffu, lk1 == k1)) - 1);
        if ((t & 31) == 0) {
            cw[t >> 5][0] = m0;
            cw[t >> 5][1] = c0;
            cw[t >> 5][2] = m1;
            cw[t >> 5][3] = c1;
            kw[t >> 5][0] = k0;
            kw[t >> 5][1] = k1;
        }
        __syncthreads();
        if (t == 0) {
            DotCand c{cw[0][0], cw[0][1], cw[0][2], cw[0][3]};
            int b0 = kw[0][0], b1 = kw[0][1];
            for (int w = 1; w < kXThreads / 32; w++) {
                c.mx = fmax(c.mx, cw[w][0]);
                c.my = fmax(c.my, cw[w][2]);
                if (kw[w][0] > b0) {
                    b0 = kw[w][0];
                    c.cx = cw[w][1];
                }
                if (kw[w][1] > b1) {
                    b1 = kw[w][1];
                    c.cy = cw[w][3];
                }
            }
            xs->cand[blockIdx.x] = c;
        }
    }
    scan_commit(&sc->vs, 0, sx.mx, lazy_key(sx), lazy_bad(sx), red);
    if (!SAME) scan_commit(&sc->vs, 1, sy.mx, lazy_key(sy), lazy_bad(sy), red);
    __syncthreads();  // every thread is done with the ring before it becomes the scratch
    if (!xreduce_finish_sh(acc, &xs->xr, &res_sh, &cert_sh, reinterpret_cast<double *>(dring))) return;
    if (t == 0) {
        xs->result = res_sh;
        xs->certified = cert_sh;
    }
    dot_ring_publish<G, SAME>(sc, xs, rho, maxS, res_sh, cert_sh);
}

template <int G, bool SAME>
__global__ void __launch_bounds__(kXThreads) k_dot_prove(int n, const double *__restrict__ x,
                                                         const double *__restrict__ y, int rho, int maxS,
                                                         int ncand, DotScratch *__restrict__ sc,
                                                         DotExactScratch *__restrict__ xs) {
    __shared__ TreePlan pl;
    __shared__ int done_sh, last;
    const int t = threadIdx.x;
    plan_in_block(&sc->vs, rho, maxS, SAME, pl);
    __syncthreads();
    unsigned prov[2] = {0u, 0u};  // per warp (uniform)
    const unsigned need0 = pl.need[0], need1 = SAME ? 0u : pl.need[1];
    if (pl.valid && (need0 | need1) && (int)blockIdx.x * kXThreads < ncand) {
        // first the ring kernel's per-block candidates (its largest and its
        // lowest-bit elements), one per thread: on ordinary data they prove
        // every level, deep ones included, in this single round
        const int i = (int)blockIdx.x * kXThreads + t;
        DotCand c{0.0, 0.0, 0.0, 0.0};
        if (i < ncand)
            c = DotCand{__ldcg(&xs->cand[i].mx), __ldcg(&xs->cand[i].cx), __ldcg(&xs->cand[i].my),
                        __ldcg(&xs->cand[i].cy)};
        prove_element<G, SAME>(c.mx, c.my, c.cx, c.cy, pl, prov);
        if ((t & 31) == 0) {
            if (prov[0]) atomicOr(&xs->proven[0], prov[0]);
            if (!SAME && prov[1]) atomicOr(&xs->proven[1], prov[1]);
        }
        __threadfence();
        __syncthreads();  // the block's own witnesses are published before its first check
    }
    if (pl.valid && (need0 | need1)) {
        // kPP pairs per lane per round (their loads in flight together), then
        // the global proof state decides whether the block goes on
        constexpr int kPP = 4;
        const int64_t stride = (int64_t)gridDim.x * kXThreads * kPP;  // in element pairs (two per lane)
        const int64_t npairs = ((int64_t)n + 1) >> 1;
        for (int64_t base = (int64_t)blockIdx.x * kXThreads * kPP; base < npairs; base += stride) {
            if (t == 0) {
                const unsigned g0 = __ldcg(&xs->proven[0]), g1 = __ldcg(&xs->proven[1]);
                done_sh = (g0 & need0) == need0 && (g1 & need1) == need1;
            }
            __syncthreads();
            const int stop = done_sh;
            __syncthreads();
            if (stop) break;
            double xv[kPP][2], yv[kPP][2];
#pragma unroll
            for (int q = 0; q < kPP; q++) {
                const int64_t i = base + q * kXThreads + t, e0 = 2 * i, e1 = 2 * i + 1;
                xv[q][0] = e0 < n ? x[e0] : 0.0;
                xv[q][1] = e1 < n ? x[e1] : 0.0;
                yv[q][0] = SAME ? xv[q][0] : (e0 < n ? y[e0] : 0.0);
                yv[q][1] = SAME ? xv[q][1] : (e1 < n ? y[e1] : 0.0);
            }
            const unsigned before0 = prov[0], before1 = prov[1];
#pragma unroll
            for (int q = 0; q < kPP; q++) prove_element<G, SAME>(xv[q][0], yv[q][0], xv[q][1], yv[q][1], pl, prov);
            if ((t & 31) == 0) {
                if (prov[0] != before0) atomicOr(&xs->proven[0], prov[0]);
                if (!SAME && prov[1] != before1) atomicOr(&xs->proven[1], prov[1]);
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&xs->ticket2, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (t == 0) {
        int valid = pl.valid;
        if ((__ldcg(&xs->proven[0]) & need0) != need0 || (__ldcg(&xs->proven[1]) & need1) != need1) valid = 0;
        const int nA = pl.ns[0], nB = SAME ? pl.ns[0] : pl.ns[1];
        // a complete split: the first all-zero level lies within the levels the count keeps
        const int zA = pl.z[0], zB = SAME ? pl.z[0] : pl.z[1];
        if (zA > nA - 1 || zB > nB - 1) valid = 0;
        if (!__ldcg(&xs->certified)) valid = 0;
        sc->out.ns0 = nA;
        sc->out.ns1 = nB;
        sc->out.status = valid;
        sc->out.pad = 0;
        sc->out.result = fma(1.0, __ldcg(&xs->result), 0.0 * 0.0);  // alpha = 1, beta = 0 as the DOT driver passes them
        // leave the scratch zeroed for the next use
        xs->proven[0] = xs->proven[1] = 0u;
        xs->ticket2 = 0u;
        xs->certified = 0;
        sc->vs = VecStats{};
    }
}

// Returns SUCCESS with *done = true and the result in *ret when the one-pass
// NearSum DOT is proven; *done = false leaves the call to the two-pass DOT.
int dot_exact(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret, bool *done, int *nA,
              int *nB) {
    State *st = state(h);
    *done = false;
    if (n <= 0) return CUOZBLAS_STATUS_SUCCESS;
    // the handle's persistent scratch: zeroed at create, left zeroed by the kernels below
    static_assert(sizeof(DotScratch) + 256 + sizeof(DotExactScratch) <= kPersistBytes, "persistent scratch size");
    DotScratch *sc = reinterpret_cast<DotScratch *>(st->d_persist);
    DotExactScratch *xs = reinterpret_cast<DotExactScratch *>(reinterpret_cast<char *>(st->d_persist) +
                                                              (sizeof(DotScratch) + 255) / 256 * 256);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    const bool same = (x == y);
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15u) == 0;
    const int nsm = sm_count();
    span_begin(h);
    int blocks = (int)(((int64_t)n + 8LL * kXThreads - 1) / (8LL * kXThreads));
    if (blocks > nsm * 4) blocks = nsm * 4;
    if (blocks > kXMaxBlocks) blocks = kXMaxBlocks;
    if (blocks < 1) blocks = 1;
    const int G = chain_group(rho, 4);
    counted(h);
    int ncand = 0;  // blocks of the ring kernel, each leaving its witness candidates
    static_assert(sizeof(DotStatus) == 24, "status block layout");
    auto read_status = [&](DotStatus &res) -> int {
        OZB_CHECK(cudaMemcpyAsync(st->h_dbl, &sc->out, sizeof(DotStatus), cudaMemcpyDeviceToHost, st->stream));
        OZB_CHECK(cudaStreamSynchronize(st->stream));
        memcpy(&res, st->h_dbl, sizeof(res));
        return CUOZBLAS_STATUS_SUCCESS;
    };
    DotStatus res{};
    bool need_prove = true;
    if (aligned) {
        // one wave of the ring kernel: its resident blocks per SM x SMs
        static std::atomic<uint64_t> attr[2][4];
        static std::atomic<int> occs[2][4];
        const void *fn = nullptr;
#define OZB_RING_FN(GG) fn = same ? (const void *)k_dot_exact_ring<GG, true> : (const void *)k_dot_exact_ring<GG, false>
        switch (G) {
            case 1: OZB_RING_FN(1); break;
            case 2: OZB_RING_FN(2); break;
            case 3: OZB_RING_FN(3); break;
            default: OZB_RING_FN(4); break;
        }
#undef OZB_RING_FN
        const int gi = (G < 1 ? 1 : (G > 4 ? 4 : G)) - 1, si = same ? 1 : 0;
        const int smem = same ? dot_ring_bytes<true>() : dot_ring_bytes<false>();
        if (smem_optin(fn, smem, attr[si][gi]) != cudaSuccess) return CUOZBLAS_STATUS_CUDA_ERROR;
        int occ = occs[si][gi].load();
        if (occ == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kXThreads, smem) != cudaSuccess || occ < 1)
                occ = 1;
            occs[si][gi].store(occ);
        }
        int rb = (int)(((int64_t)n / 2 + (int64_t)kXU * kXThreads - 1) / ((int64_t)kXU * kXThreads));
        if (rb > nsm * occ) rb = nsm * occ;
        if (rb > kXMaxBlocks) rb = kXMaxBlocks;
        if (rb < 1) rb = 1;
        ncand = rb;
#define OZB_RING(GG)                                                                                          \
    do {                                                                                                    \
        if (same)                                                                                           \
            k_dot_exact_ring<GG, true><<<rb, kXThreads, smem, st->stream>>>(n, x, y, sc, xs, rho, maxS);     \
        else                                                                                                \
            k_dot_exact_ring<GG, false><<<rb, kXThreads, smem, st->stream>>>(n, x, y, sc, xs, rho, maxS);    \
    } while (0)
        switch (G) {
            case 1: OZB_RING(1); break;
            case 2: OZB_RING(2); break;
            case 3: OZB_RING(3); break;
            default: OZB_RING(4); break;
        }
#undef OZB_RING
        OZB_CHECK(cudaGetLastError());
        span_end(h);
        // the ring kernel's last block proved the chains from its candidates (status 1),
        // found the one-pass result unusable (0), or left levels for the proof kernel (2)
        OZB_TRY(read_status(res));
        need_prove = res.status == 2;
    } else {
        if (same)
            k_dot_exact<true, false><<<blocks, kXThreads, 0, st->stream>>>(n, x, y, sc, xs);
        else
            k_dot_exact<false, false><<<blocks, kXThreads, 0, st->stream>>>(n, x, y, sc, xs);
        OZB_CHECK(cudaGetLastError());
    }
    if (need_prove) {
        int pblocks = (int)((((int64_t)n + 1) / 2 + 4 * kXThreads - 1) / (4 * kXThreads));  // kPP = 4 pairs per lane
        if (pblocks > nsm * 2) pblocks = nsm * 2;
        if (pblocks < (ncand + kXThreads - 1) / kXThreads) pblocks = (ncand + kXThreads - 1) / kXThreads;
        if (pblocks < 1) pblocks = 1;
        counted(h);
#define OZB_PROVE(GG)                                                                                       \
    do {                                                                                                  \
        if (same)                                                                                         \
            k_dot_prove<GG, true><<<pblocks, kXThreads, 0, st->stream>>>(n, x, y, rho, maxS, ncand, sc, xs); \
        else                                                                                              \
            k_dot_prove<GG, false><<<pblocks, kXThreads, 0, st->stream>>>(n, x, y, rho, maxS, ncand, sc, xs); \
    } while (0)
        switch (G) {
            case 1: OZB_PROVE(1); break;
            case 2: OZB_PROVE(2); break;
            case 3: OZB_PROVE(3); break;
            default: OZB_PROVE(4); break;
        }
#undef OZB_PROVE
        OZB_CHECK(cudaGetLastError());
        span_end(h);
        OZB_TRY(read_status(res));
    }
    if (res.status == 1) {
        *done = true;
        *nA = res.ns0;
        *nB = res.ns1;
        *ret = res.result;
    } else if (st->env.dot_trace) {
        fprintf(stderr, "cuozblas: one-pass NearSum dot not used (n=%d)\n", n);
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
