// dot_i8.cu — pass 2 of the plain-form DOT on the INT8 tensor cores.
//
// After pass 1 (dot_fused.cu) the chain of each vector is the predicted one:
// level s rounds to the grid g_s = 2^(G0 - s d), d = 54 - rho, and slice s of
// an element is a_s g_s with an integer |a_s| <= 2^(d-1).  The reference's
// pair products P(ia, ib) = sum_k x_ia[k] y_ib[k] are exact, so they equal
// g_ia g_ib sum_k a_ia[k] b_ib[k] computed in integers, whatever the order.
// This pass computes those integer sums on tcgen05:
//
//  * digits: a thread cuts E consecutive elements level by level as the tree
//    cut does (t_s = base + sigma_s; within a group of G levels one base).
//    Because ulp(sigma_s) = g_s, the low 32 bits of t_s hold the cumulative
//    integer RN_{g_s}(base) / g_s modulo 2^32, so a_s = lo(t_s) - lo(t_{s-1})
//    * 2^d (mod 2^32) with no conversion.  a_s is written as D balanced base-256
//    digits c_j in [-128, 127] (bytes of (a + 0x80808080) ^ 0x80808080), D = 2
//    for d <= 15 and 3 for d <= 23;
//  * operands: a chunk of 128 elements has RP digit rows (p = s D + j; RP = 16
//    for two digits, 32 for three), a job is 128 / RP chunks, and chunk c's
//    row p is row RP c + p of a 128 x 128-byte tile (128-byte swizzle); x's
//    tile is A and y's is B (x = y: B is A).  One M = N = 128, K = 128 product
//    (four tcgen05.mma of K = 32) gives diagonal RP x RP blocks that are the
//    per-chunk digit-pair sums (the other blocks are not read).  All jobs of a
//    CTA accumulate into one TMEM tile; at most 512 jobs per CTA keep every
//    INT32 sum below 2^30;
//  * exactness of the sums: sum_j 256^(i+j) T[(ia,i),(ib,j)] is the integer
//    pair sum (< 2^53 by the rho rule), converted exactly and scaled by the
//    power of two g_ia g_ib; pairs whose scale would leave the range where
//    the reference's FP64 products are exact make the result invalid (the
//    host then runs the general path);
//  * the proof of the predicted chain is the tree pass's, on integers:
//    level s holds if some |a_{s+1}| exceeds floor((thr_s + g_{s+1}) / g_{s+1}).
//
// CTA (one per SM): 3 producer groups of 4 warps, two 32 KiB stages per group.
// Each group cuts its jobs into its stages in turn, loading the next job's
// elements before cutting the current one; one thread of the group waits for
// its four warps (a per-stage mbarrier) and issues the group's MMAs into the
// group's own 128-column TMEM accumulator, so no other thread touches it.
// Proven levels are shared through DotScratch::proven at once, so warps stop
// voting on them.  The first group sums the three accumulators at the end.
// Every wait is bounded and every warp collective is reached by all lanes
// (exits are agreed by a warp vote); a timeout sets DotScratch::err and the
// result is not used.  The pass pays off from about 2^22 elements; shorter
// vectors take the FP64 tree pass.
#include "fused.h"
#include "ozb_internal.h"
#include "sum.cuh"
#include "tc05.cuh"

namespace ozb {

constexpr int kDiQuads = 3;                      // producer groups of 4 warps
constexpr int kDiStagesPerQuad = 2;              // each group fills its two stages in turn
constexpr int kDiStages = kDiQuads * kDiStagesPerQuad;
constexpr int kDiProducers = kDiQuads * 128;     // producer threads
constexpr int kDiThreads = kDiProducers;         // each group issues its own MMAs
constexpr int kDiTile = 128 * 128;               // 128 rows x 128 bytes
constexpr int kDiStage = 2 * kDiTile;            // A and B tiles
constexpr int kDiMaxJobs = 512;                  // per CTA: 128 * 512 products of at most 2^14 each
constexpr int kDiSmem = kDiStages * kDiStage + 1024 /*alignment slack*/;
constexpr uint64_t kDiWaitNs = 2000000000ull;   // 2 s without progress

// Bytes j of four digit words, j = 0..D-1, as D words (byte e = element e).
template <int D>
__device__ __forceinline__ void di_transpose4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t (&o)[D]) {
    const uint32_t t01 = __byte_perm(w0, w1, 0x5140), t23 = __byte_perm(w2, w3, 0x5140);
    o[0] = __byte_perm(t01, t23, 0x5410);
    o[1] = __byte_perm(t01, t23, 0x7632);
    if (D > 2) {
        const uint32_t u01 = __byte_perm(w0, w1, 0x7362), u23 = __byte_perm(w2, w3, 0x7362);
        o[D > 2 ? 2 : 0] = __byte_perm(u01, u23, 0x5410);
    }
}

// Cut E consecutive elements into all kDotLevels levels (levels past the
// plan only fill rows that are never read) and write their digit rows (row
// s D + j below `rows`, K bytes E u .. E u + E - 1; `rows` is the chunk's first
// row plus this thread's byte offset, `ub16` its 16-byte chunk index times 16,
// before the swizzle).  sk[s] = sigma_s + K g_s with K = 0x80808080: t = base
// + sk[s] is rounded on the same grid, and its low word is (RN_{g_s}(base) /
// g_s + K) mod 2^32, so w = lo(t_s) - lo(t_{s-1}) * 2^d + K * 2^d is a_s + K
// (at a group start lo(t_{s-1}) is taken as K); the bytes of w are the
// balanced digits of a_s plus 0x80 each, removed after the byte transpose.
// Every G levels the base becomes the remainder.  VOTE: levels still waiting
// for their proof (`pending`) are voted on with |a_s|.  No branch depends on
// data or on the plan inside the level loop.
template <int D, int E, int G, bool VOTE>
__device__ __forceinline__ void di_digits(const double (&v)[E], const double *sk, int d, const int *ith,
                                          uint32_t rows, unsigned pending, unsigned &prov) {
    static_assert(E == 4 || E == 8, "4 or 8 elements per thread");
    constexpr uint32_t K = 0x80808080u;
    const uint32_t kd = K << d;
    // the 128-byte swizzle XORs bits 4-6 of the address with the row's low 3
    // bits; `rows` has its own 16-byte chunk index there and row multiples of
    // 1024 above, so row r's address is (rows ^ ((r & 7) << 4)) + r * 128
    uint32_t bx[8];
#pragma unroll
    for (int k = 0; k < 8; k++) bx[k] = rows ^ (uint32_t)(k << 4);
    double base[E], tprev[E];
    uint32_t lop[E];
#pragma unroll
    for (int e = 0; e < E; e++) base[e] = v[e];
#pragma unroll
    for (int s = 0; s < kDotLevels; s++) {
        const double sg = sk[s];
        if (s > 0 && s % G == 0) {  // compile-time: the next group cuts the remainder
            const double sp = sk[s - 1];
#pragma unroll
            for (int e = 0; e < E; e++) base[e] = base[e] - (tprev[e] - sp);
        }
        uint32_t w[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const double tt = base[e] + sg;
            const uint32_t lo = (uint32_t)__double2loint(tt);
            w[e] = (s % G == 0) ? lo : lo - (lop[e] << d) + kd;
            lop[e] = lo;
            tprev[e] = tt;
        }
        if (VOTE && s >= 1) {
            bool hit = false;
            const int th = ith[s - 1];
#pragma unroll
            for (int e = 0; e < E; e++) hit |= abs((int)(w[e] - K)) > th;
            if ((pending >> (s - 1)) & 1u)
                if (__any_sync(0xffffffffu, hit)) prov |= 1u << (s - 1);
        }
        uint32_t lo4[D];
        di_transpose4<D>(w[0], w[1], w[2], w[3], lo4);
        if (E == 8) {
            uint32_t hi4[D];
            di_transpose4<D>(w[E == 8 ? 4 : 0], w[E == 8 ? 5 : 1], w[E == 8 ? 6 : 2], w[E == 8 ? 7 : 3], hi4);
#pragma unroll
            for (int j = 0; j < D; j++) {
                const int r = s * D + j;
                asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(bx[r & 7] + (uint32_t)(r * 128)),
                             "r"(lo4[j] ^ K), "r"(hi4[j] ^ K)
                             : "memory");
            }
        } else {
#pragma unroll
            for (int j = 0; j < D; j++) {
                const int r = s * D + j;
                asm volatile("st.shared.u32 [%0], %1;" ::"r"(bx[r & 7] + (uint32_t)(r * 128)), "r"(lo4[j] ^ K)
                             : "memory");
            }
        }
    }
}

template <int E>
__device__ __forceinline__ void di_load(const double *__restrict__ v, int64_t i0, int n, double (&o)[E]) {
    if (i0 + E <= n) {
        const double2 *p = reinterpret_cast<const double2 *>(v + i0);
#pragma unroll
        for (int h = 0; h < E / 2; h++) {
            const double2 q = __ldcs(p + h);
            o[2 * h] = q.x;
            o[2 * h + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < E; e++) o[e] = i0 + e < n ? v[i0 + e] : 0.0;
    }
}

// The pairs from the digit sums, the scale check, then FSum / NearSum (one
// thread of the last CTA).
__device__ void di_finish(DotScratch *sc, const TreePlan &pl, bool same, int sum_mode, int D, double *Pv,
                          double *tmp) {
    const int nA = pl.ns[0], nB = same ? pl.ns[0] : pl.ns[1];
    const int gx0 = pl.G0[0], gy0 = same ? pl.G0[0] : pl.G0[1];
    int ok = __ldcg(&sc->err) == 0;
    for (int i = 0; i < kDotLevels * kDotLevels; i++) Pv[i] = 0.0;
    for (int ia = 0; ia < nA; ia++)
        for (int ib = 0; ib < nB; ib++) {
            long long S = 0;
            for (int i = 0; i < D; i++)
                for (int j = 0; j < D; j++)
                    S += __ldcg(&sc->T[(ia * D + i) * kDotDigitRows + ib * D + j]) * (1LL << (8 * (i + j)));
            const int e = (gx0 - ia * pl.d) + (gy0 - ib * pl.d);
            if (e < -1074 || e > 971 || S > (1LL << 53) || S < -(1LL << 53)) ok = 0;
            Pv[ia * kDotLevels + ib] = (double)S * pow2(e);
        }
    // why a result is not used (traced by the host): 1 plan, 2 wait, 4 scale, 8 / 16 proof of x / y
    int why = (pl.valid ? 0 : 1) | (__ldcg(&sc->err) ? 2 : 0) | (ok || __ldcg(&sc->err) ? 0 : 4);
    for (int v = 0; v < (same ? 1 : 2); v++)
        if ((__ldcg(&sc->proven[v]) & pl.need[v]) != pl.need[v]) why |= 8 << v;
    const int valid = why == 0;
    sc->out.pad = why;
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

// RP digit rows per chunk of 128 elements: 16 (two digits, up to 8 levels) or
// 32 (three digits, up to 8 levels); a job is 128 / RP chunks.
template <bool SAME, int D, int RP, int G>
__global__ void __launch_bounds__(kDiThreads, 1)
    k_dot_i8(int n, const double *__restrict__ x, const double *__restrict__ y, int rho, int maxS, int sum_mode,
             DotScratch *__restrict__ sc, const int *__restrict__ gate) {
    constexpr int CH = 128 / RP;   // chunks per job
    constexpr int JOB = 128 * CH;  // elements per job
    constexpr int E = CH;          // elements per producer thread (128 threads per job)
    constexpr int LPC = 128 / E;   // threads per chunk
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    extern __shared__ uint8_t di_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)di_raw + 1023) & ~(uintptr_t)1023);
    __shared__ TreePlan pl;
    __shared__ __align__(8) uint64_t full[kDiStages], empty[kDiStages], done;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ unsigned long long red[RP * RP];
    __shared__ double fin[2][kDotLevels * kDotLevels];
    __shared__ int last;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    __shared__ double sk[2][kDotLevels];
    plan_in_block(&sc->vs, rho, maxS, SAME, pl);
    for (int i = t; i < RP * RP; i += kDiThreads) red[i] = 0ull;
    __syncthreads();
    if (t < 2 * kDotLevels) {  // sigma_s + 0x80808080 g_s: exact (an integer below 2^53 times g_s)
        const int v = t / kDotLevels, s = t % kDotLevels;
        sk[v][s] = pl.sig[v][s] + 2155905152.0 * pow2(pl.G0[v] - s * pl.d);
    }
    __syncthreads();
    const int L = pl.L;
    const bool work = pl.valid != 0 && L * D <= RP;  // (L * D > RP cannot happen for a valid plan)
    // (the group size G is the plan's, chain_group(rho, 4); the launch picks it)
    const int64_t njobs = ((int64_t)n + JOB - 1) / JOB;
    const int myjobs = work && blockIdx.x < njobs ? (int)((njobs - 1 - blockIdx.x) / gridDim.x + 1) : 0;

    if (t == 0) {
        for (int q = 0; q < kDiStages; q++) {
            tc::mbar_init(&full[q], 4);  // one arrival per warp of the group
            tc::mbar_init(&empty[q], 1);
        }
        tc::mbar_init(&done, kDiQuads);
        abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, 512);  // one 128-column accumulator per group
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = tmem_slot;
    unsigned prov[2] = {0u, 0u};  // per warp (uniform)

    if (t < kDiProducers) {
        // ------------------------------------------------------------ producers
        const int quad = t >> 7, tq = t & 127;
        const int c = tq / LPC, u = tq % LPC;
        const int rowoff = RP * c * 128 + (E == 8 ? (u & 1) << 3 : (u & 3) << 2);
        const int ub16 = (E == 8 ? u >> 1 : u >> 2) << 4;
        const int d = pl.d;
        auto first = [&](int i) {
            return ((int64_t)blockIdx.x + (int64_t)i * gridDim.x) * JOB + c * 128 + E * u;
        };
        const uint32_t idesc = tc::idesc_i8(128, 128);
        const uint32_t acc = tmem_base + 128 * quad;  // this group's accumulator columns
        // job k of this group (i = quad + k * kDiQuads), elements in xv / yv;
        // thread 0 of the group issues the group's MMAs once all its warps
        // have written the stage (group barrier 1 + quad)
        auto produce = [&](int k, const double (&xv)[E], const double (&yv)[E]) -> bool {
            const int st = quad * kDiStagesPerQuad + (k & 1);
            // every lane leaves on the same job (the warp collectives below need all lanes)
            const bool ok = tc::mbar_wait(&empty[st], ((k >> 1) & 1) ^ 1, &abort_flag, &sc->err, 1, kDiWaitNs);
            if (!__all_sync(0xffffffffu, ok)) return false;
            uint8_t *tileA = smem + st * kDiStage;
            const uint32_t ra = tc::smem_u32(tileA) + rowoff + ub16;
#pragma unroll
            for (int v = 0; v < (SAME ? 1 : 2); v++) {
                // prov is uniform across the warp (the vote variant's __any_sync
                // needs every lane on the same path): lane 0's read of the levels
                // other warps proved is broadcast to all lanes
                unsigned pend = pl.need[v] & ~prov[v];
                if (pend) {  // uniform: levels some other warp proved need no vote here
                    prov[v] |= __shfl_sync(0xffffffffu, __ldcg(&sc->proven[v]), 0);
                    pend = pl.need[v] & ~prov[v];
                }
                const unsigned before = prov[v];
                if (pend)
                    di_digits<D, E, G, true>(v ? yv : xv, sk[v], d, pl.ith[v], ra + v * kDiTile, pend, prov[v]);
                else
                    di_digits<D, E, G, false>(v ? yv : xv, sk[v], d, pl.ith[v], ra + v * kDiTile, 0u, prov[v]);
                if (lane == 0 && prov[v] != before) atomicOr(&sc->proven[v], prov[v]);  // share at once
            }
            tc::fence_proxy_async();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&full[st]);
            // the group's issuer, once all four warps have written the stage; on a
            // timeout it issues nothing (the abort flag then stops every wait)
            if (tq == 0 && tc::mbar_wait(&full[st], (k >> 1) & 1, &abort_flag, &sc->err, 2, kDiWaitNs)) {
                tc::fence_after_sync();
                const uint32_t sa = tc::smem_u32(tileA), sb = SAME ? sa : sa + kDiTile;
                const uint64_t adesc = tc::smem_desc_k_sw128(sa), bdesc = tc::smem_desc_k_sw128(sb);
#pragma unroll
                for (int kk = 0; kk < 4; kk++)  // +32 bytes along K = +2 in 16-byte units
                    tc::mma_i8(acc, adesc + 2 * kk, bdesc + 2 * kk, idesc, (k > 0 || kk > 0) ? 1u : 0u);
                tc::mma_commit(&empty[st]);
            }
            return true;
        };
        // two register sets: the next job's elements load while this one is cut
        double xa[E], ya[E], xb[E], yb[E];
#pragma unroll
        for (int e = 0; e < E; e++) xa[e] = ya[e] = xb[e] = yb[e] = 0.0;
        if (quad < myjobs) {
            di_load<E>(x, first(quad), n, xa);
            if (!SAME) di_load<E>(y, first(quad), n, ya);
        }
        for (int k = 0, i = quad; i < myjobs; k += 2, i += 2 * kDiQuads) {
            if (i + kDiQuads < myjobs) {
                di_load<E>(x, first(i + kDiQuads), n, xb);
                if (!SAME) di_load<E>(y, first(i + kDiQuads), n, yb);
            }
            if (!produce(k, xa, ya)) break;
            if (i + kDiQuads >= myjobs) break;
            if (i + 2 * kDiQuads < myjobs) {
                di_load<E>(x, first(i + 2 * kDiQuads), n, xa);
                if (!SAME) di_load<E>(y, first(i + 2 * kDiQuads), n, ya);
            }
            if (!produce(k + 1, xb, yb)) break;
        }
        if (tq == 0) {
            tc::mma_commit(&done);  // also when nothing was issued or the group gave up
            // every MMA of this group completes before TMEM is released (bounded)
            const uint64_t t0 = tc::globaltimer();
            while (!tc::mbar_try_wait(&done, 0) && tc::globaltimer() - t0 < 100000000ull) {
            }
        }
    }

    // ---------------------------------------------------------------- accumulator
    __syncwarp();
    if (warp < 4 && myjobs > 0) {
        // tcgen05.ld is warp-collective: every lane takes the same branch
        const bool ok = tc::mbar_wait(&done, 0, &abort_flag, &sc->err, 3, kDiWaitNs) && !abort_flag;
        if (__all_sync(0xffffffffu, ok)) {
            tc::fence_after_sync();
            long long sum[32];
#pragma unroll
            for (int q = 0; q < 32; q++) sum[q] = 0;
            for (int g = 0; g < kDiQuads && g < myjobs; g++) {  // groups that ran a job
                uint32_t v[32];
                tc::tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(32 * warp) << 16) + 128 * g + 32 * warp, v);
                tc::tmem_ld_wait();
#pragma unroll
                for (int q = 0; q < 32; q++) sum[q] += (long long)(int)v[q];
            }
            const int rows = L * D;
            // lane l holds TMEM row 32 warp + l: chunk c, digit row p; its
            // diagonal block starts at column RP c
            const int p = lane % RP, off = RP == 16 ? 16 * (lane >> 4) : 0;
            if (p < rows) {
#pragma unroll
                for (int q = 0; q < RP; q++) {
                    const long long val = off ? sum[(16 + q) & 31] : sum[q & 31];
                    if (q < rows && val != 0) atomicAdd(&red[p * RP + q], (unsigned long long)val);
                }
            }
        }
    }
    if (lane == 0) {
        if (prov[0]) atomicOr(&sc->proven[0], prov[0]);
        if (!SAME && prov[1]) atomicOr(&sc->proven[1], prov[1]);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, 512);
    }
    for (int i = t; i < RP * RP; i += kDiThreads)
        if (red[i])
            atomicAdd(reinterpret_cast<unsigned long long *>(&sc->T[(i / RP) * kDotDigitRows + i % RP]), red[i]);
    // the last CTA forms the pairs and sums them
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (t == 0) di_finish(sc, pl, SAME, sum_mode, D, fin[0], fin[1]);
    __syncthreads();
    // leave the accumulators zeroed for the next use (replayed graphs skip the memset)
    for (int i = t; i < kDotDigitRows * kDotDigitRows; i += kDiThreads) sc->T[i] = 0;
    if (t == 0) {
        sc->proven[0] = sc->proven[1] = 0u;
        sc->ticket = 0u;
        sc->err = 0;
        sc->vs = VecStats{};  // every CTA has read the statistics (the ticket comes after)
    }
}

// Digits per level for rho (0: the tensor-core pass does not apply).
int dot_i8_digits(int rho) {
    const int d = 54 - rho, G = chain_group(rho, 4);
    if (d <= 15) return (G == 3 || G == 4) ? 2 : 0;
    if (d <= 23) return (G == 2 || G == 3) ? 3 : 0;
    return 0;
}

template <bool SAME, int D, int G>
static int launch_i8(int grid, cudaStream_t s, int n, const double *x, const double *y, int rho, int maxS,
                     int sum_mode, DotScratch *sc, const int *gate) {
    constexpr int RP = D == 2 ? 16 : 32;
    static std::atomic<uint64_t> attr{0};  // devices already opted in, per instantiation
    if (smem_optin((const void *)k_dot_i8<SAME, D, RP, G>, kDiSmem, attr) != cudaSuccess)
        return CUOZBLAS_STATUS_CUDA_ERROR;
    k_dot_i8<SAME, D, RP, G><<<grid, kDiThreads, kDiSmem, s>>>(n, x, y, rho, maxS, sum_mode, sc, gate);
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

template <bool SAME>
static int prepare_i8() {
    int r = 0;
    r |= cudaFuncSetAttribute(k_dot_i8<SAME, 2, 16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiSmem);
    r |= cudaFuncSetAttribute(k_dot_i8<SAME, 2, 16, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiSmem);
    r |= cudaFuncSetAttribute(k_dot_i8<SAME, 3, 32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiSmem);
    r |= cudaFuncSetAttribute(k_dot_i8<SAME, 3, 32, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiSmem);
    return r;
}

int dot_i8_prepare() {
    return (prepare_i8<true>() | prepare_i8<false>()) ? CUOZBLAS_STATUS_CUDA_ERROR : CUOZBLAS_STATUS_SUCCESS;
}

template <bool SAME>
static int launch_i8_g(int D, int G, int grid, cudaStream_t s, int n, const double *x, const double *y, int rho,
                       int maxS, int sum_mode, DotScratch *sc, const int *gate) {
    if (D == 2 && G == 3) return launch_i8<SAME, 2, 3>(grid, s, n, x, y, rho, maxS, sum_mode, sc, gate);
    if (D == 2 && G == 4) return launch_i8<SAME, 2, 4>(grid, s, n, x, y, rho, maxS, sum_mode, sc, gate);
    if (D == 3 && G == 2) return launch_i8<SAME, 3, 2>(grid, s, n, x, y, rho, maxS, sum_mode, sc, gate);
    if (D == 3 && G == 3) return launch_i8<SAME, 3, 3>(grid, s, n, x, y, rho, maxS, sum_mode, sc, gate);
    return CUOZBLAS_STATUS_INVALID_VALUE;
}

int dot_i8_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, int rho, int maxS,
                  int sum_mode, DotScratch *sc, const int *gate) {
    const int D = dot_i8_digits(rho);
    const int G = chain_group(rho, 4);  // levels cut from one base value, as the tree pass
    const int job = D == 2 ? 1024 : 512;
    const int64_t njobs = ((int64_t)n + job - 1) / job;
    int64_t grid = njobs < nsm ? njobs : nsm;
    const int64_t need = (njobs + kDiMaxJobs - 1) / kDiMaxJobs;
    if (grid < need) grid = need;
    if (grid < 1) grid = 1;
    return x == y ? launch_i8_g<true>(D, G, (int)grid, s, n, x, y, rho, maxS, sum_mode, sc, gate)
                  : launch_i8_g<false>(D, G, (int)grid, s, n, x, y, rho, maxS, sum_mode, sc, gate);
}

}  // namespace ozb
