// gemm_i8.cu — INT8 precision form of the Ozaki DGEMM on tcgen05 tensor cores.
//
// This form has no reference implementation (the reference stubs an integer
// path at src/cuda/cuozblas_gemm.cu:292 and src/cuda/cuozblas_common.h:53-56).
//
// Split: each line (row of op(A), column of op(B)) gets an exponent E with
// max|x| < 2^E; x * 2^-E in (-1, 1) is cut into base-2^7 digits by
// truncation, d_s = trunc(r * 128), r <- r * 128 - d_s, so every digit is an
// int8 in [-127, 127] with the sign of x and
//     x = 2^E * sum_s d_s 2^(-7(s+1))   (exact once enough digits are kept).
// Products: C(i,j) = 2^(EA_i + EB_j) * sum_L 2^(-7(L+2)) V_L(i,j) with
// V_L = sum over digit pairs ia + ib = L of the int8 dot products.  All pairs
// of one level share the scale, so they accumulate in one INT32 tensor-memory
// accumulator; a group holds at most floor((2^31 - 1) / (127^2)) products per
// output, which keeps every partial sum exact (k is chunked beyond that).
// Sum: levels are visited from the largest (L = 0) to the smallest.  Runs of
// consecutive levels, formed from level 0 upward, are first combined
// exactly, as an integer below 2^53 held in an FP64 register (V_L shifted by
// 7 bits per level); each run is then added once to the FP64 sum R, which
// lives in tensor memory, the most significant run first.  A cancellation
// between runs therefore happens while R is still exact (the difference of
// the two leading runs is representable), and each later run, 2^-28 or less
// of R, moves it by at most one rounding: with a complete split the output
// is within one ulp of the correctly rounded product, also when the exact
// value is far smaller than its products.  Finally t = R * 2^(EA_i + EB_j)
// and C = fma(alpha, t, beta * C).
//
// Kernel: persistent, one CTA per SM, warp-specialised:
//   warp 0      TMA producer (128 x 128-byte tiles, 128-byte swizzle)
//   warp 1      TMEM allocator and single-thread tcgen05.mma issuer
//   warps 2-9   epilogue: tcgen05.ld of the INT32 level sums, FP64 sum, store
// Two 128-column TMEM accumulators let the epilogue of one level overlap the
// MMAs of the next; the other 256 columns hold R.  Every mbarrier wait is bounded (global timer) and shares
// an abort flag; a timeout reports CUOZBLAS_STATUS_DEVICE_TIMEOUT.
#include <cuda.h>

#include <mutex>
#include <vector>

#include <algorithm>

#include "autotune.h"
#include "gemm_i8_blk.h"
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "tc05.cuh"

namespace ozb {

constexpr int I8_BM = 128, I8_BN = 128, I8_BK = 128, I8_NST = 6;
constexpr int I8_THREADS = 320;
constexpr int I8_TMEM_COLS = 512;     // 2 x 128 INT32 accumulators + 128 x 128 FP64 sums
constexpr int I8_RCOL = 2 * 128;      // first column of the FP64 sums
constexpr int I8_TILE_A = I8_BM * I8_BK, I8_TILE_B = I8_BN * I8_BK, I8_STAGE = I8_TILE_A + I8_TILE_B;
constexpr int I8_SMEM = I8_NST * I8_STAGE + 1024 /*align slack*/ + 256 /*barriers*/;
constexpr int64_t I8_MAX_TERMS = 2147483647LL / (127 * 127);  // 133143 int8 products per INT32 sum
constexpr uint64_t I8_WAIT_NS = 2000000000ull;                  // 2 s per wait

enum { ERR_TIMEOUT_PRODUCER = 1, ERR_TIMEOUT_MMA = 2, ERR_TIMEOUT_EPI = 3 };

// Limit of every bounded mbarrier wait in k_i8_gemm, and a test switch that
// makes its producer issue no copies, so that the MMA issuer's first wait
// runs out (set by cuozblasSetI8WaitTest; tests only).
__device__ uint64_t g_i8_wait_ns = I8_WAIT_NS;
__device__ int g_i8_hold_copies = 0;
// host copies, passed to the level-blocked kernel (gemm_i8_blk.cu) as parameters
static std::atomic<uint64_t> h_i8_wait_ns{I8_WAIT_NS};
static std::atomic<int> h_i8_hold_copies{0};
uint64_t i8_test_wait_ns() { return h_i8_wait_ns.load(); }
int i8_test_hold_copies() { return h_i8_hold_copies.load(); }

struct I8Params {
    int m, n, m_pad, n_pad, ldc;
    int tiles_m, tiles_n, n_items, n_groups;
    int strip;           // tile rows per rasterisation strip
    const int4 *items;   // {ia, ib, kb0, kb1} in processing order
    const int4 *groups;  // {item_begin, item_end, flush scale exponent, meta: shift | flush<<8 | first<<9 | last<<10}
    const int *ea, *eb;  // line exponents
    // MODE 1 (the <double,float,float> form): slice exponents per level and line,
    // [s][m] and [s][n], and the common scale 2 (rho - 53) of an INT8 slice product
    const short *eas, *ebs;
    int sbias;
    // MODE 2 (exact FP64 pair products of digit-cut slices) writes the pair
    // buffer [pair][n][m] through C and reads the digit planes per slice level
    // from ldc (no new fields: a larger parameter block makes MODE 0 spill more);
    // eas/ebs (or null) add tauA + tauB per element
    double alpha, beta;
    double *C;
    int *err;
};

// Tile order: strips of `strip` tile rows, column-major inside a strip, so
// the CTAs resident at one time share A and B panels in L2.
__device__ __forceinline__ void tile_coords(int tile, const I8Params &p, int &tm, int &tn) {
    const int per_strip = p.strip * p.tiles_n;
    const int s = tile / per_strip, w = tile - s * per_strip;
    const int rows = min(p.strip, p.tiles_m - s * p.strip);
    tm = s * p.strip + w % rows;
    tn = w / rows;
}

// MODE 0: the precision form (level groups, runs, correctly rounded sum).
// MODE 2: exact FP64 products of slice pairs whose slices are cut into int8
// digits: a group is one (pair, digit level L) with the INT32 products of its
// digit pairs; the epilogue adds W 2^(group.w >> 8) to its FP64 sums (exact:
// every partial sum of the pair is an integer below 2^53) and at the pair's
// last level (group.w & 1) stores scalbn(sum, sbias) to pbuf[pair][col][row].
// MODE 1: the mixed form <double,float,float> with INT8 slices (each group is
// one slice pair; its exact INT32 product V is added as scalbn(V, tauA + tauB +
// sbias) to the FP64 sums in pair order, then C = fma(alpha, t, beta C)).
template <int MODE>
__global__ void __launch_bounds__(I8_THREADS, 1)
    k_i8_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, I8Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *bar = (uint64_t *)(smem + I8_NST * I8_STAGE);
    uint64_t *full = bar, *empty = bar + I8_NST, *acc_full = bar + 2 * I8_NST, *acc_empty = bar + 2 * I8_NST + 2;
    uint64_t *drain = bar + 2 * I8_NST + 4;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = p.tiles_m * p.tiles_n;
    const uint64_t wait_ns = g_i8_wait_ns;

    if (threadIdx.x == 0) {
        for (int s = 0; s < I8_NST; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&acc_full[b], 1);
            tc::mbar_init(&acc_empty[b], 256);
        }
        tc::mbar_init(drain, 1);
        abort_flag = 0;
        tc::fence_mbar_init();
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, I8_TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t stage = 0, phase = 0;
            uint32_t issued = 0, issued_phase = 0;  // per stage: a copy was issued, and the phase it completes
            bool ok = g_i8_hold_copies == 0;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int tm, tn;
                tile_coords(tile, p, tm, tn);
                for (int it = 0; it < p.n_items && ok; it++) {
                    const int4 item = p.items[it];
                    for (int kb = item.z; kb < item.w; kb++) {
                        if (!tc::mbar_wait(&empty[stage], phase ^ 1, &abort_flag, p.err, ERR_TIMEOUT_PRODUCER,
                                           wait_ns)) {
                            ok = false;
                            break;
                        }
                        uint8_t *sa = smem + stage * I8_STAGE, *sb = sa + I8_TILE_A;
                        tc::mbar_arrive_expect_tx(&full[stage], I8_STAGE);
                        tc::tma_load_2d(sa, &tmA, &full[stage], kb * I8_BK, item.x * p.m_pad + tm * I8_BM);
                        tc::tma_load_2d(sb, &tmB, &full[stage], kb * I8_BK, item.y * p.n_pad + tn * I8_BN);
                        issued |= 1u << stage;
                        issued_phase = (issued_phase & ~(1u << stage)) | (phase << stage);
                        if (++stage == I8_NST) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
            }
            if (!ok) tc::drain_copies(full, I8_NST, issued, issued_phase);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(I8_BM, I8_BN);
            uint32_t stage = 0, phase = 0, abuf = 0, aphase = 0;
            bool ok = true, issued = false;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                for (int g = 0; g < p.n_groups && ok; g++) {
                    const int4 grp = p.groups[g];
                    if (!tc::mbar_wait(&acc_empty[abuf], aphase ^ 1, &abort_flag, p.err, ERR_TIMEOUT_MMA,
                                       wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t tmem_d = tmem_base + abuf * I8_BN;
                    uint32_t accumulate = 0;
                    for (int it = grp.x; it < grp.y && ok; it++) {
                        const int4 item = p.items[it];
                        for (int kb = item.z; kb < item.w; kb++) {
                            if (!tc::mbar_wait(&full[stage], phase, &abort_flag, p.err, ERR_TIMEOUT_MMA,
                                               wait_ns)) {
                                ok = false;
                                break;
                            }
                            tc::fence_after_sync();
                            const uint32_t sa = tc::smem_u32(smem + stage * I8_STAGE), sb = sa + I8_TILE_A;
                            const uint64_t adesc = tc::smem_desc_k_sw128(sa), bdesc = tc::smem_desc_k_sw128(sb);
#pragma unroll
                            for (int kk = 0; kk < I8_BK / 32; kk++) {
                                // +32 bytes along K inside the 128-byte swizzle row = +2 in 16-byte units
                                tc::mma_i8(tmem_d, adesc + 2 * kk, bdesc + 2 * kk, idesc, accumulate);
                                accumulate = 1;
                            }
                            issued = true;
                            tc::mma_commit(&empty[stage]);
                            if (++stage == I8_NST) {
                                stage = 0;
                                phase ^= 1;
                            }
                        }
                    }
                    if (!ok) break;
                    tc::mma_commit(&acc_full[abuf]);
                    abuf ^= 1;
                    if (abuf == 0) aphase ^= 1;
                }
            }
            if (!ok && issued) {  // drain MMAs still in flight before TMEM is released
                tc::mma_commit(drain);
                const uint64_t t0 = tc::globaltimer();
                while (!tc::mbar_try_wait(drain, 0) && tc::globaltimer() - t0 < 100000000ull) {
                }
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3, half = (warp - 2) >> 2;
        const int row = q * 32 + lane;
        const uint32_t lane_base = tmem_base + ((uint32_t)(q * 32) << 16);
        const uint32_t rcol = I8_RCOL + half * 128;  // this thread's 64 FP64 sums (lo, hi word pairs)
        uint32_t abuf = 0, aphase = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            int tm, tn;
            tile_coords(tile, p, tm, tn);
            const int gr = tm * I8_BM + row;
            double acc[64];  // exact integer-valued run of levels (< 2^53)
#pragma unroll
            for (int c = 0; c < 64; c++) acc[c] = 0.0;
            for (int g = 0; g < p.n_groups; g++) {
                const int4 grp = p.groups[g];
                const int meta = grp.w;
                // MODE 1: the pair's exponents do not depend on the MMAs, so they are
                // loaded before the wait and arrive while the accumulator fills
                int era = 0, eb0 = 0, eb1 = 0;
                if constexpr (MODE == 1) {
                    const int4 pr = p.items[grp.x];
                    era = (gr < p.m ? (int)p.eas[(size_t)pr.x * p.m + gr] : 0) + p.sbias;
                    const short *ebr = p.ebs + (size_t)pr.y * p.n;
                    const int c0 = tn * I8_BN + half * 64 + lane, c1 = c0 + 32;
                    eb0 = c0 < p.n ? (int)__ldg(ebr + c0) : 0;
                    eb1 = c1 < p.n ? (int)__ldg(ebr + c1) : 0;
                }
                bool wok = tc::mbar_wait(&acc_full[abuf], aphase, &abort_flag, p.err, ERR_TIMEOUT_EPI, wait_ns);
                if constexpr (MODE == 1) wok = __all_sync(0xffffffffu, wok);  // the lanes agree before any shuffle
                if (!wok) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t taddr = lane_base + abuf * I8_BN + half * 64;
                uint32_t v[32];
                if constexpr (MODE == 2) {
                    const double sc = pow2(grp.w >> 8);
#pragma unroll
                    for (int hh = 0; hh < 2; hh++) {
                        tc::tmem_ld_32x32b_x32(taddr + 32 * hh, v);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int c = 0; c < 32; c++)
                            acc[32 * hh + c] = __dadd_rn(acc[32 * hh + c], __dmul_rn((double)(int32_t)v[c], sc));
                    }
                    tc::fence_before_sync();
                    tc::mbar_arrive(&acc_empty[abuf]);
                    abuf ^= 1;
                    if (abuf == 0) aphase ^= 1;
                    if (grp.w & 1) {  // the pair is complete
                        if (gr < p.m) {
                            const int4 it = p.items[grp.x];
                            const short *ebr = p.ebs ? p.ebs + (size_t)(it.y / p.ldc) * p.n : nullptr;
                            const int er = p.sbias + (p.eas ? (int)p.eas[(size_t)(it.x / p.ldc) * p.m + gr] : 0);
#pragma unroll
                            for (int c = 0; c < 64; c++) {
                                const int gc = tn * I8_BN + half * 64 + c;
                                if (gc < p.n)
                                    p.C[((size_t)grp.z * p.n + gc) * p.m + gr] =
                                        scale2(acc[c], er + (ebr ? (int)ebr[gc] : 0));
                            }
                        }
#pragma unroll
                        for (int c = 0; c < 64; c++) acc[c] = 0.0;
                    }
                    continue;
                }
                if constexpr (MODE == 1) {
                    // the warp's 64 columns are the same for all its lanes: lane l holds the
                    // exponents of columns gc0 + l and gc0 + 32 + l, shuffles hand them round
                    const int ebmin = __reduce_min_sync(0xffffffffu, eb0 < eb1 ? eb0 : eb1);
                    const int ebmax = __reduce_max_sync(0xffffffffu, eb0 > eb1 ? eb0 : eb1);
                    // V * 2^e is exact (normal) for |V| < 2^31 and e in [-1000, 1000]: one multiply
                    const bool fast = __all_sync(0xffffffffu, era + ebmin >= -1000 && era + ebmax <= 1000);
#pragma unroll
                    for (int hh = 0; hh < 2; hh++) {
                        tc::tmem_ld_32x32b_x32(taddr + 32 * hh, v);
                        tc::tmem_ld_wait();
                        const int ebh = hh ? eb1 : eb0;
                        if (fast) {
#pragma unroll
                            for (int c = 0; c < 32; c++) {
                                const int e = era + __shfl_sync(0xffffffffu, ebh, c);
                                acc[32 * hh + c] = __dadd_rn(acc[32 * hh + c],
                                                             __dmul_rn((double)(int32_t)v[c],
                                                                       from_bits((uint64_t)(e + 1023) << 52)));
                            }
                        } else {
#pragma unroll
                            for (int c = 0; c < 32; c++) {
                                const int e = era + __shfl_sync(0xffffffffu, ebh, c);
                                acc[32 * hh + c] = __dadd_rn(acc[32 * hh + c], scale2((double)(int32_t)v[c], e));
                            }
                        }
                    }
                    tc::fence_before_sync();
                    tc::mbar_arrive(&acc_empty[abuf]);
                    abuf ^= 1;
                    if (abuf == 0) aphase ^= 1;
                    continue;
                }
                const double sc = pow2(meta & 0xff);
                tc::tmem_ld_32x32b_x32(taddr, v);
                tc::tmem_ld_wait();
#pragma unroll
                for (int c = 0; c < 32; c++) acc[c] += (double)(int32_t)v[c] * sc;
                tc::tmem_ld_32x32b_x32(taddr + 32, v);
                tc::tmem_ld_wait();
#pragma unroll
                for (int c = 0; c < 32; c++) acc[32 + c] += (double)(int32_t)v[c] * sc;
                tc::fence_before_sync();
                tc::mbar_arrive(&acc_empty[abuf]);
                abuf ^= 1;
                if (abuf == 0) aphase ^= 1;
                if (meta & (1 << 8)) {  // end of a run: R += acc * 2^(exponent)
                    const double fs = pow2(grp.z);
                    const bool first = meta & (1 << 9), last = meta & (1 << 10);
                    // the exact rounding error of R + run goes into the next run's
                    // accumulator (scaled to its units), so R + carries stays exact
                    const double cs = last ? 0.0 : pow2(32768 - ((meta >> 16) & 0xffff));
#pragma unroll
                    for (int ch = 0; ch < 4; ch++) {
                        const uint32_t raddr = lane_base + rcol + ch * 32;
                        uint32_t u[32];
                        double r[16];
                        if (first) {
#pragma unroll
                            for (int e = 0; e < 16; e++) {
                                r[e] = acc[ch * 16 + e] * fs;
                                acc[ch * 16 + e] = 0.0;
                            }
                        } else {
                            tc::tmem_ld_32x32b_x32(raddr, u);
                            tc::tmem_ld_wait();
#pragma unroll
                            for (int e = 0; e < 16; e++) {
                                const double ro = __hiloint2double((int)u[2 * e + 1], (int)u[2 * e]);
                                const double a = acc[ch * 16 + e] * fs;
                                const double sm = ro + a;
                                const double bb = sm - ro;
                                acc[ch * 16 + e] = ((ro - (sm - bb)) + (a - bb)) * cs;  // TwoSum error
                                r[e] = sm;
                            }
                        }
                        if (last) {
                            if (gr < p.m) {
                                const int ea = p.ea[gr];
#pragma unroll
                                for (int e = 0; e < 16; e++) {
                                    const int gc = tn * I8_BN + half * 64 + ch * 16 + e;
                                    if (gc < p.n) {
                                        double *cp = &p.C[(size_t)gc * p.ldc + gr];
                                        const double t = scalbn(r[e], ea + p.eb[gc]);
                                        *cp = fma(p.alpha, t, p.beta * *cp);
                                    }
                                }
                            }
                        } else {
#pragma unroll
                            for (int e = 0; e < 16; e++) {
                                u[2 * e] = (uint32_t)__double2loint(r[e]);
                                u[2 * e + 1] = (uint32_t)__double2hiint(r[e]);
                            }
                            tc::tmem_st_32x32b_x32(raddr, u);
                        }
                    }
                    if (!last) tc::tmem_st_wait();
                }
            }
            if constexpr (MODE == 1) {
                if (ok && gr < p.m) {
#pragma unroll
                    for (int c = 0; c < 64; c++) {
                        const int gc = tn * I8_BN + half * 64 + c;
                        if (gc < p.n) {
                            double *cp = &p.C[(size_t)gc * p.ldc + gr];
                            *cp = fma(p.alpha, acc[c], p.beta * *cp);
                        }
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, I8_TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// Digit split
// ---------------------------------------------------------------------------
__device__ __forceinline__ int exp_above(double v) {  // E with v < 2^E, v > 0
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    const int be = (int)(b >> 52);
    if (be == 0) {
        const uint64_t f = b & ((1ULL << 52) - 1);
        if (f == 0) return 0;
        return (63 - clz64(f)) - 1073;
    }
    return be - 1022;
}

__device__ __forceinline__ int lsb_exp(double v) {  // exponent of the lowest set bit, v != 0
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    const int be = (int)(b >> 52);
    uint64_t f = b & ((1ULL << 52) - 1);
    if (be == 0) return -1074 + __ffsll((long long)f) - 1;
    f |= (1ULL << 52);
    return (be - 1075) + __ffsll((long long)f) - 1;
}

// Line exponent E (max|x| < 2^E) and the digit count that makes the line
// exact, need = max over its nonzero x of ceil((E - lsb(x)) / 7) =
// ceil((E - min lsb) / 7): both statistics in one pass.
__device__ __forceinline__ void line_stat(double v, double &mx, int &lsb) {
    mx = ref_max(mx, fabs(v));
    if (v != 0.0) lsb = min(lsb, lsb_exp(v));
}
__device__ __forceinline__ int line_need(double mx, int lsb, int &E) {
    E = mx > 0.0 ? exp_above(mx) : 0;
    return mx > 0.0 ? (E - lsb + 6) / 7 : 0;
}

// k contiguous (element i of line l at X[l * ldx + i]): one CTA per line.
__global__ void __launch_bounds__(256) k_digit_count(int k, int nl, const double *__restrict__ X, int ldx,
                                                     int *__restrict__ e_out, int *__restrict__ need_max) {
    __shared__ double red[8];
    __shared__ int redi[8];
    const int line = blockIdx.x;
    const double *x = X + (size_t)line * ldx;
    double mx = 0.0;
    int lsb = 0x7fffffff;
    if ((reinterpret_cast<uintptr_t>(x) & 15) == 0) {
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        for (int i = threadIdx.x; i < (k >> 1); i += blockDim.x) {
            const double2 v = x2[i];
            line_stat(v.x, mx, lsb);
            line_stat(v.y, mx, lsb);
        }
        if ((k & 1) && threadIdx.x == 0) line_stat(x[k - 1], mx, lsb);
    } else {
        for (int i = threadIdx.x; i < k; i += blockDim.x) line_stat(x[i], mx, lsb);
    }
    mx = block_max_nonneg(mx, red);
    lsb = __reduce_min_sync(0xffffffffu, lsb);
    if ((threadIdx.x & 31) == 0) redi[threadIdx.x >> 5] = lsb;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) lsb = min(lsb, redi[w]);
        int E;
        const int need = line_need(mx, lsb, E);
        e_out[line] = E;
        atomicMax(need_max, need);
    }
}

// Lines contiguous (element i of line l at X[i * ldx + l], op(A) = A with A
// column-major): blocks of 128 lines x a slice of k, per-line partial results
// merged by atomics; the block that finishes last computes every line's E and
// the largest need.  mxb / lsbm / ticket start at 0 / above every exponent / 0.
__global__ void __launch_bounds__(256) k_digit_count_rows(int k, int nl, const double *__restrict__ X, int ldx,
                                                          unsigned long long *__restrict__ mxb, int *__restrict__ lsbm,
                                                          unsigned *__restrict__ ticket, int *__restrict__ e_out,
                                                          int *__restrict__ need_max) {
    __shared__ double smx[256];
    __shared__ int slsb[256];
    __shared__ int last;
    const int t = threadIdx.x, r = t & 127, l = blockIdx.x * 128 + r;
    const int kper = (k + gridDim.y - 1) / gridDim.y;
    const int kb = blockIdx.y * kper, ke = min(k, kb + kper);
    double mx = 0.0;
    int lsb = 0x7fffffff;
    if (l < nl) {
#pragma unroll 4
        for (int i = kb + (t >> 7); i < ke; i += 2) line_stat(X[(size_t)i * ldx + l], mx, lsb);
    }
    smx[t] = mx;
    slsb[t] = lsb;
    __syncthreads();
    if (t < 128 && l < nl) {
        mx = ref_max(smx[t], smx[t + 128]);
        lsb = min(slsb[t], slsb[t + 128]);
        if (mx > 0.0) atomicMax(&mxb[l], (unsigned long long)__double_as_longlong(mx));
        if (lsb != 0x7fffffff) atomicMin(&lsbm[l], lsb);
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(ticket, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    int nmax = 0;
    for (int i = t; i < nl; i += blockDim.x) {
        const double m = __longlong_as_double((long long)__ldcg(&mxb[i]));
        int E;
        const int nd = line_need(m, __ldcg(&lsbm[i]), E);
        e_out[i] = E;
        nmax = max(nmax, nd);
    }
    nmax = __reduce_max_sync(0xffffffffu, nmax);
    if ((t & 31) == 0) atomicMax(need_max, nmax);
}

// Digits: thread handles 16 consecutive k of one line; writes S slices of
// lines_pad x k_pad int8 (zero padded in both directions).  The digits are cut
// with integer operations (digit_cut), one 16-byte store per level.
__global__ void __launch_bounds__(256) k_digit_write(int k, int nl, int nl_pad, int k_pad, int S,
                                                     const double *__restrict__ X, int ldx,
                                                     const int *__restrict__ e_line, int8_t *__restrict__ out) {
    const int64_t chunk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int per_line = k_pad / 16;
    const int64_t total = (int64_t)nl_pad * per_line;
    if (chunk >= total) return;
    const int line = (int)(chunk / per_line), k0 = (int)(chunk % per_line) * 16;
    uint64_t m7[16];
    int f[16];
    uint32_t neg[4] = {0u, 0u, 0u, 0u};  // 0xff in the bytes of negative elements
    const int E = line < nl ? e_line[line] : 0;
    const double *x = X + (size_t)(line < nl ? line : 0) * ldx;
    if (line < nl && k0 + 16 <= k && ((reinterpret_cast<uintptr_t>(x + k0) & 15) == 0)) {
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(x + k0 + i);
            const DigitCut c0 = digit_cut(v.x, E), c1 = digit_cut(v.y, E);
            m7[i] = c0.m7;
            f[i] = c0.f;
            m7[i + 1] = c1.m7;
            f[i + 1] = c1.f;
            if (v.x < 0.0) neg[i >> 2] |= 0xffu << (8 * (i & 3));
            if (v.y < 0.0) neg[i >> 2] |= 0xffu << (8 * ((i + 1) & 3));
        }
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const double v = (line < nl && k0 + i < k) ? x[k0 + i] : 0.0;
            const DigitCut c = digit_cut(v, E);
            m7[i] = c.m7;
            f[i] = c.f;
            if (v < 0.0) neg[i >> 2] |= 0xffu << (8 * (i & 3));
        }
    }
    for (int s = 0; s < S; s++) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 16; i++) {
            w[i >> 2] |= digit_mag(m7[i], f[i]) << (8 * (i & 3));
            f[i] -= 7;
        }
        int4 *o = reinterpret_cast<int4 *>(out + ((size_t)s * nl_pad + line) * k_pad + k0);
        *o = make_int4((int)digits_signed(w[0], neg[0]), (int)digits_signed(w[1], neg[1]),
                       (int)digits_signed(w[2], neg[2]), (int)digits_signed(w[3], neg[3]));
    }
}

// Digits of lines contiguous in memory (element i of line l at X[i * ldx + l]):
// thread (line r of a 128-line tile, 16 consecutive k), loads coalesced across
// the lines, the same digits and layout as k_digit_write (no transposed copy).
__global__ void __launch_bounds__(256) k_digit_write_rows(int k, int nl, int nl_pad, int k_pad, int S,
                                                          const double *__restrict__ X, int ldx,
                                                          const int *__restrict__ e_line, int8_t *__restrict__ out) {
    const int t = threadIdx.x, line = blockIdx.x * 128 + (t & 127);
    const int k0 = (blockIdx.y * 2 + (t >> 7)) * 16;
    if (line >= nl_pad || k0 >= k_pad) return;
    uint64_t m7[16];
    int f[16];
    uint32_t neg[4] = {0u, 0u, 0u, 0u};
    const int E = line < nl ? e_line[line] : 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const double v = (line < nl && k0 + i < k) ? X[(size_t)(k0 + i) * ldx + line] : 0.0;
        const DigitCut c = digit_cut(v, E);
        m7[i] = c.m7;
        f[i] = c.f;
        if (v < 0.0) neg[i >> 2] |= 0xffu << (8 * (i & 3));
    }
    for (int s = 0; s < S; s++) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 16; i++) {
            w[i >> 2] |= digit_mag(m7[i], f[i]) << (8 * (i & 3));
            f[i] -= 7;
        }
        int4 *o = reinterpret_cast<int4 *>(out + ((size_t)s * nl_pad + line) * k_pad + k0);
        *o = make_int4((int)digits_signed(w[0], neg[0]), (int)digits_signed(w[1], neg[1]),
                       (int)digits_signed(w[2], neg[2]), (int)digits_signed(w[3], neg[3]));
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
typedef CUresult (*PFN_TensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                             const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                             const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_TensorMapEncodeTiled get_encode() {
    static PFN_TensorMapEncodeTiled fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_TensorMapEncodeTiled)ptr;
    }
    return fn;
}

// rows x cols int8 matrix (row stride = cols bytes), box 128 (cols) x box_rows.
static int make_map(CUtensorMap *map, const int8_t *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
    PFN_TensorMapEncodeTiled enc = get_encode();
    if (!enc) return CUOZBLAS_STATUS_CUDA_ERROR;
    cuuint64_t gdim[2] = {cols, rows};
    cuuint64_t gstride[1] = {cols};
    cuuint32_t box[2] = {(cuuint32_t)I8_BK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)base, gdim, gstride, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

// Column-major FP64 matrix, rows x cols with leading dimension ld: boxes of
// box_rows (inner, contiguous) x box_cols, no swizzle, zero fill outside.
// Needs base 16-byte aligned and ld even (a stride of whole 16-byte units).
int make_map_f64(CUtensorMap *map, const double *base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows,
                 uint32_t box_cols) {
    PFN_TensorMapEncodeTiled enc = get_encode();
    if (!enc || ((uintptr_t)base & 15) != 0 || (ld & 1) != 0 || rows == 0 || cols == 0 || ld < rows)
        return CUOZBLAS_STATUS_NOT_SUPPORTED;
    cuuint64_t gdim[2] = {rows, cols};
    cuuint64_t gstride[1] = {ld * sizeof(double)};
    cuuint32_t box[2] = {box_rows, box_cols};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)base, gdim, gstride, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_NOT_SUPPORTED;
}

struct DigitOperand {
    int8_t *digits = nullptr;  // S x lines_pad x k_pad
    int *e = nullptr;          // line exponents
    int S = 0, need = 0, lines_pad = 0;
};

// Lines of op(X): `strided` = element (line l, i) at X[i*ldx + l].
static int split_digits(cuozblasHandle_t *h, bool strided, int nl, int k, const double *X, int ldx, int cap,
                        int k_pad, int line_quantum, DigitOperand &op, Arena &ar) {
    State *st = state(h);
    op.lines_pad = (nl + line_quantum - 1) / line_quantum * line_quantum;
    op.e = ar.take<int>(nl > 0 ? nl : 1);
    unsigned long long *mxb = nullptr;
    int *lsbm = nullptr;
    unsigned *ticket = nullptr;
    if (strided) {  // lines contiguous: per-line statistics merged across blocks
        mxb = ar.take<unsigned long long>(nl > 0 ? nl : 1);
        lsbm = ar.take<int>(nl > 0 ? nl : 1);
        ticket = ar.take<unsigned>(1);
    }
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemsetAsync(st->d_ints, 0, sizeof(int), st->stream));
    if (nl > 0 && k > 0) {
        if (strided) {
            OZB_CHECK(cudaMemsetAsync(mxb, 0, sizeof(unsigned long long) * nl, st->stream));
            OZB_CHECK(cudaMemsetAsync(lsbm, 0x7f, sizeof(int) * nl, st->stream));  // above every exponent
            OZB_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st->stream));
            const int tiles = (nl + 127) / 128;
            int ky = (4 * sm_count() + tiles - 1) / tiles;
            const int kmax = (k + 255) / 256;  // at least 256 k per block (128 per thread)
            ky = ky < 1 ? 1 : (ky > kmax ? kmax : ky);
            counted(h);
            k_digit_count_rows<<<dim3(tiles, ky), 256, 0, st->stream>>>(k, nl, X, ldx, mxb, lsbm, ticket, op.e,
                                                                        st->d_ints);
        } else {
            counted(h);
            k_digit_count<<<nl, 256, 0, st->stream>>>(k, nl, X, ldx, op.e, st->d_ints);
        }
    } else if (nl > 0) {
        OZB_CHECK(cudaMemsetAsync(op.e, 0, sizeof(int) * nl, st->stream));  // k = 0: zero digits
    }
    OZB_CHECK(cudaGetLastError());
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, st->d_ints, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    op.need = st->h_ints[0];
    op.S = op.need < 1 ? 1 : op.need;
    if (cap > 0 && op.S > cap) op.S = cap;
    op.digits = ar.take<int8_t>((uint64_t)op.S * op.lines_pad * k_pad);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    if (op.lines_pad == 0) return CUOZBLAS_STATUS_SUCCESS;
    counted(h);
    if (strided) {
        k_digit_write_rows<<<dim3(op.lines_pad / 128, k_pad / 32), 256, 0, st->stream>>>(k, nl, op.lines_pad, k_pad,
                                                                                         op.S, X, ldx, op.e,
                                                                                         op.digits);
    } else {
        const int64_t chunks = (int64_t)op.lines_pad * (k_pad / 16);
        k_digit_write<<<(unsigned)((chunks + 255) / 256), 256, 0, st->stream>>>(k, nl, op.lines_pad, k_pad, op.S, X,
                                                                                 ldx, op.e, op.digits);
    }
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

// The schedule of one product: items {ia, ib, kb0, kb1} (a digit pair over a
// range of 128-k blocks) grouped per level into INT32 groups of at most
// I8_MAX_TERMS products per output, levels visited from the largest, and the
// runs of levels that combine exactly below 2^53 (group meta: shift |
// flush << 8 | first << 9 | last << 10 | (next flush exponent + 32768) << 16,
// group.z the flush exponent).  Pair
// set: full, or the triangle ia + ib <= min(nA, nB) - 1
// (src/cuda/cuozblas_gemm.cu:138).  Returns the number of pairs.
// Fixed-capacity form: writes at most max_items items and max_groups groups
// (counts to *ni, *ng); returns the number of pairs, or -1 when a capacity or
// the 128-level bound of the run table is exceeded (nothing usable written).
int i8_schedule_into(int nA, int nB, int nkb, bool triangular, int4 *items, int max_items, int *ni, int4 *groups,
                     int max_groups, int *ng) {
    const int maxlevel = triangular ? (nA < nB ? nA : nB) - 1 : nA + nB - 2;
    constexpr int kMaxLevels = 128;
    if (maxlevel + 1 > kMaxLevels || max_groups < 1) return -1;
    // products per output in one INT32 group: (kb1 - kb0) * 128 each
    const int64_t kb_cap = I8_MAX_TERMS / I8_BK;  // k-blocks per group
    unsigned __int128 lbound[kMaxLevels];  // max |V| of each level (products x 127^2)
    for (int L = 0; L <= maxlevel; L++) lbound[L] = 0;
    int n_it = 0, n_gr = 0, npairs = 0;
    auto close_group = [&](int gbeg, int L, int64_t used) {
        if (n_gr >= max_groups) return false;
        groups[n_gr++] = make_int4(gbeg, n_it, L, 0);
        lbound[L] += (unsigned __int128)(used * I8_BK * 127 * 127);
        return true;
    };
    for (int L = 0; L <= maxlevel; L++) {  // largest level sums first
        const int lo = L - (nB - 1) > 0 ? L - (nB - 1) : 0, hi = L < nA - 1 ? L : nA - 1;
        int64_t used = 0;
        int gbeg = n_it;
        for (int ia = lo; ia <= hi; ia++) {
            npairs++;
            for (int kb0 = 0; kb0 < nkb;) {
                int64_t room = kb_cap - used;
                if (room <= 0) {
                    if (!close_group(gbeg, L, used)) return -1;
                    gbeg = n_it;
                    used = 0;
                    room = kb_cap;
                }
                const int kb1 = (int)((nkb - kb0) < room ? nkb : kb0 + room);
                if (n_it >= max_items) return -1;
                items[n_it++] = make_int4(ia, L - ia, kb0, kb1);
                used += kb1 - kb0;
                kb0 = kb1;
            }
        }
        if (n_it > gbeg && !close_group(gbeg, L, used)) return -1;
    }
    // Runs of consecutive levels whose exact combination stays below 2^53,
    // formed from the most significant level up (levels 0..3, 4..7, ...):
    // extending a run [L_lo, L_hi] by L_hi + 1 multiplies its bound by 2^7 and
    // adds the new level's bound.  Groups are visited in ascending level order
    // (largest sums first, so a cancellation between runs happens while the
    // FP64 sum is still exact); level L of run [L_lo, L_hi] is shifted by
    // 7 (L_hi - L) bits and the run's last visited group (level L_hi) flushes
    // acc * 2^(-7 (L_hi + 2)).
    const unsigned __int128 lim = (unsigned __int128)1 << 53;
    int run_hi[kMaxLevels];
    for (int L0 = 0; L0 <= maxlevel;) {
        unsigned __int128 b = lbound[L0];
        int L1 = L0;
        while (L1 + 1 <= maxlevel && (b << 7) + lbound[L1 + 1] < lim) {
            b = (b << 7) + lbound[L1 + 1];
            L1++;
        }
        for (int L = L0; L <= L1; L++) run_hi[L] = L1;
        L0 = L1 + 1;
    }
    bool first = true;
    for (int g = 0; g < n_gr; g++) {
        const int L = groups[g].z;
        int meta = 7 * (run_hi[L] - L);
        const bool last_of_level = (g + 1 == n_gr) || groups[g + 1].z != L;
        if (last_of_level && L == run_hi[L]) {
            meta |= (1 << 8) | (first ? (1 << 9) : 0);
            first = false;
            groups[g].z = -7 * (run_hi[L] + 2);
            // the next run's flush exponent: the rounding error of this flush is carried there
            if (L < maxlevel) meta |= (-7 * (run_hi[L + 1] + 2) + 32768) << 16;
        } else {
            groups[g].z = 0;
        }
        groups[g].w = meta;
    }
    if (n_gr > 0) groups[n_gr - 1].w |= (1 << 10);
    *ni = n_it;
    *ng = n_gr;
    return npairs;
}

int i8_schedule(int nA, int nB, int nkb, bool triangular, std::vector<int4> &items, std::vector<int4> &groups) {
    // every pair spans at most ceil(nkb / kb_cap) + 1 items, and a group holds at least one item
    const int64_t per_pair = (int64_t)nkb / (I8_MAX_TERMS / I8_BK) + 2;
    const int64_t cap = (int64_t)(nA > 0 ? nA : 1) * (nB > 0 ? nB : 1) * per_pair;
    items.assign((size_t)cap, make_int4(0, 0, 0, 0));
    groups.assign((size_t)cap, make_int4(0, 0, 0, 0));
    int ni = 0, ng = 0;
    const int np = i8_schedule_into(nA, nB, nkb, triangular, items.data(), (int)cap, &ni, groups.data(), (int)cap, &ng);
    items.resize(np < 0 ? 0 : (size_t)ni);
    groups.resize(np < 0 ? 0 : (size_t)ng);
    return np;
}

int i8_blk_launch(cuozblasHandle_t *h, const CUtensorMap &tmA, const CUtensorMap &tmB, int m, int n, int m_pad,
                  int n_pad, int k_pad, int nA, int nB, bool triangular, const int *ea, const int *eb, double alpha,
                  double beta, double *C, int ldc, int strip, int width, int *d_err, Arena &ar);  // gemm_i8_blk.cu

// Default digit cap when nSplitMax is 0 (enough for an exact split of
// values whose lines span ~2^80; larger spans are truncated).
constexpr int kI8DefaultCap = 19;

int gemm_i8_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc) {
    State *st = state(h);
    Arena ar(h);
    const int k_pad = k > 0 ? (k + I8_BK - 1) / I8_BK * I8_BK : I8_BK;  // k = 0: zero digits, C = beta * C
    const int cap = h->nSplitMax > 0 ? h->nSplitMax : kI8DefaultCap;
    DigitOperand da, db;
    ev_record(h, 0);
    OZB_TRY(split_digits(h, !is_trans(ta), m, k, A, lda, cap, k_pad, I8_BM, da, ar));
    ev_record(h, 1);
    OZB_TRY(split_digits(h, is_trans(tb), n, k, B, ldb, cap, k_pad, I8_BN, db, ar));
    const int nA = da.S, nB = db.S;
    const int nkb = k_pad / I8_BK;
    std::vector<int4> items, groups;
    const int npairs = i8_schedule(nA, nB, nkb, h->fastMode != 0, items, groups);
    if (npairs < 0) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    h->nSplitA = (float)nA;
    h->nSplitB = (float)nB;
    h->nSplitC = (float)npairs;
    h->mbk = m;
    h->nbk = n;
    int4 *d_sched = ar.take<int4>(items.size() + groups.size());
    int *d_err = ar.take<int>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    std::vector<int4> sched(items);
    sched.insert(sched.end(), groups.begin(), groups.end());
    OZB_CHECK(cudaMemcpyAsync(d_sched, sched.data(), sizeof(int4) * sched.size(), cudaMemcpyHostToDevice,
                              st->stream));
    OZB_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), st->stream));

    CUtensorMap tmA, tmB;
    OZB_TRY(make_map(&tmA, da.digits, (uint64_t)nA * da.lines_pad, k_pad, I8_BM));
    OZB_TRY(make_map(&tmB, db.digits, (uint64_t)nB * db.lines_pad, k_pad, I8_BN));
    I8Params p;
    p.m = m;
    p.n = n;
    p.m_pad = da.lines_pad;
    p.n_pad = db.lines_pad;
    p.ldc = ldc;
    p.tiles_m = da.lines_pad / I8_BM;
    p.tiles_n = db.lines_pad / I8_BN;
    p.strip = p.tiles_m < 12 ? p.tiles_m : 12;
    p.n_items = (int)items.size();
    p.n_groups = (int)groups.size();
    p.items = d_sched;
    p.groups = d_sched + items.size();
    p.ea = da.e;
    p.eb = db.e;
    p.alpha = alpha;
    p.beta = beta;
    p.C = C;
    p.err = d_err;
    int dev = 0, nsm = 0;
    OZB_CHECK(cudaGetDevice(&dev));
    OZB_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ntiles = p.tiles_m * p.tiles_n;
    const int grid = ntiles < nsm ? ntiles : nsm;
    OZB_CHECK(cudaFuncSetAttribute(k_i8_gemm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, I8_SMEM));
    // Launch shape, measured once per shape (every choice gives the same bits;
    // candidates write a scratch product with beta = 0): the product kernel
    // (level-blocked or level-wise), the block width of the level-blocked
    // schedule (levels accumulated together: 4 or 3 within the runs, or equal
    // cuts of at most 4 levels across them) and the rasterisation
    // strip height.  OZBLAS_I8_LEVELWISE keeps the level-wise kernel (strip
    // tuned), OZBLAS_I8_BLOCK=w the level-blocked kernel at width w (negative:
    // the cuts across runs).
    struct Shape {
        int width;  // 0: level-wise kernel; < 0: blocks of at most -width levels cut across runs
        int strip;
    };
    std::vector<Shape> cand;
    auto add = [&](int w, int sv) {
        const int v = sv < p.tiles_m ? sv : p.tiles_m;
        for (const Shape &c : cand)
            if (c.width == w && c.strip == v) return;
        cand.push_back(Shape{w, v});
    };
    if (st->env.i8_levelwise) {
        for (int sv : {12, 4, 8, 16, 24}) add(0, sv);
    } else if (st->env.i8_block != 0) {
        for (int sv : {12, 4, 8, 16, 24}) add(st->env.i8_block, sv);
    } else {
        for (int sv : {12, 4, 8, 16, 24}) add(4, sv);
        // the cut across runs where it applies (a crossing block is one K chunk);
        // narrower blocks measured slower on every bench shape and only add
        // chances for timing noise to pick them (OZBLAS_I8_BLOCK still forces them)
        std::vector<BlkStep> cut;
        if (blk_schedule(nA, nB, k_pad / I8_BK, h->fastMode != 0, 4, cut, true)) add(-4, 12);
        add(3, 12);
        add(0, 12);
    }
    auto launch = [&](const Shape &c, I8Params &pp) {
        if (c.width != 0) {
            const uint64_t mk2 = ar.mark();
            const int r = i8_blk_launch(h, tmA, tmB, m, n, pp.m_pad, pp.n_pad, k_pad, nA, nB, h->fastMode != 0, da.e,
                                        db.e, pp.alpha, pp.beta, pp.C, pp.ldc, c.strip, c.width, d_err, ar);
            ar.release(mk2);
            if (r != CUOZBLAS_STATUS_NOT_SUPPORTED) return r;
        }
        // the level-wise kernel: chosen, or where the blocked schedule does not apply
        pp.strip = c.strip;
        counted(h);
        k_i8_gemm<0><<<grid, I8_THREADS, I8_SMEM, st->stream>>>(tmA, tmB, pp);
        return cudaGetLastError() == cudaSuccess ? (int)CUOZBLAS_STATUS_SUCCESS : (int)CUOZBLAS_STATUS_CUDA_ERROR;
    };
    int pick = 0;
    if (cand.size() > 1) {
        const uint64_t mk = ar.mark();
        double *scratch = ar.take<double>((uint64_t)m * n);
        if (ar.ok) {
            char key[160];
            snprintf(key, sizeof(key), "i8s%d:%d:%d:%d:%d:%d:%d:%d",
                     st->env.i8_levelwise ? -1 : st->env.i8_block, p.tiles_m, p.tiles_n, nkb, nA, nB,
                     h->fastMode != 0 ? 1 : 0, grid);
            I8Params pt = p;
            pt.C = scratch;
            pt.ldc = m;
            pt.alpha = 1.0;
            pt.beta = 0.0;
            pick = tune_pick(key, (int)cand.size(), 0, st->stream, [&](int i) { return launch(cand[(size_t)i], pt); });
        }
        ar.ok = true;
        ar.release(mk);
    }
    ev_record(h, 2);
    {
        const int r = launch(cand[(size_t)pick], p);
        if (r != CUOZBLAS_STATUS_SUCCESS) return r;
    }
    ev_record(h, 3);
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, d_err, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    if (st->h_ints[0] != 0) {
        fprintf(stderr, "cuozblas: INT8 GEMM kernel wait timed out (code %d)\n", st->h_ints[0]);
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    h->t_SplitA = ev_ms(h, 0, 1) * 1e-3f;
    h->t_SplitB = ev_ms(h, 1, 2) * 1e-3f;
    h->t_comp = ev_ms(h, 2, 3) * 1e-3f;
    h->t_sum = 0.f;  // fused into the product kernel
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// The mixed form <double,float,float> on the INT8 tensor cores.  Its FP32
// slice f = scalbn(s, -tau) is q 2^(rho - 53) with q an integer of magnitude at
// most 2^(53 - rho) (src/cpu/ozblas_split.cpp:181-221), so for rho >= 47
// (k > 1024 under splitEpsMode 0) every slice is an int8 q, and the FP32 slice
// product sum(f_a f_b) = 2^(2 rho - 106) V with V the exact INT32 sum of the
// q_a q_b (|V| <= 2^24 by the rho rule).  The ordered sum adds
// scalbn(V, tauA + tauB + 2 rho - 106), the same value the reference adds.
// ---------------------------------------------------------------------------
// One CTA per line, the plain split arithmetic; writes q (int8) of every
// level s at digits[(s * lines_pad + line) * k_pad + i] (the buffer is zeroed
// before) and tau at exps[s * nl + line].  rem: k doubles per line (global).
__global__ void __launch_bounds__(256) k_ds_digits(int k, int nl, const double *__restrict__ X, int ldx, int rho,
                                                   int ns, int lines_pad, int k_pad, int8_t *__restrict__ digits,
                                                   short *__restrict__ exps, double *__restrict__ rem) {
    __shared__ double red[8];
    const int line = blockIdx.x;
    if (line >= nl) return;
    const double *x = X + (size_t)line * ldx;
    double *r = rem + (size_t)line * k;
    double mx = 0.0;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double v = x[i];
        r[i] = v;
        mx = ref_max(mx, fabs(v));
    }
    mx = block_max_nonneg(mx, red);
    for (int s = 0; s < ns; s++) {
        const int tau = tau_rule(mx);
        const double sigma = 0.75 * pow2(rho + tau);
        if (threadIdx.x == 0) exps[(size_t)s * nl + line] = (short)tau;
        int8_t *o = digits + ((size_t)s * lines_pad + line) * k_pad;
        double nm = 0.0;
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            double v = r[i];
            const double sl = (v + sigma) - sigma;
            v = v - sl;
            r[i] = v;
            nm = ref_max(nm, fabs(v));
            // slices are q 2^(rho + tau - 53); scalbn is exact here and, unlike a
            // multiplication by 2^(53 - rho - tau), cannot overflow for tiny tau
            o[i] = (int8_t)(int)scalbn(sl, 53 - rho - tau);
        }
        mx = block_max_nonneg(nm, red);
    }
}

// C = alpha op(A) op(B) + beta C in the <double,float,float> form with INT8
// slices; the caller checks rho >= 47.  Returns the split counts in *nA, *nB.
int gemm_ds_i8_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta, double *C, int ldc, int rho, int fastMode,
                    int *nA_out, int *nB_out, int *np_out) {
    State *st = state(h);
    Arena ar(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int k_pad = (k + I8_BK - 1) / I8_BK * I8_BK;
    int ns[2];
    int8_t *dig[2];
    short *ex[2];
    int lpad[2];
    ev_record(h, 0);
    for (int o = 0; o < 2; o++) {
        const bool strided = o == 0 ? !is_trans(ta) : is_trans(tb);
        const int nl = o == 0 ? m : n;
        const double *X = o == 0 ? A : B;
        const int ldx = o == 0 ? lda : ldb;
        const double *src = X;
        int lds = ldx;
        const uint64_t mk = ar.mark();
        if (strided) {
            double *tmp = ar.take<double>((uint64_t)nl * k);
            if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
            OZB_TRY(transpose(h, nl, k, X, ldx, tmp, k));
            src = tmp;
            lds = k;
        }
        OZB_TRY(split_lines_count(h, k, nl, src, lds, rho, maxS, &ns[o]));
        lpad[o] = (nl + I8_BM - 1) / I8_BM * I8_BM;
        // slices and exponents stay below the temporaries
        ar.release(mk);
        dig[o] = ar.take<int8_t>((uint64_t)ns[o] * lpad[o] * k_pad);
        ex[o] = ar.take<short>((uint64_t)ns[o] * nl);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        const uint64_t mk2 = ar.mark();
        if (strided) {  // the transposed copy again, above the slices
            double *tmp = ar.take<double>((uint64_t)nl * k);
            if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
            OZB_TRY(transpose(h, nl, k, X, ldx, tmp, k));
            src = tmp;
        }
        double *rem = ar.take<double>((uint64_t)nl * k);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_CHECK(cudaMemsetAsync(dig[o], 0, (size_t)ns[o] * lpad[o] * k_pad, st->stream));
        counted(h);
        k_ds_digits<<<nl, 256, 0, st->stream>>>(k, nl, src, lds, rho, ns[o], lpad[o], k_pad, dig[o], ex[o], rem);
        OZB_CHECK(cudaGetLastError());
        ar.release(mk2);
        ev_record(h, o + 1);
    }
    const int nA = ns[0], nB = ns[1];
    int maxlevel = (nA - 1) + (nB - 1);
    {
        const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
        maxlevel = (maxlevel - fastMode) > mn ? (maxlevel - fastMode) : mn;  // src/cpu/ozblas_gemm.cpp:163-164
    }
    const int nkb = k_pad / I8_BK;
    std::vector<int4> sched;
    for (int ik = 0; ik <= maxlevel; ik++)  // FSum order: ik ascending, ia ascending
        for (int ia = 0; ia < nA; ia++) {
            const int ib = ik - ia;
            if (ib >= 0 && ib < nB) sched.push_back(make_int4(ia, ib, 0, nkb));
        }
    const int np = (int)sched.size();
    for (int g = 0; g < np; g++) sched.push_back(make_int4(g, g + 1, 0, 0));
    int4 *d_sched = ar.take<int4>(sched.size());
    int *d_err = ar.take<int>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemcpyAsync(d_sched, sched.data(), sizeof(int4) * sched.size(), cudaMemcpyHostToDevice,
                              st->stream));
    OZB_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), st->stream));
    CUtensorMap tmA, tmB;
    OZB_TRY(make_map(&tmA, dig[0], (uint64_t)nA * lpad[0], k_pad, I8_BM));
    OZB_TRY(make_map(&tmB, dig[1], (uint64_t)nB * lpad[1], k_pad, I8_BN));
    I8Params p;
    memset(&p, 0, sizeof(p));
    p.m = m;
    p.n = n;
    p.m_pad = lpad[0];
    p.n_pad = lpad[1];
    p.ldc = ldc;
    p.tiles_m = lpad[0] / I8_BM;
    p.tiles_n = lpad[1] / I8_BN;
    p.strip = p.tiles_m < 12 ? p.tiles_m : 12;
    p.n_items = np;
    p.n_groups = np;
    p.items = d_sched;
    p.groups = d_sched + np;
    p.eas = ex[0];
    p.ebs = ex[1];
    p.sbias = 2 * (rho - 53);
    p.alpha = alpha;
    p.beta = beta;
    p.C = C;
    p.err = d_err;
    const int nsm = sm_count();
    const int ntiles = p.tiles_m * p.tiles_n;
    OZB_CHECK(cudaFuncSetAttribute(k_i8_gemm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, I8_SMEM));
    counted(h);
    k_i8_gemm<1><<<ntiles < nsm ? ntiles : nsm, I8_THREADS, I8_SMEM, st->stream>>>(tmA, tmB, p);
    OZB_CHECK(cudaGetLastError());
    ev_record(h, 3);
    ev_record(h, 4);
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, d_err, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    if (st->h_ints[0] != 0) {
        fprintf(stderr, "cuozblas: INT8 mixed-form kernel wait timed out (code %d)\n", st->h_ints[0]);
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    *nA_out = nA;
    *nB_out = nB;
    *np_out = np;
    return CUOZBLAS_STATUS_SUCCESS;
}

// Exact FP64 pair products on the INT8 tensor cores for slices cut into
// `D` int8 digit planes (digits[(s D + d) * lines_pad + line][k_pad], most
// significant first): for every pair of `pairs` (FSum order),
// pbuf[pair][col][row] = 2^(sbias + tauA + tauB) sum_k qa qb with
// q = sum_d digit_d 2^(7(D-1-d)) (tauA = eas[ia][row], tauB = ebs[ib][col], or 0
// without them), rounded once if it is subnormal.
// The caller guarantees D k 127^2 < 2^31 (INT32 groups) and that each pair's
// |sum| stays below 2^53.
int i8_exact_pairs(cuozblasHandle_t *h, int m, int n, int k_pad, const int8_t *digA, int lpadA, int planesA,
                   const int8_t *digB, int lpadB, int planesB, int D, const std::vector<int2> &pairs, int sbias,
                   const short *eas, const short *ebs, double *pbuf) {
    State *st = state(h);
    Arena ar(h);
    const uint64_t mk = ar.mark();
    const int nkb = k_pad / I8_BK;
    std::vector<int4> items, groups;
    for (size_t pi = 0; pi < pairs.size(); pi++)
        for (int L = 0; L <= 2 * D - 2; L++) {
            const int beg = (int)items.size();
            for (int d = 0; d < D; d++) {
                const int e = L - d;
                if (e >= 0 && e < D) items.push_back(make_int4(pairs[pi].x * D + d, pairs[pi].y * D + e, 0, nkb));
            }
            groups.push_back(make_int4(beg, (int)items.size(), (int)pi, ((7 * (2 * D - 2 - L)) << 8) | (L == 2 * D - 2)));
        }
    std::vector<int4> sched(items);
    sched.insert(sched.end(), groups.begin(), groups.end());
    int4 *d_sched = ar.take<int4>(sched.size());
    int *d_err = ar.take<int>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemcpyAsync(d_sched, sched.data(), sizeof(int4) * sched.size(), cudaMemcpyHostToDevice,
                              st->stream));
    OZB_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), st->stream));
    CUtensorMap tmA, tmB;
    OZB_TRY(make_map(&tmA, digA, (uint64_t)planesA * lpadA, k_pad, I8_BM));
    OZB_TRY(make_map(&tmB, digB, (uint64_t)planesB * lpadB, k_pad, I8_BN));
    I8Params p;
    memset(&p, 0, sizeof(p));
    p.m = m;
    p.n = n;
    p.m_pad = lpadA;
    p.n_pad = lpadB;
    p.ldc = D;  // MODE 2: digit planes per slice level
    p.tiles_m = lpadA / I8_BM;
    p.tiles_n = lpadB / I8_BN;
    p.strip = p.tiles_m < 12 ? p.tiles_m : 12;
    p.n_items = (int)items.size();
    p.n_groups = (int)groups.size();
    p.items = d_sched;
    p.groups = d_sched + items.size();
    p.sbias = sbias;
    p.C = pbuf;  // MODE 2: the pair buffer
    p.eas = eas;
    p.ebs = ebs;
    p.err = d_err;
    const int nsm = sm_count();
    const int ntiles = p.tiles_m * p.tiles_n;
    OZB_CHECK(cudaFuncSetAttribute(k_i8_gemm<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, I8_SMEM));
    counted(h);
    k_i8_gemm<2><<<ntiles < nsm ? ntiles : nsm, I8_THREADS, I8_SMEM, st->stream>>>(tmA, tmB, p);
    OZB_CHECK(cudaGetLastError());
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, d_err, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    ar.release(mk);
    if (st->h_ints[0] != 0) {
        fprintf(stderr, "cuozblas: INT8 pair-product kernel wait timed out (code %d)\n", st->h_ints[0]);
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the INT8 product path (cuozblasDgemmI8Static).
//
// Some callers cannot allocate device memory at all: real-time or embedded
// hosts whose device memory is budgeted once at start-up, and hosts whose own
// allocator (a framework's caching allocator, say) already owns the whole
// device, so a cudaMalloc inside the library would fail or fight it.
// For them the digit split and the tcgen05 product kernel run on scratch in
// the file-scope array below instead of a handle's arena, so a call makes no
// cudaMalloc, no cudaFree and no other allocation.  The array is 64 MiB and
// every GPU that loads this library holds it until the process exits.  The
// host code reaches it through the device address that cudaGetSymbolAddress
// returns, looked up once per device (with that device current) on the first
// call there; that first call should therefore come before any stream capture.
// All calls share the one array and it keeps the last call's contents, so
// calls whose work overlaps on the GPU (other streams, other host threads)
// race; the counters and the error word are cleared at the start of each call.
// ---------------------------------------------------------------------------
__global__ void k_transpose(int rows, int cols, const double *__restrict__ A, int lda, double *__restrict__ out,
                            int ldo);  // split.cu

constexpr size_t kI8StaticBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_i8_static_scratch[kI8StaticBytes];

constexpr int kI8StaticMaxDevices = 64;
static unsigned char *g_i8_static_addr[kI8StaticMaxDevices];
static std::mutex g_i8_static_mu;

static int i8_static_area(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CUOZBLAS_STATUS_CUDA_ERROR;
    if (dev < 0 || dev >= kI8StaticMaxDevices) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    std::lock_guard<std::mutex> lock(g_i8_static_mu);
    if (g_i8_static_addr[dev] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_i8_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            fprintf(stderr, "cuozblasDgemmI8Static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return CUOZBLAS_STATUS_CUDA_ERROR;
        }
        g_i8_static_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_i8_static_addr[dev];
    return CUOZBLAS_STATUS_SUCCESS;
}

struct StaticBump {
    unsigned char *base;
    size_t off = 0;
    bool ok = true;
    template <typename T>
    T *take(size_t count) {
        const size_t start = (off + 255) / 256 * 256, bytes = count * sizeof(T);
        if (start + bytes > kI8StaticBytes) {
            ok = false;
            return nullptr;
        }
        off = start + bytes;
        return reinterpret_cast<T *>(base + start);
    }
};

constexpr int kI8StaticMaxItems = 2048, kI8StaticMaxGroups = 256;

static int dgemm_i8_static(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                           const double *B, int ldb, double beta, double *C, int ldc, int nsplit_max, int fast,
                           cudaStream_t stream) {
    unsigned char *area = nullptr;
    OZB_TRY(i8_static_area(&area));
    StaticBump bump{area};
    int *d_err = bump.take<int>(1);
    int *d_cnt = bump.take<int>(2);
    int4 *d_sched = bump.take<int4>(kI8StaticMaxItems + kI8StaticMaxGroups);
    const int k_pad = k > 0 ? (k + I8_BK - 1) / I8_BK * I8_BK : I8_BK;  // k = 0: zero digits, C = beta * C
    const int m_pad = (m + I8_BM - 1) / I8_BM * I8_BM, n_pad = (n + I8_BN - 1) / I8_BN * I8_BN;
    int *ea = bump.take<int>(m), *eb = bump.take<int>(n);
    const bool tA = !is_trans(ta), tB = is_trans(tb);  // lines must be made K-contiguous
    double *la = tA ? bump.take<double>((size_t)m * k) : nullptr;
    double *lb = tB ? bump.take<double>((size_t)n * k) : nullptr;
    if (!bump.ok) {
        fprintf(stderr, "cuozblasDgemmI8Static: m=%d n=%d k=%d needs more than the %zu MiB static scratch\n", m, n, k,
                kI8StaticBytes >> 20);
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    OZB_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    OZB_CHECK(cudaMemsetAsync(d_cnt, 0, 2 * sizeof(int), stream));
    const double *srcA = A, *srcB = B;
    int ldsA = lda, ldsB = ldb;
    if (tA && k > 0) {
        k_transpose<<<dim3((m + 31) / 32, (k + 31) / 32), dim3(32, 8), 0, stream>>>(m, k, A, lda, la, k);
        srcA = la;
        ldsA = k;
    }
    if (tB && k > 0) {
        k_transpose<<<dim3((n + 31) / 32, (k + 31) / 32), dim3(32, 8), 0, stream>>>(n, k, B, ldb, lb, k);
        srcB = lb;
        ldsB = k;
    }
    k_digit_count<<<m, 256, 0, stream>>>(k, m, srcA, ldsA, ea, d_cnt);
    k_digit_count<<<n, 256, 0, stream>>>(k, n, srcB, ldsB, eb, d_cnt + 1);
    OZB_CHECK(cudaGetLastError());
    int cnt[2] = {0, 0};
    OZB_CHECK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
    OZB_CHECK(cudaStreamSynchronize(stream));
    const int cap = nsplit_max > 0 ? nsplit_max : kI8DefaultCap;
    int nA = cnt[0] < 1 ? 1 : cnt[0], nB = cnt[1] < 1 ? 1 : cnt[1];
    if (nA > cap) nA = cap;
    if (nB > cap) nB = cap;
    int8_t *da = bump.take<int8_t>((size_t)nA * m_pad * k_pad);
    int8_t *db = bump.take<int8_t>((size_t)nB * n_pad * k_pad);
    if (!bump.ok) {
        fprintf(stderr,
                "cuozblasDgemmI8Static: m=%d n=%d k=%d with %d x %d digits needs more than the %zu MiB static "
                "scratch\n",
                m, n, k, nA, nB, kI8StaticBytes >> 20);
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    k_digit_write<<<(unsigned)(((int64_t)m_pad * (k_pad / 16) + 255) / 256), 256, 0, stream>>>(k, m, m_pad, k_pad, nA,
                                                                                              srcA, ldsA, ea, da);
    k_digit_write<<<(unsigned)(((int64_t)n_pad * (k_pad / 16) + 255) / 256), 256, 0, stream>>>(k, n, n_pad, k_pad, nB,
                                                                                              srcB, ldsB, eb, db);
    OZB_CHECK(cudaGetLastError());

    // the same schedule as cuozblasDgemmI8, built in fixed host arrays
    const int nkb = k_pad / I8_BK;
    int4 items[kI8StaticMaxItems], groups[kI8StaticMaxGroups];
    int ni = 0, ng = 0;
    if (i8_schedule_into(nA, nB, nkb, fast != 0, items, kI8StaticMaxItems, &ni, groups, kI8StaticMaxGroups, &ng) < 0) {
        fprintf(stderr, "cuozblasDgemmI8Static: %d x %d digits over k=%d exceed the static schedule (%d items, %d "
                "groups)\n", nA, nB, k, kI8StaticMaxItems, kI8StaticMaxGroups);
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    OZB_CHECK(cudaMemcpyAsync(d_sched, items, sizeof(int4) * ni, cudaMemcpyHostToDevice, stream));
    OZB_CHECK(cudaMemcpyAsync(d_sched + ni, groups, sizeof(int4) * ng, cudaMemcpyHostToDevice, stream));
    CUtensorMap tmA, tmB;
    OZB_TRY(make_map(&tmA, da, (uint64_t)nA * m_pad, k_pad, I8_BM));
    OZB_TRY(make_map(&tmB, db, (uint64_t)nB * n_pad, k_pad, I8_BN));
    I8Params p;
    p.m = m;
    p.n = n;
    p.m_pad = m_pad;
    p.n_pad = n_pad;
    p.ldc = ldc;
    p.tiles_m = m_pad / I8_BM;
    p.tiles_n = n_pad / I8_BN;
    p.strip = p.tiles_m < 12 ? p.tiles_m : 12;
    p.n_items = ni;
    p.n_groups = ng;
    p.items = d_sched;
    p.groups = d_sched + ni;
    p.ea = ea;
    p.eb = eb;
    p.alpha = alpha;
    p.beta = beta;
    p.C = C;
    p.err = d_err;
    int dev = 0, nsm = 0;
    OZB_CHECK(cudaGetDevice(&dev));
    OZB_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ntiles = p.tiles_m * p.tiles_n;
    OZB_CHECK(cudaFuncSetAttribute(k_i8_gemm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, I8_SMEM));
    k_i8_gemm<0><<<ntiles < nsm ? ntiles : nsm, I8_THREADS, I8_SMEM, stream>>>(tmA, tmB, p);
    OZB_CHECK(cudaGetLastError());
    int err = 0;
    OZB_CHECK(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OZB_CHECK(cudaStreamSynchronize(stream));
    if (err != 0) {
        fprintf(stderr, "cuozblasDgemmI8Static: product kernel wait timed out (code %d)\n", err);
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

// Leading dimensions of the stored A (m x k for 'n', k x m otherwise) and B
// (k x n for 'n', n x k otherwise), as a column-major BLAS checks them.
static bool i8_lds_valid(char ta, char tb, int m, int n, int k, int lda, int ldb) {
    const int ra = is_trans(ta) ? k : m, rb = is_trans(tb) ? n : k;
    return lda >= (ra > 1 ? ra : 1) && ldb >= (rb > 1 ? rb : 1);
}

}  // namespace ozb


// Testing hook (no reference counterpart), on the current device: the limit
// of every bounded wait in the INT8 product kernel in nanoseconds (0 restores
// the default of 2 s), and with hold_copies != 0 a producer that issues no
// copies, so that a wait runs out: the call then returns
// CUOZBLAS_STATUS_DEVICE_TIMEOUT after the kernel has released its tensor
// memory, and the context stays usable.
extern "C" int cuozblasSetI8WaitTest(uint64_t ns, int32_t hold_copies) {
    using namespace ozb;
    const uint64_t v = ns == 0 ? I8_WAIT_NS : ns;
    const int hold = hold_copies != 0 ? 1 : 0;
    OZB_CHECK(cudaMemcpyToSymbol(g_i8_wait_ns, &v, sizeof(v)));
    OZB_CHECK(cudaMemcpyToSymbol(g_i8_hold_copies, &hold, sizeof(hold)));
    h_i8_wait_ns.store(v);
    h_i8_hold_copies.store(hold);
    return CUOZBLAS_STATUS_SUCCESS;
}

extern "C" int cuozblasDgemmI8(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k,
                               double alpha, const double *A, int32_t lda, const double *B, int32_t ldb, double beta,
                               double *C, int32_t ldc) {
    using namespace ozb;
    OZB_TRY(counter_init(h));
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (!i8_lds_valid(transa, transb, m, n, k, lda, ldb)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->nSplitMax < 0 || h->nSplitMax > 64) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    return gemm_i8_core(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// Allocation-free INT8 product (see dgemm_i8_static above): same arguments and
// results as cuozblasDgemmI8 with the flags passed directly, no handle.
extern "C" int cuozblasDgemmI8Static(char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                                     const double *A, int32_t lda, const double *B, int32_t ldb, double beta,
                                     double *C, int32_t ldc, int32_t nSplitMax, int32_t fastMode, void *stream) {
    using namespace ozb;
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1) || nSplitMax < 0 || nSplitMax > 64)
        return CUOZBLAS_STATUS_INVALID_VALUE;
    if (!i8_lds_valid(transa, transb, m, n, k, lda, ldb)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    return dgemm_i8_static(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nSplitMax, fastMode,
                           reinterpret_cast<cudaStream_t>(stream));
}
