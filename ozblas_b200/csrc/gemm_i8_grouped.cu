// gemm_i8_grouped.cu — many INT8-form Ozaki DGEMMs of different shapes in one
// persistent grouped launch (cuozblasDgemmI8Batched).
//
// The arithmetic is that of gemm_i8.cu (line exponents, truncated 7-bit
// digits, levels, INT32 groups of at most 133143 products, exact runs of
// levels, the FP64 sum in tensor memory), so each problem's result is
// bit-identical to a cuozblasDgemmI8 call on it.  What changes, so that
// problems of any shape share one kernel:
//  * operands are split straight into tiles: every 128-line x 128-k block of
//    a digit level is 16 KiB and is stored with the tensor core's 128-byte
//    swizzle already applied (row r at r * 128, its 16-byte chunk c at chunk
//    position c ^ (r & 7)), so the producer fetches it with one contiguous
//    bulk copy and no per-problem tensor map exists;
//  * the split reads either layout of an operand in coalesced order (lines
//    contiguous, or k contiguous), so no transposed copy is made;
//  * the host lists every problem's output tiles, estimates each tile's cost
//    from its schedule (k-blocks of all pairs plus the sums) and deals the
//    tiles longest first onto the least loaded CTA; the producer, MMA and
//    epilogue warps of a CTA walk that same list.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <queue>
#include <vector>

#include "autotune.h"
#include "gemm_i8_blk.h"
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "tc05.cuh"

namespace ozb {

constexpr int G_T = 128;                    // lines and k per tile
constexpr int G_TILE_BYTES = G_T * G_T;     // one digit tile
constexpr int G_NST = 6, G_THREADS = 320, G_TMEM_COLS = 512, G_RCOL = 256;
constexpr int G_STAGE = 2 * G_TILE_BYTES;
constexpr int G_SMEM = G_NST * G_STAGE + 1024 + 256;
constexpr int64_t G_MAX_TERMS = 2147483647LL / (127 * 127);
constexpr uint64_t G_WAIT_NS = 2000000000ull;
enum { GERR_PRODUCER = 1, GERR_MMA = 2, GERR_EPI = 3 };

// One operand of one problem.  Element (line l, k index kk) of op(X) is
// X[l + kk * ld] when lines are contiguous (kcontig = 0) or X[l * ld + kk].
struct GOp {
    const double *X;
    int ld, lines, k, kcontig;
    int tiles_l, nkb, S;
    int *e;                  // line exponents
    unsigned long long *mx;  // per-line max |x| (bit pattern)
    int *lsb;                // per-line lowest set bit of a nonzero element
    int8_t *digits;          // S x tiles_l x nkb tiles
};

// Bytes of one operand's digit tiles, rounded up to 256 (the carving step).
__host__ __device__ inline unsigned long long g_digit_bytes(int S, int tiles_l, int nkb) {
    return ((unsigned long long)S * tiles_l * nkb * G_TILE_BYTES + 255ull) & ~255ull;
}

struct GProb {
    int m, n, ldc, nkb, tiles_m, tiles_n;
    int group0, n_groups;
    const int8_t *da, *db;
    const int *ea, *eb;
    double alpha, beta;
    double *C;
};

struct GParams {
    const GProb *probs;
    const int4 *items;      // {ia, ib, kb0, kb1}
    const int4 *groups;     // {item_begin, item_end, flush exponent, meta}, absolute item indices
    const int4 *tiles;      // {problem, tm, tn, 0}
    const int *cta_begin;   // CTA c runs tiles [cta_begin[c], cta_begin[c + 1])
    int *err;
};

__device__ __forceinline__ int g_exp_above(double v) {  // E with v < 2^E, v > 0
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    const int be = (int)(b >> 52);
    if (be == 0) {
        const uint64_t f = b & ((1ULL << 52) - 1);
        if (f == 0) return 0;
        return (63 - clz64(f)) - 1073;
    }
    return be - 1022;
}

__device__ __forceinline__ int g_lsb(double v) {  // exponent of the lowest set bit, v != 0
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    const int be = (int)(b >> 52);
    uint64_t f = b & ((1ULL << 52) - 1);
    if (be == 0) return -1074 + __ffsll((long long)f) - 1;
    f |= (1ULL << 52);
    return (be - 1075) + __ffsll((long long)f) - 1;
}

__device__ __forceinline__ void g_stat(double v, double &mx, int &lsb) {
    mx = ref_max(mx, fabs(v));
    if (v != 0.0) lsb = min(lsb, g_lsb(v));
}

// Per-line max and lowest set bit of one 128 x 128 block (op, line tile, k block).
__global__ void __launch_bounds__(256) k_g_stats(const int4 *__restrict__ blocks, const GOp *__restrict__ ops) {
    const int4 bk = blocks[blockIdx.x];
    const GOp o = ops[bk.x];
    const int l0 = bk.y * G_T, k0 = bk.z * G_T;
    const int t = threadIdx.x;
    if (!o.kcontig) {
        __shared__ double smx[256];
        __shared__ int slsb[256];
        const int l = l0 + (t & 127), kh = k0 + (t >> 7) * 64;
        double mx = 0.0;
        int lsb = 0x7fffffff;
        if (l < o.lines) {
#pragma unroll 8
            for (int j = 0; j < 64; j++) {
                const int kk = kh + j;
                if (kk < o.k) g_stat(o.X[(size_t)l + (size_t)kk * o.ld], mx, lsb);
            }
        }
        smx[t] = mx;
        slsb[t] = lsb;
        __syncthreads();
        if (t < 128 && l < o.lines) {
            mx = ref_max(smx[t], smx[t + 128]);
            lsb = min(slsb[t], slsb[t + 128]);
            if (mx > 0.0) atomicMax(&o.mx[l], (unsigned long long)__double_as_longlong(mx));
            if (lsb != 0x7fffffff) atomicMin(&o.lsb[l], lsb);
        }
    } else {
        const int w = t >> 5, lane = t & 31;
        for (int i = 0; i < G_T / 8; i++) {
            const int l = l0 + w + 8 * i;
            if (l >= o.lines) break;  // uniform per warp
            double mx = 0.0;
            int lsb = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int kk = k0 + 4 * lane + q;
                if (kk < o.k) g_stat(o.X[(size_t)l * o.ld + kk], mx, lsb);
            }
            for (int s = 16; s > 0; s >>= 1) {
                mx = ref_max(mx, __shfl_xor_sync(0xffffffffu, mx, s));
                lsb = min(lsb, __shfl_xor_sync(0xffffffffu, lsb, s));
            }
            if (lane == 0) {
                if (mx > 0.0) atomicMax(&o.mx[l], (unsigned long long)__double_as_longlong(mx));
                if (lsb != 0x7fffffff) atomicMin(&o.lsb[l], lsb);
            }
        }
    }
}

// Line exponent and the digit count that makes the line exact
// (need = max over its nonzero entries of ceil((E - lsb) / 7)).
__global__ void __launch_bounds__(256) k_g_lines(const GOp *__restrict__ ops, const int *__restrict__ line0,
                                                 int nops, int total, int *__restrict__ need) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = nops - 1;  // op with line0[op] <= g < line0[op + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (line0[mid] <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    const GOp &o = ops[lo];
    const int l = g - line0[lo];
    const double mx = __longlong_as_double((long long)o.mx[l]);
    const int E = mx > 0.0 ? g_exp_above(mx) : 0;
    o.e[l] = E;
    if (mx > 0.0) atomicMax(&need[lo], (E - o.lsb[l] + 6) / 7);
}

// Digit tiles of one 128 x 128 block: S levels, truncated 7-bit digits of
// x * 2^-E (as k_digit_write, cut with integer operations), written in the
// swizzled tile layout.  Each thread holds 16 elements at a time.
template <bool CG>
__device__ __forceinline__ int g_line_e(const int *e, int l) {
    return CG ? __ldcg(e + l) : e[l];
}

// One block of 512 threads cuts block bk of operand o.  CG: the line
// exponents were written by other blocks of the same launch.
template <bool CG>
__device__ __forceinline__ void g_digits_tile(const int4 bk, const GOp &o) {
    const int l0 = bk.y * G_T, k0 = bk.z * G_T;
    const int t = threadIdx.x;
    const size_t level_stride = (size_t)o.tiles_l * o.nkb * G_TILE_BYTES;
    int8_t *tile0 = o.digits + ((size_t)bk.y * o.nkb + bk.z) * G_TILE_BYTES;
    uint64_t m7[16];
    int f[16];
    uint32_t neg[4];
    if (!o.kcontig) {
        // thread: row r, k quarter q (two halves of 16 values); lines contiguous across threads
        const int r = t & 127, q = t >> 7, l = l0 + r;
        const int E = l < o.lines ? g_line_e<CG>(o.e, l) : 0;
        for (int hh = 0; hh < 2; hh++) {
            neg[0] = neg[1] = neg[2] = neg[3] = 0u;
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int kk = k0 + 32 * q + 16 * hh + j;
                const double v = (l < o.lines && kk < o.k) ? o.X[(size_t)l + (size_t)kk * o.ld] : 0.0;
                const DigitCut c = digit_cut(v, E);
                m7[j] = c.m7;
                f[j] = c.f;
                if (v < 0.0) neg[j >> 2] |= 0xffu << (8 * (j & 3));
            }
            const int ch = (2 * q + hh) ^ (r & 7);
            for (int s = 0; s < o.S; s++) {
                uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    w[j >> 2] |= digit_mag(m7[j], f[j]) << (8 * (j & 3));
                    f[j] -= 7;
                }
                int8_t *row = tile0 + s * level_stride + r * 128;
                *reinterpret_cast<int4 *>(row + ch * 16) =
                    make_int4((int)digits_signed(w[0], neg[0]), (int)digits_signed(w[1], neg[1]),
                              (int)digits_signed(w[2], neg[2]), (int)digits_signed(w[3], neg[3]));
            }
        }
    } else {
        // warp: rows w + 16 i (two passes of four rows); lane: k 4 lane .. 4 lane + 3 (k contiguous)
        const int w = t >> 5, lane = t & 31;
        for (int pass = 0; pass < 2; pass++) {
            int E[4];
            neg[0] = neg[1] = neg[2] = neg[3] = 0u;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int l = l0 + w + 16 * (4 * pass + i);
                E[i] = l < o.lines ? g_line_e<CG>(o.e, l) : 0;
#pragma unroll
                for (int qq = 0; qq < 4; qq++) {
                    const int kk = k0 + 4 * lane + qq;
                    const double v = (l < o.lines && kk < o.k) ? o.X[(size_t)l * o.ld + kk] : 0.0;
                    const DigitCut c = digit_cut(v, E[i]);
                    m7[4 * i + qq] = c.m7;
                    f[4 * i + qq] = c.f;
                    if (v < 0.0) neg[i] |= 0xffu << (8 * qq);
                }
            }
            for (int s = 0; s < o.S; s++) {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int r = w + 16 * (4 * pass + i);
                    uint32_t word = 0u;
#pragma unroll
                    for (int qq = 0; qq < 4; qq++) {
                        word |= digit_mag(m7[4 * i + qq], f[4 * i + qq]) << (8 * qq);
                        f[4 * i + qq] -= 7;
                    }
                    int8_t *row = tile0 + s * level_stride + r * 128;
                    *reinterpret_cast<uint32_t *>(row + (((lane >> 2) ^ (r & 7)) * 16) + (lane & 3) * 4) =
                        digits_signed(word, neg[i]);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(512) k_g_digits(const int4 *__restrict__ blocks, const GOp *__restrict__ ops) {
    const int4 bk = blocks[blockIdx.x];
    g_digits_tile<false>(bk, ops[bk.x]);
}

// ---- the whole split in one launch ------------------------------------------
// Statistics, line exponents, digit counts and digits of all operands as one
// cooperative launch (every block resident): three grid barriers separate the
// phases, each a bounded wait (2 s) that reports a timeout instead of hanging.
// The digit buffers are carved, in operand order, from a region the host
// reserved for the largest digit count; the host repeats the same carving
// from the counts it reads back.  err: 1 a barrier timed out, 2 the digits
// need more than the region (the host then allocates and cuts them itself).
struct GSplitArgs {
    const int4 *blocks;
    int nblocks;
    GOp *ops;
    int nops;
    const int *line0;
    int total_lines;
    int *need;
    int cap;
    int8_t *dig_base;
    unsigned long long dig_capacity;
    unsigned *bar;  // three barrier counters and two work counters, zero at launch
    int *err;
    int *mail;      // host-mapped: [0] tag, [1] error so far, [2 + i] digit count of operand i (or null)
    int tag;
};

__device__ __forceinline__ bool g_grid_barrier(unsigned *ctr, int *err) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1u);
        const uint64_t t0 = tc::globaltimer();
        int ok = 1;
        while (*(volatile unsigned *)ctr < gridDim.x) {
            if (tc::globaltimer() - t0 > 2000000000ull) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
            __nanosleep(128);
        }
        __threadfence();
        ok_sh = ok && *(volatile int *)err == 0;
    }
    __syncthreads();
    return ok_sh != 0;
}

// Statistics of one block with 512 threads (as k_g_stats).
__device__ __forceinline__ void g_stats_tile512(const int4 bk, const GOp &o, double *smx, int *slsb) {
    const int l0 = bk.y * G_T, k0 = bk.z * G_T;
    const int t = threadIdx.x;
    if (!o.kcontig) {
        const int l = l0 + (t & 127), kh = k0 + (t >> 7) * 32;
        double mx = 0.0;
        int lsb = 0x7fffffff;
        if (l < o.lines) {
            double v[32];  // every load in flight before the first use
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const int kk = kh + j;
                v[j] = kk < o.k ? o.X[(size_t)l + (size_t)kk * o.ld] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 32; j++) g_stat(v[j], mx, lsb);
        }
        smx[t] = mx;
        slsb[t] = lsb;
        __syncthreads();
        if (t < 128 && l < o.lines) {
            mx = ref_max(ref_max(smx[t], smx[t + 128]), ref_max(smx[t + 256], smx[t + 384]));
            lsb = min(min(slsb[t], slsb[t + 128]), min(slsb[t + 256], slsb[t + 384]));
            if (mx > 0.0) atomicMax(&o.mx[l], (unsigned long long)__double_as_longlong(mx));
            if (lsb != 0x7fffffff) atomicMin(&o.lsb[l], lsb);
        }
        __syncthreads();
    } else {
        const int w = t >> 5, lane = t & 31;
        double v[G_T / 16][4];  // every load of the thread in flight together
#pragma unroll
        for (int i = 0; i < G_T / 16; i++) {
            const int l = l0 + w + 16 * i;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int kk = k0 + 4 * lane + q;
                v[i][q] = (l < o.lines && kk < o.k) ? o.X[(size_t)l * o.ld + kk] : 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < G_T / 16; i++) {
            const int l = l0 + w + 16 * i;
            if (l >= o.lines) break;  // uniform per warp
            double mx = 0.0;
            int lsb = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < 4; q++) g_stat(v[i][q], mx, lsb);
            for (int sft = 16; sft > 0; sft >>= 1) {
                mx = ref_max(mx, __shfl_xor_sync(0xffffffffu, mx, sft));
                lsb = min(lsb, __shfl_xor_sync(0xffffffffu, lsb, sft));
            }
            if (lane == 0) {
                if (mx > 0.0) atomicMax(&o.mx[l], (unsigned long long)__double_as_longlong(mx));
                if (lsb != 0x7fffffff) atomicMin(&o.lsb[l], lsb);
            }
        }
    }
}

__device__ __forceinline__ GOp g_load_op(const GOp *p) {  // through L2: written in this launch
    static_assert(sizeof(GOp) % 8 == 0, "GOp words");
    GOp o;
    unsigned long long w[sizeof(GOp) / 8];
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(GOp) / 8); i++) w[i] = __ldcg(src + i);
    memcpy(&o, w, sizeof(GOp));
    return o;
}

// The next block of the list for this CTA (taken in order from a counter, so
// CTAs that finish early take more).
__device__ __forceinline__ int g_next_block(unsigned *ctr, int *slot) {
    __syncthreads();  // every thread is done with the previous block and its slot
    if (threadIdx.x == 0) *slot = (int)atomicAdd(ctr, 1u);
    __syncthreads();
    return *slot;
}

__global__ void __launch_bounds__(512, 1) k_g_split(const GSplitArgs a) {
    __shared__ double smx[512];
    __shared__ int slsb[512];
    __shared__ int next_sh;
    // 1: per-line max and lowest set bit
    for (int b = g_next_block(&a.bar[3], &next_sh); b < a.nblocks; b = g_next_block(&a.bar[3], &next_sh)) {
        const int4 bk = a.blocks[b];
        g_stats_tile512(bk, a.ops[bk.x], smx, slsb);
    }
    if (!g_grid_barrier(&a.bar[0], a.err)) return;
    // 2: line exponents and each operand's digit need
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < a.total_lines; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = a.nops - 1;  // operand with line0[op] <= g < line0[op + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.line0[mid] <= g)
                lo = mid;
            else
                hi = mid - 1;
        }
        const GOp &o = a.ops[lo];
        const int l = g - a.line0[lo];
        const double mx = __longlong_as_double((long long)__ldcg(&o.mx[l]));
        const int E = mx > 0.0 ? g_exp_above(mx) : 0;
        o.e[l] = E;
        if (mx > 0.0) atomicMax(&a.need[lo], (E - __ldcg(&o.lsb[l]) + 6) / 7);
    }
    if (!g_grid_barrier(&a.bar[1], a.err)) return;
    // digit counts and buffers (the host carves the same ones)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long off = 0;
        for (int i = 0; i < a.nops; i++) {
            int S = __ldcg(&a.need[i]);
            S = S < 1 ? 1 : S;
            if (a.cap > 0 && S > a.cap) S = a.cap;
            a.ops[i].S = S;
            a.ops[i].digits = a.dig_base + off;
            off += g_digit_bytes(S, a.ops[i].tiles_l, a.ops[i].nkb);
        }
        if (off > a.dig_capacity) atomicExch(a.err, 2);
        if (a.mail) {  // post the counts: the host builds the schedules while the digits are cut
            for (int i = 0; i < a.nops; i++) ((volatile int *)a.mail)[2 + i] = a.ops[i].S;
            ((volatile int *)a.mail)[1] = *(volatile int *)a.err;
            __threadfence_system();
            ((volatile int *)a.mail)[0] = a.tag;
            __threadfence_system();
        }
    }
    if (!g_grid_barrier(&a.bar[2], a.err)) return;
    // 3: digits
    for (int b = g_next_block(&a.bar[4], &next_sh); b < a.nblocks; b = g_next_block(&a.bar[4], &next_sh)) {
        const int4 bk = a.blocks[b];
        const GOp o = g_load_op(&a.ops[bk.x]);
        g_digits_tile<true>(bk, o);
    }
}

// ---------------------------------------------------------------------------
// The grouped product kernel (roles and waits as k_i8_gemm)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(G_THREADS, 1) k_i8_grouped(const GParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *bar = (uint64_t *)(smem + G_NST * G_STAGE);
    uint64_t *full = bar, *empty = bar + G_NST, *acc_full = bar + 2 * G_NST, *acc_empty = bar + 2 * G_NST + 2;
    uint64_t *drain = bar + 2 * G_NST + 4;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t_begin = p.cta_begin[blockIdx.x], t_end = p.cta_begin[blockIdx.x + 1];

    if (threadIdx.x == 0) {
        for (int s = 0; s < G_NST; s++) {
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
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, G_TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t stage = 0, phase = 0;
            uint32_t issued = 0, issued_phase = 0;  // per stage: a copy was issued, and the phase it completes
            bool ok = true;
            for (int ti = t_begin; ti < t_end && ok; ti++) {
                const int4 tl = p.tiles[ti];
                const GProb pr = p.probs[tl.x];
                for (int g = 0; g < pr.n_groups && ok; g++) {
                    const int4 grp = p.groups[pr.group0 + g];
                    for (int it = grp.x; it < grp.y && ok; it++) {
                        const int4 item = p.items[it];
                        const int8_t *a0 = pr.da + ((size_t)(item.x * pr.tiles_m + tl.y) * pr.nkb) * G_TILE_BYTES;
                        const int8_t *b0 = pr.db + ((size_t)(item.y * pr.tiles_n + tl.z) * pr.nkb) * G_TILE_BYTES;
                        for (int kb = item.z; kb < item.w; kb++) {
                            if (!tc::mbar_wait(&empty[stage], phase ^ 1, &abort_flag, p.err, GERR_PRODUCER,
                                               G_WAIT_NS)) {
                                ok = false;
                                break;
                            }
                            uint8_t *sa = smem + stage * G_STAGE, *sb = sa + G_TILE_BYTES;
                            tc::mbar_arrive_expect_tx(&full[stage], G_STAGE);
                            tc::bulk_load(sa, a0 + (size_t)kb * G_TILE_BYTES, G_TILE_BYTES, &full[stage]);
                            tc::bulk_load(sb, b0 + (size_t)kb * G_TILE_BYTES, G_TILE_BYTES, &full[stage]);
                            issued |= 1u << stage;
                            issued_phase = (issued_phase & ~(1u << stage)) | (phase << stage);
                            if (++stage == G_NST) {
                                stage = 0;
                                phase ^= 1;
                            }
                        }
                    }
                }
            }
            if (!ok) tc::drain_copies(full, G_NST, issued, issued_phase);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(G_T, G_T);
            uint32_t stage = 0, phase = 0, abuf = 0, aphase = 0;
            bool ok = true, issued = false;
            for (int ti = t_begin; ti < t_end && ok; ti++) {
                const GProb pr = p.probs[p.tiles[ti].x];
                for (int g = 0; g < pr.n_groups && ok; g++) {
                    const int4 grp = p.groups[pr.group0 + g];
                    if (!tc::mbar_wait(&acc_empty[abuf], aphase ^ 1, &abort_flag, p.err, GERR_MMA, G_WAIT_NS)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t tmem_d = tmem_base + abuf * G_T;
                    uint32_t accumulate = 0;
                    for (int it = grp.x; it < grp.y && ok; it++) {
                        const int4 item = p.items[it];
                        for (int kb = item.z; kb < item.w; kb++) {
                            if (!tc::mbar_wait(&full[stage], phase, &abort_flag, p.err, GERR_MMA, G_WAIT_NS)) {
                                ok = false;
                                break;
                            }
                            tc::fence_after_sync();
                            const uint32_t sa = tc::smem_u32(smem + stage * G_STAGE), sb = sa + G_TILE_BYTES;
                            const uint64_t adesc = tc::smem_desc_k_sw128(sa), bdesc = tc::smem_desc_k_sw128(sb);
#pragma unroll
                            for (int kk = 0; kk < G_T / 32; kk++) {
                                tc::mma_i8(tmem_d, adesc + 2 * kk, bdesc + 2 * kk, idesc, accumulate);
                                accumulate = 1;
                            }
                            issued = true;
                            tc::mma_commit(&empty[stage]);
                            if (++stage == G_NST) {
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
            if (!ok && issued) {
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
        const uint32_t rcol = G_RCOL + half * 128;
        uint32_t abuf = 0, aphase = 0;
        bool ok = true;
        for (int ti = t_begin; ti < t_end && ok; ti++) {
            const int4 tl = p.tiles[ti];
            const GProb *pr = p.probs + tl.x;  // fields read where used (registers go to the sums)
            const int gr = tl.y * G_T + row;
            const int ng = __ldg(&pr->n_groups), g0 = __ldg(&pr->group0);
            double acc[64];
#pragma unroll
            for (int c = 0; c < 64; c++) acc[c] = 0.0;
            for (int g = 0; g < ng; g++) {
                const int4 grp = p.groups[g0 + g];
                const int meta = grp.w;
                if (!tc::mbar_wait(&acc_full[abuf], aphase, &abort_flag, p.err, GERR_EPI, G_WAIT_NS)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const double sc = pow2(meta & 0xff);
                const uint32_t taddr = lane_base + abuf * G_T + half * 64;
                uint32_t v[32];
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
                if (meta & (1 << 8)) {
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
                            const int pm = __ldg(&pr->m);
                            if (gr < pm) {
                                const int pn = __ldg(&pr->n), ldc = __ldg(&pr->ldc);
                                const double al = __ldg(&pr->alpha), be = __ldg(&pr->beta);
                                double *Cp = pr->C;
                                const int *ebp = pr->eb;
                                const int ea = pr->ea[gr];
#pragma unroll
                                for (int e = 0; e < 16; e++) {
                                    const int gc = tl.z * G_T + half * 64 + ch * 16 + e;
                                    if (gc < pn) {
                                        double *cp = &Cp[(size_t)gc * ldc + gr];
                                        const double t = scalbn(r[e], ea + ebp[gc]);
                                        *cp = fma(al, t, be * *cp);
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
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, G_TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int i8_schedule_into(int nA, int nB, int nkb, bool triangular, int4 *items, int max_items, int *ni, int4 *groups,
                     int max_groups, int *ng);  // gemm_i8.cu

constexpr int kI8DefaultCapG = 19;  // as gemm_i8.cu's kI8DefaultCap

// Output tiles of all problems to CTAs.  mode 0: problems by decreasing tile
// cost, each tile onto the least loaded CTA (longest first); mode 1: the same
// problem order, each problem's tiles in strips of up to 12 tile rows
// (column-major inside a strip) dealt round-robin, so CTAs running at the same
// time share a problem's panels in L2.
static void deal_tiles(int mode, int grid, const std::vector<GProb> &probs, const std::vector<int> &order,
                       const std::vector<double> &cost, std::vector<int4> &tiles, std::vector<int> &cta_begin) {
    std::vector<std::vector<int4>> per_cta((size_t)grid);
    if (mode == 0) {
        using Load = std::pair<double, int>;
        std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
        for (int c = 0; c < grid; c++) heap.push(Load(0.0, c));
        for (int b : order) {
            const GProb &pr = probs[(size_t)b];
            if (pr.m <= 0 || pr.n <= 0) continue;
            for (int tn = 0; tn < pr.tiles_n; tn++)
                for (int tm = 0; tm < pr.tiles_m; tm++) {
                    Load l = heap.top();
                    heap.pop();
                    per_cta[(size_t)l.second].push_back(make_int4(b, tm, tn, 0));
                    l.first += cost[(size_t)b];
                    heap.push(l);
                }
        }
    } else {
        int next = 0;
        for (int b : order) {
            const GProb &pr = probs[(size_t)b];
            if (pr.m <= 0 || pr.n <= 0) continue;
            const int strip = pr.tiles_m < 12 ? pr.tiles_m : 12;
            for (int s0 = 0; s0 < pr.tiles_m; s0 += strip) {
                const int rows = pr.tiles_m - s0 < strip ? pr.tiles_m - s0 : strip;
                for (int tn = 0; tn < pr.tiles_n; tn++)
                    for (int r = 0; r < rows; r++) {
                        per_cta[(size_t)next].push_back(make_int4(b, s0 + r, tn, 0));
                        next = next + 1 == grid ? 0 : next + 1;
                    }
            }
        }
    }
    tiles.clear();
    cta_begin.assign((size_t)grid + 1, 0);
    for (int c = 0; c < grid; c++) {
        cta_begin[(size_t)c + 1] = cta_begin[(size_t)c] + (int)per_cta[(size_t)c].size();
        tiles.insert(tiles.end(), per_cta[(size_t)c].begin(), per_cta[(size_t)c].end());
    }
}

int gemm_i8_batched(cuozblasHandle_t *h, char ta, char tb, int count, const int *m, const int *n, const int *k,
                    const double *alpha, const double *const *A, const int *lda, const double *const *B,
                    const int *ldb, const double *beta, double *const *C, const int *ldc) {
    State *st = state(h);
    cudaStream_t s = st->stream;
    Arena ar(h);
    const int cap = h->nSplitMax > 0 ? h->nSplitMax : kI8DefaultCapG;
    // operands 2b (op(A) of problem b) and 2b + 1 (op(B))
    std::vector<GOp> ops((size_t)2 * count);
    std::vector<int> line0((size_t)2 * count + 1, 0);
    std::vector<int4> blocks;
    for (int b = 0; b < count; b++) {
        const int nkb = k[b] > 0 ? (k[b] + G_T - 1) / G_T : 1;
        GOp &oa = ops[(size_t)2 * b], &ob = ops[(size_t)2 * b + 1];
        oa = GOp{A[b], lda[b], m[b], k[b], is_trans(ta) ? 1 : 0, (m[b] + G_T - 1) / G_T, nkb, 0,
                 nullptr, nullptr, nullptr, nullptr};
        ob = GOp{B[b], ldb[b], n[b], k[b], is_trans(tb) ? 0 : 1, (n[b] + G_T - 1) / G_T, nkb, 0,
                 nullptr, nullptr, nullptr, nullptr};
        for (int o = 0; o < 2; o++) {
            const GOp &op = ops[(size_t)2 * b + o];
            line0[(size_t)2 * b + o + 1] = line0[(size_t)2 * b + o] + op.lines;
            // k = 0 included: its single block of zero digits makes C = beta * C
            for (int tl = 0; tl < op.tiles_l; tl++)
                for (int kb = 0; kb < op.nkb; kb++) blocks.push_back(make_int4(2 * b + o, tl, kb, 0));
        }
    }
    const int nops = 2 * count, total_lines = line0[(size_t)nops];
    // per-line exponents and statistics of all operands, one array each
    const uint64_t tl_alloc = (uint64_t)(total_lines > 0 ? total_lines : 1);
    int *all_e = ar.take<int>(tl_alloc);
    unsigned long long *all_mx = ar.take<unsigned long long>(tl_alloc);
    int *all_lsb = ar.take<int>(tl_alloc);
    GOp *d_ops = ar.take<GOp>((uint64_t)nops);
    int *d_line0 = ar.take<int>((uint64_t)nops + 1);
    int *d_need = ar.take<int>((uint64_t)nops);
    int4 *d_blocks = ar.take<int4>(blocks.size() > 0 ? blocks.size() : 1);
    unsigned *d_bar = ar.take<unsigned>(8);
    int *d_serr = ar.take<int>(1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    for (int o = 0; o < nops; o++) {
        GOp &op = ops[(size_t)o];
        op.e = all_e + line0[(size_t)o];
        op.mx = all_mx + line0[(size_t)o];
        op.lsb = all_lsb + line0[(size_t)o];
    }
    // The split in one cooperative launch when every block can be resident and
    // the digits of the largest count fit a reserved region; otherwise three
    // launches (statistics, lines, digits) with the digits allocated after the
    // counts are read.
    unsigned long long dig_bound = 0;
    for (const GOp &op : ops) dig_bound += g_digit_bytes(cap, op.tiles_l, op.nkb);
    const uint64_t mk_dig = ar.mark();
    int8_t *dig_region = ar.take<int8_t>(dig_bound + 1);
    int coop_grid = 0;
    if (ar.ok && !blocks.empty() && total_lines > 0 && !st->env.g_split3) {
        int dev = 0;
        OZB_CHECK(cudaGetDevice(&dev));
        static std::atomic<int> occ_cache[64];
        int occ = dev >= 0 && dev < 64 ? occ_cache[dev].load() : 0;
        if (occ == 0) {
            int coop = 0;
            if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_g_split, 512, 0) == cudaSuccess && occ > 0) {
                if (dev >= 0 && dev < 64) occ_cache[dev].store(occ);
            } else {
                cudaGetLastError();
                occ = -1;
                if (dev >= 0 && dev < 64) occ_cache[dev].store(-1);
            }
        }
        if (occ > 0) {
            const int64_t g = (int64_t)occ * sm_count();
            coop_grid = (int)((int64_t)blocks.size() < g ? (int64_t)blocks.size() : g);
        }
    }
    if (coop_grid < 1) {
        ar.ok = true;
        ar.release(mk_dig);
        dig_region = nullptr;
    }
    OZB_CHECK(cudaMemsetAsync(all_mx, 0, tl_alloc * sizeof(unsigned long long), s));
    OZB_CHECK(cudaMemsetAsync(all_lsb, 0x7f, tl_alloc * sizeof(int), s));
    OZB_CHECK(cudaMemsetAsync(d_need, 0, (size_t)nops * sizeof(int), s));
    OZB_CHECK(cudaMemsetAsync(d_bar, 0, 8 * sizeof(unsigned), s));
    OZB_CHECK(cudaMemsetAsync(d_serr, 0, sizeof(int), s));
    size_t staged = 0;  // bytes of the handle's pinned staging used by this call
    OZB_CHECK(stage_upload(st, d_ops, ops.data(), sizeof(GOp) * nops, staged));
    OZB_CHECK(stage_upload(st, d_line0, line0.data(), sizeof(int) * (nops + 1), staged));
    OZB_CHECK(stage_upload(st, d_blocks, blocks.data(), sizeof(int4) * blocks.size(), staged));
    ev_record(h, 0);
    bool fused = coop_grid > 0;
    if (fused) {
        GSplitArgs ga;
        ga.blocks = d_blocks;
        ga.nblocks = (int)blocks.size();
        ga.ops = d_ops;
        ga.nops = nops;
        ga.line0 = d_line0;
        ga.total_lines = total_lines;
        ga.need = d_need;
        ga.cap = cap;
        ga.dig_base = dig_region;
        ga.dig_capacity = dig_bound;
        ga.bar = d_bar;
        ga.err = d_serr;
        const bool mail = st->h_mail != nullptr && nops + 2 <= kMailInts;
        if (mail) {
            st->mail_seq = st->mail_seq == 0x7fffffff ? 1 : st->mail_seq + 1;
            ((volatile int *)st->h_mail)[0] = 0;
        }
        ga.mail = mail ? st->d_mail : nullptr;
        ga.tag = st->mail_seq;
        void *args[] = {&ga};
        counted(h);
        if (cudaLaunchCooperativeKernel((const void *)k_g_split, dim3(coop_grid), dim3(512), args, 0, s) !=
            cudaSuccess) {
            cudaGetLastError();  // not launched: the three-launch split
            fused = false;
            ar.release(mk_dig);
            dig_region = nullptr;
        }
    }
    if (!fused) {
        if (!blocks.empty()) {
            counted(h);
            k_g_stats<<<(unsigned)blocks.size(), 256, 0, s>>>(d_blocks, d_ops);
        }
        if (total_lines > 0) {
            counted(h);
            k_g_lines<<<(total_lines + 255) / 256, 256, 0, s>>>(d_ops, d_line0, nops, total_lines, d_need);
        }
    }
    OZB_CHECK(cudaGetLastError());
    std::vector<int> need((size_t)nops + 1);
    // The fused split posts the digit counts to host memory before it cuts
    // the digits: wait for that post (bounded), not for the kernel.
    bool posted = false;
    if (fused && st->h_mail != nullptr && nops + 2 <= kMailInts) {
        volatile int *mb = st->h_mail;
        const double t0 = wall_seconds();
        for (uint32_t it = 0;; it++) {
            if (mb[0] == st->mail_seq) {
                posted = true;
                break;
            }
            if ((it & 1023) == 1023 && (cudaStreamQuery(s) != cudaErrorNotReady || wall_seconds() - t0 > 5.0)) {
                posted = mb[0] == st->mail_seq;
                break;
            }
        }
        if (posted) {
            std::atomic_thread_fence(std::memory_order_acquire);
            for (int o = 0; o < nops; o++) need[(size_t)o] = mb[2 + o];
            need[(size_t)nops] = mb[1];
        }
    }
    if (!posted) {
        OZB_CHECK(cudaMemcpyAsync(need.data(), d_need, sizeof(int) * nops, cudaMemcpyDeviceToHost, s));
        OZB_CHECK(cudaMemcpyAsync(need.data() + nops, d_serr, sizeof(int), cudaMemcpyDeviceToHost, s));
        OZB_CHECK(cudaStreamSynchronize(s));
    }
    const int serr = fused ? need[(size_t)nops] : 0;
    if (serr == 1) {
        fprintf(stderr, "cuozblas: grouped INT8 split: a grid barrier timed out\n");
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    if (serr == 2 && posted) OZB_CHECK(cudaStreamSynchronize(s));  // the kernel stops there: digits below
    const bool carved = fused && serr == 0;  // the launch cut the digits into the region
    if (!carved && dig_region) {
        ar.release(mk_dig);
        dig_region = nullptr;
    }
    int maxA = 0, maxB = 0;
    unsigned long long off = 0;
    for (int o = 0; o < nops; o++) {
        GOp &op = ops[(size_t)o];
        op.S = need[(size_t)o] < 1 ? 1 : need[(size_t)o];
        if (op.S > cap) op.S = cap;
        if (carved) {  // the same carving as the device's
            op.digits = dig_region + off;
            off += g_digit_bytes(op.S, op.tiles_l, op.nkb);
        } else {
            op.digits = ar.take<int8_t>((uint64_t)op.S * op.tiles_l * op.nkb * G_TILE_BYTES + 1);
        }
        if (o & 1)
            maxB = op.S > maxB ? op.S : maxB;
        else
            maxA = op.S > maxA ? op.S : maxA;
    }
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    if (!carved && !blocks.empty()) {
        OZB_CHECK(stage_upload(st, d_ops, ops.data(), sizeof(GOp) * nops, staged));
        counted(h);
        k_g_digits<<<(unsigned)blocks.size(), 512, 0, s>>>(d_blocks, d_ops);
        OZB_CHECK(cudaGetLastError());
    }
    ev_record(h, 1);
    // This runs on the host while the split is still cutting digits, so it
    // builds only what the launch needs: once the product kernel and dealing
    // order of this problem set are measured, only that kernel's schedules and
    // that dealing order.
    const bool tri = h->fastMode != 0;
    std::vector<GProb> probs((size_t)count);
    std::vector<double> cost((size_t)count, 0.0);
    int npairs_max = 0;
    {
        // per problem: its pairs and a tile cost for the deal (k-blocks over all
        // pairs plus two per INT32 group of the level-wise schedule, whose
        // groups fill G_MAX_TERMS / 128 k-blocks within one level)
        const int64_t kb_cap = G_MAX_TERMS / G_T;
        for (int b = 0; b < count; b++) {
            const GOp &oa = ops[(size_t)2 * b], &ob = ops[(size_t)2 * b + 1];
            const int nA = oa.S, nB = ob.S, nkb = oa.nkb;
            const int maxlevel = tri ? (nA < nB ? nA : nB) - 1 : nA + nB - 2;
            int64_t np = 0, ng = 0;
            for (int L = 0; L <= maxlevel; L++) {
                const int lo = L - (nB - 1) > 0 ? L - (nB - 1) : 0, hi = L < nA - 1 ? L : nA - 1;
                np += hi - lo + 1;
                ng += ((int64_t)(hi - lo + 1) * nkb + kb_cap - 1) / kb_cap;
            }
            npairs_max = np > npairs_max ? (int)np : npairs_max;
            cost[(size_t)b] = (double)np * nkb + 2.0 * (double)ng;
            probs[(size_t)b] = GProb{m[b], n[b], ldc[b], nkb, oa.tiles_l, ob.tiles_l, 0, 0,
                                     oa.digits, ob.digits, oa.e, ob.e, alpha[b], beta[b], C[b]};
        }
    }
    std::vector<int> order((size_t)count);
    for (int b = 0; b < count; b++) order[(size_t)b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[(size_t)a] > cost[(size_t)b]; });
    const int nsm = sm_count();
    int ntile_total = 0;
    for (int b = 0; b < count; b++)
        if (m[b] > 0 && n[b] > 0) ntile_total += probs[(size_t)b].tiles_m * probs[(size_t)b].tiles_n;
    const int grid = ntile_total < nsm ? (ntile_total > 0 ? ntile_total : 1) : nsm;
    // Candidates {kernel, dealing order}: kernel 2 level-blocked with blocks cut
    // across the runs (per problem, where the cut applies: a crossing block
    // needs a single K chunk), 1 level-blocked within the runs, 0 level-wise.
    // OZBLAS_I8_BLOCK = w > 0 keeps kernel 1 at width w, w < 0 kernel 2 at -w;
    // OZBLAS_I8_LEVELWISE kernel 0.
    const int eb = st->env.i8_block;
    const bool want_lw = st->env.i8_levelwise || eb == 0;
    const int bw = eb != 0 ? (eb < 0 ? -eb : eb) : kBlkMaxWidth;
    const bool blk_on = !st->env.i8_levelwise && ntile_total > 0;
    const bool forms[2] = {blk_on && eb >= 0, blk_on && eb <= 0};
    std::vector<std::pair<int, int>> cands;
    for (int f = 1; f >= 0; f--)
        if (forms[f]) {
            cands.push_back({f + 1, 0});
            cands.push_back({f + 1, 1});
        }
    if (want_lw || cands.empty()) {
        cands.push_back({0, 0});
        cands.push_back({0, 1});
    }
    uint64_t hk = tune_hash(&count, sizeof(count));
    for (const GOp &o : ops) {
        const int sig[3] = {o.lines, o.k, o.S};
        hk = tune_hash(sig, sizeof(sig), hk);
    }
    char key[112];
    snprintf(key, sizeof(key), "i8grouped:%016llx:%d:%d:%d:%d:%d", (unsigned long long)hk, tri ? 1 : 0, grid, bw,
             (forms[0] ? 1 : 0) + (forms[1] ? 2 : 0), want_lw ? 1 : 0);
    int pick = ntile_total > 0 ? tune_cached(key, (int)cands.size(), 0) : 0;  // -1: not measured yet
    auto needed = [&](int kernel, int deal) {
        if (pick >= 0) return cands[(size_t)pick].first == kernel && (deal < 0 || cands[(size_t)pick].second == deal);
        for (const auto &c : cands)
            if (c.first == kernel && (deal < 0 || c.second == deal)) return true;
        return false;
    };
    // the level-blocked schedules of the forms needed
    std::vector<BlkStep> bsteps;  // the forms' step lists, one after the other
    std::vector<BlkProb> bprobs[2];
    bool blk_failed = false;
    for (int f = 0; f < 2 && !blk_failed; f++) {
        if (!forms[f] || !needed(f + 1, -1)) continue;
        bprobs[f].resize((size_t)count);
        std::vector<BlkStep> one;
        for (int b = 0; b < count && !blk_failed; b++) {
            const GOp &oa = ops[(size_t)2 * b], &ob = ops[(size_t)2 * b + 1];
            const GProb &pr = probs[(size_t)b];
            blk_failed = !((f == 1 && blk_schedule(oa.S, ob.S, oa.nkb, tri, bw, one, true)) ||
                           blk_schedule(oa.S, ob.S, oa.nkb, tri, bw, one));
            bprobs[f][(size_t)b] = BlkProb{pr.m, pr.n, pr.ldc, pr.nkb, pr.tiles_m, pr.tiles_n,
                                           blk_kq_last(oa.k, pr.nkb), oa.S, ob.S,
                                           (int)bsteps.size(), (int)one.size(), pr.da, pr.db, pr.ea, pr.eb,
                                           pr.alpha, pr.beta, pr.C};
            bsteps.insert(bsteps.end(), one.begin(), one.end());
        }
    }
    if (blk_failed) {  // levels beyond the level-blocked kernel's range: the level-wise kernel, measured
        cands = {{0, 0}, {0, 1}};
        pick = -1;
        bsteps.clear();
        bprobs[0].clear();
        bprobs[1].clear();
    }
    const bool blk = !bsteps.empty();
    // the level-wise schedules, written in place: a pair spans at most
    // nkb / (k-blocks per INT32 group) + 2 items, a group holds at least one item
    std::vector<int4> items, groups;
    if (needed(0, -1)) {
        size_t cap_items = 0;
        for (int b = 0; b < count; b++) {
            const GOp &oa = ops[(size_t)2 * b], &ob = ops[(size_t)2 * b + 1];
            cap_items += (size_t)oa.S * ob.S * (size_t)(oa.nkb / (G_MAX_TERMS / G_T) + 2);
        }
        items.resize(cap_items > 0 ? cap_items : 1);
        groups.resize(cap_items > 0 ? cap_items : 1);
        size_t ni_tot = 0, ng_tot = 0;
        for (int b = 0; b < count; b++) {
            const GOp &oa = ops[(size_t)2 * b], &ob = ops[(size_t)2 * b + 1];
            const size_t cap_b = (size_t)oa.S * ob.S * (size_t)(oa.nkb / (G_MAX_TERMS / G_T) + 2);
            int ni = 0, ng = 0;
            const int np = i8_schedule_into(oa.S, ob.S, oa.nkb, tri, items.data() + ni_tot, (int)cap_b, &ni,
                                            groups.data() + ng_tot, (int)cap_b, &ng);
            if (np < 0) return CUOZBLAS_STATUS_NOT_SUPPORTED;
            for (int g = 0; g < ng; g++) {
                groups[ng_tot + (size_t)g].x += (int)ni_tot;
                groups[ng_tot + (size_t)g].y += (int)ni_tot;
            }
            probs[(size_t)b].group0 = (int)ng_tot;
            probs[(size_t)b].n_groups = ng;
            ni_tot += (size_t)ni;
            ng_tot += (size_t)ng;
        }
        items.resize(ni_tot);
        groups.resize(ng_tot);
    }
    // the tile deals needed
    std::vector<int4> tiles[2];
    std::vector<int> cta_begin[2];
    for (int d = 0; d < 2; d++) {
        bool use = false;
        for (int kernel = 0; kernel < 3; kernel++) use = use || needed(kernel, d);
        if (use) deal_tiles(d, grid, probs, order, cost, tiles[d], cta_begin[d]);
        cta_begin[d].resize((size_t)grid + 1, 0);
    }
    GProb *d_probs = ar.take<GProb>((uint64_t)count);
    int4 *d_sched = ar.take<int4>(items.size() + groups.size() + tiles[0].size() + tiles[1].size() + 1);
    int *d_cta = ar.take<int>(2 * ((uint64_t)grid + 1));
    int *d_err = ar.take<int>(1);
    BlkProb *d_bprobs = nullptr;  // form 0's problems, then form 1's
    BlkStep *d_bsteps = nullptr;
    double *rbuf = nullptr;
    if (blk) {
        d_bprobs = ar.take<BlkProb>((uint64_t)2 * count);
        d_bsteps = ar.take<BlkStep>(bsteps.size() + 1);
        rbuf = ar.take<double>((uint64_t)grid * G_T * G_T);
    }
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(stage_upload(st, d_probs, probs.data(), sizeof(GProb) * count, staged));
    {  // items, groups, both tile lists and both CTA ranges, one after the other
        int4 *dst = d_sched;
        for (const std::vector<int4> *v : {&items, &groups, &tiles[0], &tiles[1]}) {
            OZB_CHECK(stage_upload(st, dst, v->data(), sizeof(int4) * v->size(), staged));
            dst += v->size();
        }
        for (int d = 0; d < 2; d++)
            OZB_CHECK(stage_upload(st, d_cta + (size_t)d * (grid + 1), cta_begin[d].data(),
                                   sizeof(int) * cta_begin[d].size(), staged));
    }
    if (blk) {
        for (int f = 0; f < 2; f++)
            if (!bprobs[f].empty())
                OZB_CHECK(stage_upload(st, d_bprobs + (size_t)f * count, bprobs[f].data(), sizeof(BlkProb) * count,
                                       staged));
        OZB_CHECK(stage_upload(st, d_bsteps, bsteps.data(), sizeof(BlkStep) * bsteps.size(), staged));
    }
    OZB_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    GParams gp;
    gp.probs = d_probs;
    gp.items = d_sched;
    gp.groups = d_sched + items.size();
    gp.tiles = d_sched + items.size() + groups.size();
    gp.cta_begin = d_cta;
    gp.err = d_err;
    const int4 *tiles_dev[2] = {gp.tiles, gp.tiles + tiles[0].size()};
    const int *cta_dev[2] = {d_cta, d_cta + grid + 1};
    auto launch = [&](int kernel, int deal, const GProb *pl, const BlkProb *pb) -> int {
        if (kernel >= 1)
            return i8_blk_grouped_kernel(grid, pb + (size_t)(kernel - 1) * count, d_bsteps, tiles_dev[deal],
                                         cta_dev[deal], rbuf, d_err, s) ==
                           cudaSuccess
                       ? 0
                       : (int)CUOZBLAS_STATUS_CUDA_ERROR;
        GParams gt = gp;
        gt.probs = pl;
        gt.tiles = tiles_dev[deal];
        gt.cta_begin = cta_dev[deal];
        k_i8_grouped<<<grid, G_THREADS, G_SMEM, s>>>(gt);
        return cudaGetLastError() == cudaSuccess ? 0 : (int)CUOZBLAS_STATUS_CUDA_ERROR;
    };
    if (ntile_total > 0) {
        static std::atomic<uint64_t> attr{0};  // devices already opted in
        OZB_CHECK(smem_optin((const void *)k_i8_grouped, G_SMEM, attr));
    }
    if (ntile_total > 0 && pick < 0) {
        // kernel and dealing order: same bits either way, the fastest is measured
        // once per problem set (candidates write scratch products with beta = 0)
        pick = 0;
        const uint64_t mk = ar.mark();
        size_t outs = 0;
        for (const GProb &pr : probs) outs += (size_t)(pr.m > 0 ? pr.m : 0) * (size_t)(pr.n > 0 ? pr.n : 0);
        double *scratch = ar.take<double>(outs + 1);
        GProb *d_trial = ar.take<GProb>((uint64_t)count);
        BlkProb *d_btrial = blk ? ar.take<BlkProb>((uint64_t)2 * count) : nullptr;
        if (ar.ok && cands.size() > 1) {
            std::vector<GProb> trial(probs);
            std::vector<BlkProb> btrial[2] = {bprobs[0], bprobs[1]};
            size_t off = 0;
            for (int b = 0; b < count; b++) {
                GProb &pr = trial[(size_t)b];
                pr.C = scratch + off;
                pr.ldc = pr.m > 1 ? pr.m : 1;
                pr.beta = 0.0;
                for (int f = 0; f < 2; f++)
                    if (!btrial[f].empty()) {
                        btrial[f][(size_t)b].C = pr.C;
                        btrial[f][(size_t)b].ldc = pr.ldc;
                        btrial[f][(size_t)b].beta = 0.0;
                    }
                off += (size_t)(pr.m > 0 ? pr.m : 0) * (size_t)(pr.n > 0 ? pr.n : 0);
            }
            OZB_CHECK(stage_upload(st, d_trial, trial.data(), sizeof(GProb) * count, staged));
            for (int f = 0; f < 2; f++)
                if (!btrial[f].empty())
                    OZB_CHECK(stage_upload(st, d_btrial + (size_t)f * count, btrial[f].data(),
                                           sizeof(BlkProb) * count, staged));
            pick = tune_pick(key, (int)cands.size(), 0, s, [&](int i) {
                return launch(cands[(size_t)i].first, cands[(size_t)i].second, d_trial, d_btrial);
            });
        }
        ar.ok = true;
        ar.release(mk);
    }
    if (pick < 0) pick = 0;
    h->nSplitA = (float)maxA;
    h->nSplitB = (float)maxB;
    h->nSplitC = (float)npairs_max;
    ev_record(h, 2);
    if (ntile_total > 0) {
        counted(h);
        const int r = launch(cands[(size_t)pick].first, cands[(size_t)pick].second, d_probs, d_bprobs);
        if (r != 0) {
            OZB_CHECK(cudaGetLastError());
            return r;
        }
    }
    ev_record(h, 3);
    int herr = 0, serr_end = 0;
    OZB_CHECK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (carved) OZB_CHECK(cudaMemcpyAsync(&serr_end, d_serr, sizeof(int), cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaStreamSynchronize(s));
    if (serr_end != 0) {
        fprintf(stderr, "cuozblas: grouped INT8 split: a grid barrier timed out\n");
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    if (herr != 0) {
        fprintf(stderr, "cuozblas: grouped INT8 GEMM kernel wait timed out (code %d)\n", herr);
        return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
    }
    h->t_SplitA = ev_ms(h, 0, 1) * 1e-3f;
    h->t_SplitB = 0.f;
    h->t_comp = ev_ms(h, 2, 3) * 1e-3f;
    h->t_sum = 0.f;
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb

extern "C" int cuozblasDgemmI8Batched(cuozblasHandle_t *h, char transa, char transb, int32_t count, const int32_t *m,
                                      const int32_t *n, const int32_t *k, const double *alpha,
                                      const double *const *A, const int32_t *lda, const double *const *B,
                                      const int32_t *ldb, const double *beta, double *const *C,
                                      const int32_t *ldc) {
    using namespace ozb;
    OZB_TRY(counter_init(h));
    if (count < 0 || h->nSplitMax < 0 || h->nSplitMax > 64) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (count == 0) return CUOZBLAS_STATUS_SUCCESS;
    if (!m || !n || !k || !alpha || !A || !lda || !B || !ldb || !beta || !C || !ldc)
        return CUOZBLAS_STATUS_INVALID_VALUE;
    for (int b = 0; b < count; b++) {
        if (m[b] < 0 || n[b] < 0 || k[b] < 0 || ldc[b] < (m[b] > 1 ? m[b] : 1)) return CUOZBLAS_STATUS_INVALID_VALUE;
        const int rows_a = is_trans(transa) ? k[b] : m[b], rows_b = is_trans(transb) ? n[b] : k[b];
        if (lda[b] < (rows_a > 1 ? rows_a : 1) || ldb[b] < (rows_b > 1 ? rows_b : 1))
            return CUOZBLAS_STATUS_INVALID_VALUE;
    }
    return gemm_i8_batched(h, transa, transb, count, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}
