// gemm_i8_blk_grouped.cu — the level-blocked INT8 product kernel for the
// grouped call (cuozblasDgemmI8Batched): many problems of different shapes,
// digit counts and schedules in one persistent launch.
//
// The arithmetic, the roles and the schedule are those of k_i8_blk
// (gemm_i8_blk.cu): per output tile, blocks of up to four consecutive levels
// accumulated at once in four INT32 tensor-memory accumulators, one A plane
// and at most one new B plane loaded per A plane of a K step, two MMA issuers
// owning alternate levels, eight epilogue warps combining each block into the
// run accumulator and each run into R with the TwoSum carry.  So every problem
// is bit-identical to its own cuozblasDgemmI8 call.  What differs here:
//  * each CTA walks its own list of output tiles {problem, tm, tn}, dealt by
//    the host, and reads the tile's problem (shape, digit counts, schedule,
//    operands, alpha, beta, C) from a table;
//  * the digit planes are stored as 16 KB tiles with the 128-byte swizzle
//    already applied (the grouped split's layout), so the producer fetches
//    each with one contiguous bulk copy (cp.async.bulk, no tensor map, no
//    multicast);
//  * the last K step of a problem issues only the 32-wide MMAs that reach k
//    (the digits beyond k are zeros, so the skipped MMAs would add nothing):
//    the batch's small problems have k tails of every length;
//  * at the end of a tile the epilogue scales R into C in a pass of its own,
//    so the problem's output fields are not held in registers across the
//    steps (with them held, the epilogue warps spilled);
//  * a problem's schedule may cut its blocks across the runs of levels (as
//    k_i8_blk<true> does): the epilogue then walks a block in one or two
//    segments, flushing the run that ends inside the block before it reads
//    the levels above.
#include <cuda.h>

#include <atomic>

#include "gemm_i8_blk.h"
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "tc05.cuh"

namespace ozb {

struct BlkGParams {
    const BlkProb *probs;
    const BlkStep *steps;  // every problem's schedule, problem b's at steps[probs[b].step0]
    const int4 *tiles;     // {problem, tm, tn, 0}
    const int *cta_begin;  // CTA c runs tiles [cta_begin[c], cta_begin[c + 1])
    double *rbuf;          // per CTA: 128 x 128 doubles, [col][row]
    int *err;
};

// What the three roles need of one output tile.
struct BlkCtx {
    int tm, tn, nA, nB, n_steps, tiles_m, tiles_n, nkb, kq_last;
    const BlkStep *steps;
    const int8_t *da, *db;
};

__device__ __forceinline__ BlkCtx blk_ctx(const BlkGParams &p, int t) {
    BlkCtx c;
    const int4 tl = p.tiles[t];
    const BlkProb *pr = p.probs + tl.x;
    c.tm = tl.y;
    c.tn = tl.z;
    c.nA = pr->nA;
    c.nB = pr->nB;
    c.n_steps = pr->n_steps;
    c.tiles_m = pr->tiles_m;
    c.tiles_n = pr->tiles_n;
    c.nkb = pr->nkb;
    c.kq_last = pr->kq_last;
    c.steps = p.steps + pr->step0;
    c.da = pr->da;
    c.db = pr->db;
    return c;
}

// A grouped tile's output: read when its R is complete.
struct BlkOut {
    int tn, m, n, ldc;
    const int *ea, *eb;
    double alpha, beta;
    double *C;
};

__device__ __forceinline__ BlkOut blk_out(const BlkGParams &p, int t) {
    BlkOut o;
    const int4 tl = p.tiles[t];
    const BlkProb *pr = p.probs + tl.x;
    o.tn = tl.z;
    o.m = pr->m;
    o.n = pr->n;
    o.ldc = pr->ldc;
    o.ea = pr->ea;
    o.eb = pr->eb;
    o.alpha = pr->alpha;
    o.beta = pr->beta;
    o.C = pr->C;
    return o;
}

__global__ void __launch_bounds__(KB_THREADS, 1)
    k_i8_blk_grouped(const __grid_constant__ BlkGParams p, uint64_t wait_ns, int hold_copies) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *ringA = smem, *ringB = smem + KB_RA * KB_TILE;
    uint64_t *bar = (uint64_t *)(smem + (KB_RA + KB_RB) * KB_TILE);
    uint64_t *fullA = bar, *emptyA = bar + KB_RA, *fullB = bar + 2 * KB_RA, *emptyB = bar + 2 * KB_RA + KB_RB;
    uint64_t *acc_full = bar + 2 * KB_RA + 2 * KB_RB, *acc_empty = acc_full + 1, *drain = acc_full + 2;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t_begin = p.cta_begin[blockIdx.x], t_end = p.cta_begin[blockIdx.x + 1];

    if (threadIdx.x == 0) {
        for (int s = 0; s < KB_RA; s++) {
            tc::mbar_init(&fullA[s], 1);
            tc::mbar_init(&emptyA[s], KB_ISSUERS);
        }
        for (int s = 0; s < KB_RB; s++) {
            tc::mbar_init(&fullB[s], 1);
            tc::mbar_init(&emptyB[s], KB_ISSUERS);
        }
        tc::mbar_init(acc_full, KB_ISSUERS);
        tc::mbar_init(acc_empty, 256);
        for (int e = 0; e < KB_ISSUERS; e++) tc::mbar_init(drain + e, 1);
        abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, 512);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = tmem_slot;

    if (warp < 4) {
      tc::reg_dealloc<KB_REG_LO>();
      if (warp == 0) {
        // ---------------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t na = 0, nb = 0;  // planes loaded into each ring
            uint32_t issuedA = 0, phaseA = 0, issuedB = 0, phaseB = 0;  // per slot: copy issued / its phase
            bool ok = hold_copies == 0;  // a test switch holds back every copy (a wait then runs out)
            auto loadA = [&](const BlkCtx &c, int ia, int kb) {
                const uint32_t s = na % KB_RA, ph = (na / KB_RA) & 1u;
                if (!tc::mbar_wait(&emptyA[s], ph ^ 1u, &abort_flag, p.err, 1, wait_ns)) return false;
                tc::mbar_arrive_expect_tx(&fullA[s], KB_TILE);
                tc::bulk_load(ringA + s * KB_TILE, c.da + ((size_t)(ia * c.tiles_m + c.tm) * c.nkb + kb) * KB_TILE,
                              KB_TILE, &fullA[s]);
                issuedA |= 1u << s;
                phaseA = (phaseA & ~(1u << s)) | (ph << s);
                na++;
                return true;
            };
            auto loadB = [&](const BlkCtx &c, int ib, int kb) {
                const uint32_t s = nb % KB_RB, ph = (nb / KB_RB) & 1u;
                if (!tc::mbar_wait(&emptyB[s], ph ^ 1u, &abort_flag, p.err, 1, wait_ns)) return false;
                tc::mbar_arrive_expect_tx(&fullB[s], KB_TILE);
                tc::bulk_load(ringB + s * KB_TILE, c.db + ((size_t)(ib * c.tiles_n + c.tn) * c.nkb + kb) * KB_TILE,
                              KB_TILE, &fullB[s]);
                issuedB |= 1u << s;
                phaseB = (phaseB & ~(1u << s)) | (ph << s);
                nb++;
                return true;
            };
            for (int tile = t_begin; tile < t_end && ok; tile++) {
                const BlkCtx c = blk_ctx(p, tile);
                for (int st = 0; st < c.n_steps && ok; st++) {
                    const BlkStep sp = c.steps[st];
                    const int ia_lo = sp.L0 - (c.nB - 1) > 0 ? sp.L0 - (c.nB - 1) : 0;
                    const int ia_hi = sp.L1 < c.nA - 1 ? sp.L1 : c.nA - 1;
                    for (int kb = sp.kb0; kb < sp.kb1 && ok; kb++) {
                        // the first plane's window, largest ib first (the order B planes retire)
                        const int whi0 = blk_whi(sp.L1, ia_lo, c.nB), wlo0 = blk_wlo(sp.L0, ia_lo);
                        for (int ib = whi0; ib >= wlo0 && ok; ib--) ok = loadB(c, ib, kb);
                        for (int ia = ia_lo; ia <= ia_hi && ok; ia++) {
                            if (ia > ia_lo && blk_wlo(sp.L0, ia) < blk_wlo(sp.L0, ia - 1))
                                ok = loadB(c, blk_wlo(sp.L0, ia), kb);
                            if (ok) ok = loadA(c, ia, kb);
                        }
                    }
                }
            }
            if (!ok) {
                tc::drain_copies(fullA, KB_RA, issuedA, phaseA);
                tc::drain_copies(fullB, KB_RB, issuedB, phaseB);
            }
        }
      } else if (warp == 1 || warp == 2) {
        // ---------------------------------------------------------------- MMA issuers
        // Two threads issue, each the pairs of alternate levels of a block
        // (its own accumulators), so one thread's waits and commits between A
        // planes overlap the other's queued MMAs.  Both wait for every plane,
        // and every release and accumulator barrier counts both.
        if (lane == 0) {
            const int issuer = warp - 1;
            const uint32_t idesc = tc::idesc_i8(KB_BM, KB_BN);
            uint32_t na = 0, nb = 0, nbw = 0;  // A planes consumed, B planes retired, B planes waited for
            uint32_t step_no = 0;
            bool ok = true, issued = false;
            for (int tile = t_begin; tile < t_end && ok; tile++) {
                const BlkCtx c = blk_ctx(p, tile);
                for (int st = 0; st < c.n_steps && ok; st++, step_no++) {
                    const BlkStep sp = c.steps[st];
                    // the epilogue has read the accumulators of the previous step
                    if (step_no > 0 && !tc::mbar_wait(acc_empty, (step_no - 1) & 1u, &abort_flag, p.err, 2, wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const int ia_lo = sp.L0 - (c.nB - 1) > 0 ? sp.L0 - (c.nB - 1) : 0;
                    const int ia_hi = sp.L1 < c.nA - 1 ? sp.L1 : c.nA - 1;
                    uint32_t written = 0;  // accumulators written in this step
                    for (int kb = sp.kb0; kb < sp.kb1 && ok; kb++) {
                        const int whi0 = blk_whi(sp.L1, ia_lo, c.nB);
                        // the last K step stops at the 32-wide MMA that reaches k (the
                        // digits beyond k are zeros)
                        const int nkk = kb == c.nkb - 1 ? c.kq_last : KB_BK / 32;
                        const uint32_t b0 = nb;  // ring index of this K step's first B plane (= ib whi0)
                        for (int ia = ia_lo; ia <= ia_hi && ok; ia++) {
                            const int wlo = blk_wlo(sp.L0, ia), whi = blk_whi(sp.L1, ia, c.nB);
                            // wait for A_ia and the B planes down to ib = wlo
                            const uint32_t sa = na % KB_RA;
                            if (!tc::mbar_wait(&fullA[sa], (na / KB_RA) & 1u, &abort_flag, p.err, 2, wait_ns)) {
                                ok = false;
                                break;
                            }
                            const uint32_t need = b0 + (uint32_t)(whi0 - wlo) + 1u;
                            while (nbw < need && ok) {
                                if (!tc::mbar_wait(&fullB[nbw % KB_RB], (nbw / KB_RB) & 1u, &abort_flag, p.err, 2,
                                                   wait_ns))
                                    ok = false;
                                else
                                    nbw++;
                            }
                            if (!ok) break;
                            tc::fence_after_sync();
                            const uint64_t adesc = tc::smem_desc_k_sw128(tc::smem_u32(ringA + sa * KB_TILE));
                            for (int ib = wlo; ib <= whi; ib++) {
                                if (((ia + ib - sp.L0) & 1) != issuer) continue;  // the other issuer's level
                                const uint32_t sb = (b0 + (uint32_t)(whi0 - ib)) % KB_RB;
                                const uint64_t bdesc = tc::smem_desc_k_sw128(tc::smem_u32(ringB + sb * KB_TILE));
                                const int slot = ia + ib - sp.L0;
                                const uint32_t tmem_d = tmem_base + (uint32_t)slot * KB_BN;
                                uint32_t accumulate = (written >> slot) & 1u;
                                if (nkk == KB_BK / 32) {
#pragma unroll
                                    for (int kk = 0; kk < KB_BK / 32; kk++) {
                                        tc::mma_i8(tmem_d, adesc + 2 * kk, bdesc + 2 * kk, idesc, accumulate);
                                        accumulate = 1;
                                    }
                                } else {
                                    for (int kk = 0; kk < nkk; kk++) {
                                        tc::mma_i8(tmem_d, adesc + 2 * kk, bdesc + 2 * kk, idesc, accumulate);
                                        accumulate = 1;
                                    }
                                }
                                written |= 1u << slot;
                                issued = true;
                            }
                            // A_ia is done; B_whi retires when the next ia no longer reaches it
                            tc::mma_commit(&emptyA[sa]);
                            na++;
                            const int nwhi = ia < ia_hi ? blk_whi(sp.L1, ia + 1, c.nB) : -1;
                            const int nwlo = ia < ia_hi ? blk_wlo(sp.L0, ia + 1) : 0x7fffffff;
                            // retire (FIFO: largest ib first) every B plane above the next window
                            for (int ib = whi; ib >= wlo && ib > nwhi; ib--) {
                                (void)nwlo;
                                tc::mma_commit(&emptyB[nb % KB_RB]);
                                nb++;
                            }
                        }
                    }
                    if (!ok) break;
                    tc::mma_commit(acc_full);  // this step's accumulators are complete
                }
            }
            if (!ok && issued) {  // drain MMAs still in flight before tensor memory is released
                tc::mma_commit(drain + issuer);
                const uint64_t t0 = tc::globaltimer();
                while (!tc::mbar_try_wait(drain + issuer, 0) && tc::globaltimer() - t0 < 100000000ull) {
                }
            }
        }
      }
    } else {
        tc::reg_alloc<KB_REG_HI>();
        // ---------------------------------------------------------------- epilogue
        const int q = warp & 3, half = (warp - 4) >> 2;
        const int row = q * 32 + lane;
        const uint32_t lane_base = tmem_base + ((uint32_t)(q * 32) << 16);
        double *R = p.rbuf + (size_t)blockIdx.x * (KB_BM * KB_BN);  // [col][row]
        uint32_t step_no = 0;
        bool ok = true;
        for (int tile = t_begin; tile < t_end && ok; tile++) {
            const BlkCtx ct = blk_ctx(p, tile);
            const int gr = ct.tm * KB_BM + row;
            double acc[64];  // exact integer-valued run of levels (< 2^53)
#pragma unroll
            for (int c = 0; c < 64; c++) acc[c] = 0.0;
            for (int st = 0; st < ct.n_steps; st++, step_no++) {
                const BlkStep sp = ct.steps[st];
                if (!tc::mbar_wait(acc_full, step_no & 1u, &abort_flag, p.err, 3, wait_ns)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                // one or two segments: levels L0..mid, ending a run flushed here, when
                // the block crosses a run boundary; then the levels up to L1
                int L = sp.L0;
#pragma unroll 1
                for (int seg = sp.mid < sp.L1 ? 0 : 1; seg < 2; seg++) {
                    const int hi = seg == 0 ? sp.mid : sp.L1;
                    const int run_hi = seg == 0 ? sp.mid : sp.run_hi;
                    for (; L <= hi; L++) {
                        const double sc = pow2(7 * (run_hi - L));
                        const uint32_t taddr = lane_base + (uint32_t)(L - sp.L0) * KB_BN + half * 64;
                        uint32_t v[32];
                        tc::tmem_ld_32x32b_x32(taddr, v);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int c = 0; c < 32; c++) acc[c] += (double)(int32_t)v[c] * sc;
                        tc::tmem_ld_32x32b_x32(taddr + 32, v);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int c = 0; c < 32; c++) acc[32 + c] += (double)(int32_t)v[c] * sc;
                    }
                    if (seg == 1) {
                        tc::fence_before_sync();
                        tc::mbar_arrive(acc_empty);
                    }
                    if (seg == 0 || (sp.flags & 1)) {  // end of a run: R += acc * 2^fexp, the exact error carried on
                        const double fs = pow2(seg == 0 ? sp.fexp_mid : sp.fexp);
                        const bool first = seg == 0 ? sp.first_mid != 0 : (sp.flags & 2) != 0;
                        const bool last = seg == 1 && (sp.flags & 4);
                        const double cs = last ? 0.0 : pow2(seg == 0 ? sp.cexp_mid : sp.cexp);
#pragma unroll
                        for (int c = 0; c < 64; c++) {
                            double *rp = &R[(size_t)(half * 64 + c) * KB_BM + row];
                            if (first) {
                                *rp = acc[c] * fs;
                                acc[c] = 0.0;
                            } else {
                                const double ro = *rp;
                                const double a = acc[c] * fs;
                                const double sm = ro + a;
                                const double bb = sm - ro;
                                acc[c] = ((ro - (sm - bb)) + (a - bb)) * cs;  // TwoSum error, in the next run's units
                                *rp = sm;
                            }
                        }
                    }
                }
            }
            if (ok) {
                // the tile's R, complete, scaled into C in a pass of its own: the
                // problem's output fields are read here, not held in registers
                // across the steps; 8 columns' loads in flight at a time
                const BlkOut o = blk_out(p, tile);
                const int c0 = o.tn * KB_BN + half * 64;
                const int ncol = o.n - c0;
                if (gr < o.m && ncol > 0) {
                    const int ea = o.ea[gr];
                    double *cb = o.C + (size_t)c0 * o.ldc + gr;
                    const int *eb = o.eb + c0;
                    const double *rb = R + (size_t)(half * 64) * KB_BM + row;
                    for (int cc = 0; cc < 64; cc += 8) {
                        double rv[8], cv[8];
                        int ev[8];
#pragma unroll
                        for (int j = 0; j < 8; j++)
                            if (cc + j < ncol) {
                                rv[j] = rb[(size_t)(cc + j) * KB_BM];
                                ev[j] = eb[cc + j];
                                cv[j] = cb[(size_t)(cc + j) * o.ldc];
                            }
#pragma unroll
                        for (int j = 0; j < 8; j++)
                            if (cc + j < ncol)
                                cb[(size_t)(cc + j) * o.ldc] = fma(o.alpha, scalbn(rv[j], ea + ev[j]), o.beta * cv[j]);
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, 512);
    }
}

static std::atomic<uint64_t> g_blk_grouped_attr{0};

uint64_t i8_test_wait_ns();  // gemm_i8.cu: the wait limit and copy switch of cuozblasSetI8WaitTest
int i8_test_hold_copies();

cudaError_t i8_blk_grouped_kernel(int grid, const BlkProb *probs, const BlkStep *steps, const int4 *tiles,
                                  const int *cta_begin, double *rbuf, int *err, cudaStream_t stream) {
    cudaError_t e = smem_optin((const void *)k_i8_blk_grouped, KB_SMEM, g_blk_grouped_attr);
    if (e != cudaSuccess) return e;
    BlkGParams p;
    p.probs = probs;
    p.steps = steps;
    p.tiles = tiles;
    p.cta_begin = cta_begin;
    p.rbuf = rbuf;
    p.err = err;
    k_i8_blk_grouped<<<grid, KB_THREADS, KB_SMEM, stream>>>(p, i8_test_wait_ns(), i8_test_hold_copies());
    return cudaGetLastError();
}

}  // namespace ozb
