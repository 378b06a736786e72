// gemm_i8_blk.cu — the INT8 precision form's product kernel, level-blocked.
//
// Same arithmetic as k_i8_gemm (gemm_i8.cu): C(i,j) = 2^(EA_i + EB_j)
// sum_L 2^(-7(L+2)) V_L with V_L the INT32 sums of the digit-pair products of
// level L, runs of consecutive levels combined exactly in FP64, runs flushed
// into the FP64 sum R largest first with the TwoSum error carried into the next
// run, so the results are bit-identical.  What changes is the order of the
// products.  k_i8_gemm streams every pair's A and B panels through shared
// memory for every level; a level-L pair shares no digit plane with the other
// pairs of its level, so a 128 x 128 tile moves 2 x 16 KB per 4 MMAs, about
// 128 bytes per clock per SM from L2 at full tensor rate, which L2 cannot
// deliver.  Here up to four consecutive levels ("a block") are accumulated at
// once, each in its own INT32 tensor-memory accumulator (4 x 128 columns):
// within a 128-wide K step, the A plane ia serves the pairs (ia, ib) of every
// level of the block, and the B planes of those pairs slide by one plane per
// ia.  So per ia one A plane and at most one new B plane are loaded for up to
// four pairs (16 MMAs): a quarter of the operand traffic.
//
// Roles (one CTA per SM, persistent): warp 0 lane 0 loads planes by TMA into
// two rings (A: 4 slots, B: 8 slots of 16 KB, 128-byte swizzle); warp 1 holds
// the tensor memory, and lane 0 of warps 1 and 2 issue tcgen05.mma.kind::i8
// (alternate levels each); warps 4-11 read the
// accumulators after each (block, K chunk), combine the block's levels into
// the run accumulator in registers, and at a run's end add the run into R,
// which lives in a per-CTA buffer in global memory (128 KB, L2-resident).
// Every mbarrier wait is bounded as in k_i8_gemm.
#include <cuda.h>

#include <vector>

#include "gemm_i8_blk.h"
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "tc05.cuh"

namespace ozb {

struct BlkParams {
    int m, n, m_pad, n_pad, ldc;
    int tiles_m, tiles_n, strip;
    int nA, nB, n_steps;
    const BlkStep *steps;
    const int *ea, *eb;
    double alpha, beta;
    double *C;
    double *rbuf;  // per CTA: 128 x 128 doubles, [col][row]
    int *err;
};

__device__ __forceinline__ void blk_tile_coords(int tile, const BlkParams &p, int &tm, int &tn) {
    const int per_strip = p.strip * p.tiles_n;
    const int s = tile / per_strip, w = tile - s * per_strip;
    const int rows = min(p.strip, p.tiles_m - s * p.strip);
    tm = s * p.strip + w % rows;
    tn = w / rows;
}


// CROSS: the schedule has blocks that end one run and begin the next (the
// epilogue flushes a run in the middle of a block); without them the epilogue
// carries no code for it.
template <bool CROSS>
__global__ void __launch_bounds__(KB_THREADS, 1)
    k_i8_blk(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
             const __grid_constant__ BlkParams p, uint64_t wait_ns, int hold_copies) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *ringA = smem, *ringB = smem + KB_RA * KB_TILE;
    uint64_t *bar = (uint64_t *)(smem + (KB_RA + KB_RB) * KB_TILE);
    uint64_t *fullA = bar, *emptyA = bar + KB_RA, *fullB = bar + 2 * KB_RA, *emptyB = bar + 2 * KB_RA + KB_RB;
    uint64_t *acc_full = bar + 2 * KB_RA + 2 * KB_RB, *acc_empty = acc_full + 1, *drain = acc_full + 2;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = p.tiles_m * p.tiles_n;

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
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
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
            auto loadA = [&](int ia, int kb, int tm) {
                const uint32_t s = na % KB_RA, ph = (na / KB_RA) & 1u;
                if (!tc::mbar_wait(&emptyA[s], ph ^ 1u, &abort_flag, p.err, 1, wait_ns)) return false;
                tc::mbar_arrive_expect_tx(&fullA[s], KB_TILE);
                tc::tma_load_2d(ringA + s * KB_TILE, &tmA, &fullA[s], kb * KB_BK, ia * p.m_pad + tm * KB_BM);
                issuedA |= 1u << s;
                phaseA = (phaseA & ~(1u << s)) | (ph << s);
                na++;
                return true;
            };
            auto loadB = [&](int ib, int kb, int tn) {
                const uint32_t s = nb % KB_RB, ph = (nb / KB_RB) & 1u;
                if (!tc::mbar_wait(&emptyB[s], ph ^ 1u, &abort_flag, p.err, 1, wait_ns)) return false;
                tc::mbar_arrive_expect_tx(&fullB[s], KB_TILE);
                tc::tma_load_2d(ringB + s * KB_TILE, &tmB, &fullB[s], kb * KB_BK, ib * p.n_pad + tn * KB_BN);
                issuedB |= 1u << s;
                phaseB = (phaseB & ~(1u << s)) | (ph << s);
                nb++;
                return true;
            };
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int tm, tn;
                blk_tile_coords(tile, p, tm, tn);
                for (int st = 0; st < p.n_steps && ok; st++) {
                    const BlkStep sp = p.steps[st];
                    const int ia_lo = sp.L0 - (p.nB - 1) > 0 ? sp.L0 - (p.nB - 1) : 0;
                    const int ia_hi = sp.L1 < p.nA - 1 ? sp.L1 : p.nA - 1;
                    for (int kb = sp.kb0; kb < sp.kb1 && ok; kb++) {
                        // the first plane's window, largest ib first (the order B planes retire)
                        const int whi0 = blk_whi(sp.L1, ia_lo, p.nB), wlo0 = blk_wlo(sp.L0, ia_lo);
                        for (int ib = whi0; ib >= wlo0 && ok; ib--) ok = loadB(ib, kb, tn);
                        for (int ia = ia_lo; ia <= ia_hi && ok; ia++) {
                            if (ia > ia_lo && blk_wlo(sp.L0, ia) < blk_wlo(sp.L0, ia - 1))
                                ok = loadB(blk_wlo(sp.L0, ia), kb, tn);
                            if (ok) ok = loadA(ia, kb, tm);
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
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                for (int st = 0; st < p.n_steps && ok; st++, step_no++) {
                    const BlkStep sp = p.steps[st];
                    // the epilogue has read the accumulators of the previous step
                    if (step_no > 0 && !tc::mbar_wait(acc_empty, (step_no - 1) & 1u, &abort_flag, p.err, 2, wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const int ia_lo = sp.L0 - (p.nB - 1) > 0 ? sp.L0 - (p.nB - 1) : 0;
                    const int ia_hi = sp.L1 < p.nA - 1 ? sp.L1 : p.nA - 1;
                    uint32_t written = 0;  // accumulators written in this step
                    for (int kb = sp.kb0; kb < sp.kb1 && ok; kb++) {
                        const int whi0 = blk_whi(sp.L1, ia_lo, p.nB);
                        const uint32_t b0 = nb;  // ring index of this K step's first B plane (= ib whi0)
                        for (int ia = ia_lo; ia <= ia_hi && ok; ia++) {
                            const int wlo = blk_wlo(sp.L0, ia), whi = blk_whi(sp.L1, ia, p.nB);
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
#pragma unroll
                                for (int kk = 0; kk < KB_BK / 32; kk++) {
                                    tc::mma_i8(tmem_d, adesc + 2 * kk, bdesc + 2 * kk, idesc, accumulate);
                                    accumulate = 1;
                                }
                                written |= 1u << slot;
                                issued = true;
                            }
                            // A_ia is done; B_whi retires when the next ia no longer reaches it
                            tc::mma_commit(&emptyA[sa]);
                            na++;
                            const int nwhi = ia < ia_hi ? blk_whi(sp.L1, ia + 1, p.nB) : -1;
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
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            int tm, tn;
            blk_tile_coords(tile, p, tm, tn);
            const int gr = tm * KB_BM + row;
            double acc[64];  // exact integer-valued run of levels (< 2^53)
#pragma unroll
            for (int c = 0; c < 64; c++) acc[c] = 0.0;
            for (int st = 0; st < p.n_steps; st++, step_no++) {
                const BlkStep sp = p.steps[st];
                if (!tc::mbar_wait(acc_full, step_no & 1u, &abort_flag, p.err, 3, wait_ns)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                if (CROSS && sp.mid < sp.L1) {  // the block ends a run at mid: add its levels and flush it first
                    for (int L = sp.L0; L <= sp.mid; L++) {
                        const double sc = pow2(7 * (sp.mid - L));
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
                    const double fs = pow2(sp.fexp_mid), cs = pow2(sp.cexp_mid);
                    const bool first = sp.first_mid != 0;
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
                for (int L = (CROSS && sp.mid < sp.L1) ? sp.mid + 1 : sp.L0; L <= sp.L1; L++) {
                    const double sc = pow2(7 * (sp.run_hi - L));
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
                tc::fence_before_sync();
                tc::mbar_arrive(acc_empty);
                if (sp.flags & 1) {  // end of a run: R += acc * 2^fexp, the exact error carried on
                    const double fs = pow2(sp.fexp);
                    const bool first = sp.flags & 2, last = sp.flags & 4;
                    const double cs = last ? 0.0 : pow2(sp.cexp);
                    const int ea = (last && gr < p.m) ? p.ea[gr] : 0;
#pragma unroll
                    for (int c = 0; c < 64; c++) {
                        const int col = half * 64 + c;
                        double *rp = &R[(size_t)col * KB_BM + row];
                        double r;
                        if (first) {
                            r = acc[c] * fs;
                            acc[c] = 0.0;
                        } else {
                            const double ro = *rp;
                            const double a = acc[c] * fs;
                            const double sm = ro + a;
                            const double bb = sm - ro;
                            acc[c] = ((ro - (sm - bb)) + (a - bb)) * cs;  // TwoSum error, in the next run's units
                            r = sm;
                        }
                        if (last) {
                            const int gc = tn * KB_BN + col;
                            if (gr < p.m && gc < p.n) {
                                double *cp = &p.C[(size_t)gc * p.ldc + gr];
                                const double t = scalbn(r, ea + p.eb[gc]);
                                *cp = fma(p.alpha, t, p.beta * *cp);
                            }
                        } else {
                            *rp = r;
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
        tc::tmem_dealloc(tmem_base, 512);
    }
}

// The per-tile schedule: runs of consecutive levels whose exact combination
// stays below 2^53 (the same runs as i8_schedule), cut into blocks of at most
// W <= KB_W levels, each block cut into K chunks that keep every accumulator's
// INT32 sum exact.  Returns false when the levels exceed the tables' range.
// The order of the products and flushes does not depend on the cut: each
// accumulator and each run's sum is an exact integer, and the runs are flushed
// in the same order with the same values, so every cut gives the same bits.
bool blk_schedule(int nA, int nB, int nkb, bool triangular, int W, std::vector<BlkStep> &steps, bool across) {
    if (W < 1 || W > KB_W) return false;
    const int maxlevel = triangular ? (nA < nB ? nA : nB) - 1 : nA + nB - 2;
    if (maxlevel < 0 || maxlevel >= 128) return false;
    auto pairs = [&](int L) {
        const int lo = L - (nB - 1) > 0 ? L - (nB - 1) : 0, hi = L < nA - 1 ? L : nA - 1;
        return hi - lo + 1;
    };
    // the runs (bounds as i8_schedule: pairs x K x 127^2 per level)
    std::vector<unsigned __int128> lbound(maxlevel + 1);
    for (int L = 0; L <= maxlevel; L++)
        lbound[L] = (unsigned __int128)pairs(L) * (unsigned __int128)nkb * KB_BK * 127 * 127;
    const unsigned __int128 lim = (unsigned __int128)1 << 53;
    std::vector<int> run_lo, run_hi, run_of(maxlevel + 1);
    for (int L0 = 0; L0 <= maxlevel;) {
        unsigned __int128 b = lbound[L0];
        int L1 = L0;
        while (L1 + 1 <= maxlevel && (b << 7) + lbound[L1 + 1] < lim) {
            b = (b << 7) + lbound[L1 + 1];
            L1++;
        }
        for (int L = L0; L <= L1; L++) run_of[L] = (int)run_lo.size();
        run_lo.push_back(L0);
        run_hi.push_back(L1);
        L0 = L1 + 1;
    }
    const int nruns = (int)run_lo.size();
    // the blocks: within the runs, or equal cuts of all levels
    std::vector<std::pair<int, int>> blocks;
    if (across) {
        const int n = maxlevel + 1, nb = (n + W - 1) / W, base = n / nb, extra = n % nb;
        for (int i = 0, L0 = 0; i < nb; i++) {
            const int size = base + (i >= nb - extra ? 1 : 0);
            blocks.push_back({L0, L0 + size - 1});
            L0 += size;
        }
    } else {
        for (int r = 0; r < nruns; r++)
            for (int L0 = run_lo[r]; L0 <= run_hi[r]; L0 += W)
                blocks.push_back({L0, L0 + W - 1 < run_hi[r] ? L0 + W - 1 : run_hi[r]});
    }
    steps.clear();
    for (const auto &bl : blocks) {
        const int L0 = bl.first, L1 = bl.second;
        const int ra = run_of[L0], rb = run_of[L1];
        if (rb > ra + 1) return false;  // at most one run boundary inside a block
        int pmax = 0;
        for (int L = L0; L <= L1; L++) pmax = pairs(L) > pmax ? pairs(L) : pmax;
        int chunk = (int)(KB_MAX_TERMS / ((int64_t)pmax * KB_BK));  // K steps per INT32 sum
        if (chunk < 1) return false;
        if (rb != ra && chunk < nkb) return false;  // a crossing block is one K chunk
        const int next_hi = rb + 1 < nruns ? run_hi[rb + 1] : 0;
        for (int kb0 = 0; kb0 < nkb; kb0 += chunk) {
            BlkStep s;
            s.L0 = L0;
            s.L1 = L1;
            s.kb0 = kb0;
            s.kb1 = kb0 + chunk < nkb ? kb0 + chunk : nkb;
            s.run_hi = run_hi[rb];
            s.flags = 0;
            if (L1 == run_hi[rb] && s.kb1 == nkb) s.flags |= 1;
            s.fexp = -7 * (run_hi[rb] + 2);
            s.cexp = 7 * (next_hi + 2);
            s.mid = rb != ra ? run_hi[ra] : L1;
            s.fexp_mid = -7 * (run_hi[ra] + 2);
            s.cexp_mid = 7 * (run_hi[rb] + 2);
            s.first_mid = 0;
            steps.push_back(s);
        }
    }
    // the first flush of a tile writes R, the last one writes C
    for (auto &s : steps) {
        if (s.mid < s.L1) {
            s.first_mid = 1;
            break;
        }
        if (s.flags & 1) {
            s.flags |= 2;
            break;
        }
    }
    steps.back().flags |= 4;
    return (steps.back().flags & 1) != 0;
}

static std::atomic<uint64_t> g_blk_attr{0}, g_blk_attr_cross{0};

int blk_kq_last(int k, int nkb) {
    const int tail = k - (nkb - 1) * KB_BK;
    const int q = (tail + 31) / 32;
    return q < 1 ? 1 : (q > KB_BK / 32 ? KB_BK / 32 : q);
}

uint64_t i8_test_wait_ns();  // gemm_i8.cu: the wait limit and copy switch of cuozblasSetI8WaitTest
int i8_test_hold_copies();

// The level-blocked product kernel over digit operands laid out as for
// k_i8_gemm (tensor maps over [S * lines_pad][k_pad], 128 x 128-byte boxes).
// `width`: levels per block (1..4, within the runs; -4..-1: equal cuts of at
// most -width levels across the runs, or blocks of -width levels within the
// runs where the cut does not apply; every width gives the same bits).
// Returns NOT_SUPPORTED (nothing launched) when the schedule does not apply.
int i8_blk_launch(cuozblasHandle_t *h, const CUtensorMap &tmA, const CUtensorMap &tmB, int m, int n, int m_pad,
                  int n_pad, int k_pad, int nA, int nB, bool triangular, const int *ea, const int *eb, double alpha,
                  double beta, double *C, int ldc, int strip, int width, int *d_err, Arena &ar) {
    State *st = state(h);
    std::vector<BlkStep> steps;
    const int w = width < 0 ? -width : width;
    // a cut across the runs that does not apply (a crossing block would need
    // several K chunks) falls back to blocks within the runs
    if (!blk_schedule(nA, nB, k_pad / KB_BK, triangular, w, steps, width < 0) &&
        !(width < 0 && blk_schedule(nA, nB, k_pad / KB_BK, triangular, w, steps, false)))
        return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const int nsm = sm_count();
    const int tiles_m = m_pad / KB_BM, tiles_n = n_pad / KB_BN, ntiles = tiles_m * tiles_n;
    const int grid = ntiles < nsm ? ntiles : nsm;
    BlkStep *d_steps = ar.take<BlkStep>(steps.size());
    double *rbuf = ar.take<double>((uint64_t)grid * KB_BM * KB_BN);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemcpyAsync(d_steps, steps.data(), sizeof(BlkStep) * steps.size(), cudaMemcpyHostToDevice,
                              st->stream));
    BlkParams p;
    p.m = m;
    p.n = n;
    p.m_pad = m_pad;
    p.n_pad = n_pad;
    p.ldc = ldc;
    p.tiles_m = tiles_m;
    p.tiles_n = tiles_n;
    p.strip = strip < tiles_m ? strip : tiles_m;
    p.nA = nA;
    p.nB = nB;
    p.n_steps = (int)steps.size();
    p.steps = d_steps;
    p.ea = ea;
    p.eb = eb;
    p.alpha = alpha;
    p.beta = beta;
    p.C = C;
    p.rbuf = rbuf;
    p.err = d_err;
    bool cross = false;
    for (const BlkStep &sp : steps) cross = cross || sp.mid < sp.L1;
    OZB_CHECK(smem_optin(cross ? (const void *)k_i8_blk<true> : (const void *)k_i8_blk<false>, KB_SMEM,
                         cross ? g_blk_attr_cross : g_blk_attr));
    counted(h);
    if (cross)
        k_i8_blk<true><<<grid, KB_THREADS, KB_SMEM, st->stream>>>(tmA, tmB, p, i8_test_wait_ns(),
                                                                   i8_test_hold_copies());
    else
        k_i8_blk<false><<<grid, KB_THREADS, KB_SMEM, st->stream>>>(tmA, tmB, p, i8_test_wait_ns(),
                                                                    i8_test_hold_copies());
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb

extern "C" int cuozblasRuleI8Schedule(int32_t nA, int32_t nB, int32_t nkb, int32_t triangular, int32_t width,
                                      int32_t *out, int32_t max_steps) {
    if (width == 0 || width < -ozb::KB_W || width > ozb::KB_W || nA < 1 || nB < 1 || nkb < 1 || !out) return -1;
    std::vector<ozb::BlkStep> steps;
    if (!ozb::blk_schedule(nA, nB, nkb, triangular != 0, width < 0 ? -width : width, steps, width < 0)) return -1;
    if ((int64_t)steps.size() > max_steps) return -2;
    for (size_t i = 0; i < steps.size(); i++) {
        const ozb::BlkStep &s = steps[i];
        const int32_t v[12] = {s.L0, s.L1, s.kb0, s.kb1, s.run_hi, s.flags, s.fexp, s.cexp,
                               s.mid, s.fexp_mid, s.cexp_mid, s.first_mid};
        for (int j = 0; j < 12; j++) out[12 * i + j] = v[j];
    }
    return (int)steps.size();
}
