// gemm_i8_blk.h — the level-blocked INT8 product kernels' schedule, launch
// shape and helpers, shared by the single kernel (gemm_i8_blk.cu), the grouped
// kernel (gemm_i8_blk_grouped.cu) and the grouped call (gemm_i8_grouped.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace ozb {

// One (block of levels, K chunk) of the per-tile schedule.  A block may end
// one run and begin the next (then it is the block's only K chunk): its levels
// L0..mid belong to the run ending at mid, flushed before the levels above it
// are read; mid = L1 when the block lies within one run.
struct BlkStep {
    int L0, L1;         // the block's levels
    int kb0, kb1;       // K chunk, in 128-wide steps
    int run_hi;         // last level of the run of levels mid+1..L1 (or of the whole block): shift 7 (run_hi - L)
    int flags;          // 1: flush the run after this step, 2: first flush of the tile, 4: last step
    int fexp, cexp;     // flush exponent -7 (run_hi + 2), the next run's carry exponent 7 (next_hi + 2)
    int mid;            // last level of the first run when the block crosses a run boundary, else L1
    int fexp_mid, cexp_mid;  // that run's flush exponent -7 (mid + 2) and carry exponent 7 (run_hi + 2)
    int first_mid;      // 1: the flush at mid is the tile's first flush
};

// One problem of a grouped level-blocked launch.  Digit plane s of op(A) is
// tiles_m x nkb tiles of 16 KB (128 lines x 128 k, 128-byte swizzle applied),
// tile (tm, kb) at da + ((s * tiles_m + tm) * nkb + kb) * 16384; B likewise.
struct BlkProb {
    int m, n, ldc, nkb, tiles_m, tiles_n;
    int kq_last;            // 32-wide MMAs of the last K step that reach k (blk_kq_last)
    int nA, nB;             // digit counts
    int step0, n_steps;     // the problem's schedule within the launch's step list
    const int8_t *da, *db;
    const int *ea, *eb;     // line exponents
    double alpha, beta;
    double *C;
};

constexpr int kBlkMaxWidth = 4;  // most levels per block (tensor-memory accumulators)

// Launch shape shared by the single and grouped kernels.
constexpr int KB_BM = 128, KB_BN = 128, KB_BK = 128;
constexpr int KB_W = kBlkMaxWidth;
constexpr int KB_RA = 4, KB_RB = 8;           // ring slots for A and B planes
constexpr int KB_TILE = KB_BM * KB_BK;        // 16 KB plane tile
constexpr int KB_ISSUERS = 2;  // MMA issuing threads (warps 1 and 2), each owning alternate levels of a block
                                // (three measured slower: 4.21 vs 4.00 ms at 4096^3)
constexpr int KB_THREADS = 384;  // warp 0 producer, warps 1-2 MMA issuers, warp 3 idle, warps 4-11 epilogue
// Registers per thread: 168 at launch (65536 / 384, rounded down to 8); the
// producer warpgroup drops to KB_REG_LO and the two epilogue warpgroups rise to
// KB_REG_HI: 4 x 56 + 8 x 224 = 12 x 168, and per SM sub-partition (one warp of
// each warpgroup) 56 + 2 x 224 <= 512.
constexpr uint32_t KB_REG_LO = 56, KB_REG_HI = 224;
constexpr int KB_SMEM = (KB_RA + KB_RB) * KB_TILE + 1024 /*align*/ + 512 /*barriers*/;
constexpr int64_t KB_MAX_TERMS = 2147483647LL / (127 * 127);

#ifdef __CUDACC__
// The B planes of A plane ia within a block of levels [L0, L1]: ib in [wlo, whi].
__device__ __forceinline__ int blk_wlo(int L0, int ia) { return L0 - ia > 0 ? L0 - ia : 0; }
__device__ __forceinline__ int blk_whi(int L1, int ia, int nB) { return L1 - ia < nB - 1 ? L1 - ia : nB - 1; }
#endif

// 32-wide MMAs of the last of nkb 128-wide K steps that reach k (1-4; the
// digits beyond k are zeros, so the MMAs past it add nothing).
int blk_kq_last(int k, int nkb);

// Runs of consecutive levels whose exact combination stays below 2^53 (the
// runs of the level-wise schedule), cut into blocks of at most W levels, each
// block cut into K chunks that keep every INT32 sum exact.  With `across`, the
// levels are cut into equal blocks of at most W levels regardless of the runs
// (the larger blocks at the top), each crossing at most one run boundary and
// then only when it needs a single K chunk; false where that does not hold.
// False also when the levels exceed the kernel's range.
bool blk_schedule(int nA, int nB, int nkb, bool triangular, int W, std::vector<BlkStep> &steps,
                  bool across = false);

// The grouped level-blocked launch: CTA c runs the tiles {problem, tm, tn, 0}
// in [cta_begin[c], cta_begin[c + 1]); rbuf holds grid x 128 x 128 doubles;
// a wait that runs out writes its role's code (1-3) into *err.
cudaError_t i8_blk_grouped_kernel(int grid, const BlkProb *probs, const BlkStep *steps, const int4 *tiles,
                                  const int *cta_begin, double *rbuf, int *err, cudaStream_t stream);

}  // namespace ozb
