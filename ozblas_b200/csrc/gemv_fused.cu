// gemv_fused.cu — the plain GEMV y = alpha A x + beta y ('n') without
// materialised slices (src/cpu/ozblas_gemv.cpp:22-26 -> ozblas_gemm.cpp with
// n = 1; the reference transposes A, writes every slice of every row and
// multiplies them).
//
// Each row of A is one line of the split (its own tau chain, rho from the
// row length).  The chain needs the maximum of the remainders of a whole row
// before the next level.  The default path reads A twice: a TMA-streamed
// pass takes the row maxima, and a second one cuts every element on a
// predicted chain, multiplies the slices with the slices of x (split by the
// vector rule) and records the actual remainder maxima that prove the chain
// (rows whose prediction fails are redone on their corrected chains; see
// k_gemv_tma).  The fallback (A unsuited to a tensor map, a chain that stays
// unproven) reads A once per level: pass p reads A in its column-major order
// (lane = row, coalesced 256-byte row segments), recomputes each element's
// remainder through the p known levels with the split's own arithmetic,
// (r + sigma) - sigma, and records max |r_p| per row; the pass that finds
// every remainder zero fixes the slice count by the reference's termination
// rule, and one more pass forms the products.  The partial products are sums
// of exact terms below 2^53 on one grid, so they combine exactly in any order
// (shared-memory and global atomics).  The ordered sum over the pairs is
// k_sum_rows, as for the materialised path.
#include <stdlib.h>

#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "tc05.cuh"

namespace ozb {

constexpr int kGvCols = 64;    // columns per warp per pass
constexpr int kGvWarps = 8;    // warps per block (same 32 rows, different column chunks)
constexpr int kGvMaxLevels = 8;

// Pass p: M[p * m + row] = max |r_p| over the row (r_0 = a), with
// sigma_l = 0.75 2^(rho + tau(M[l * m + row])) for l < p.  M zeroed before.
__global__ void __launch_bounds__(256) k_gemv_level(int m, int n, const double *__restrict__ A, int lda, int rho, int p,
                                                    double *__restrict__ M, double *__restrict__ gmax) {
    __shared__ double red[kGvWarps][32];
    if (p >= 2 && gmax[p - 1] == 0.0) return;  // uniform: an earlier pass left every remainder zero
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = blockIdx.x * 32 + lane;
    const int col0 = (blockIdx.y * kGvWarps + warp) * kGvCols;
    double sig[kGvMaxLevels];
#pragma unroll
    for (int l = 0; l < kGvMaxLevels; l++) sig[l] = (l < p && row < m) ? dense_sigma(rho, M[(size_t)l * m + row], 1) : 0.0;
    double mx = 0.0;
    if (row < m) {
        const int cend = col0 + kGvCols < n ? col0 + kGvCols : n;
#pragma unroll 8
        for (int j = col0; j < cend; j++) {
            double r = A[(size_t)j * lda + row];
#pragma unroll
            for (int l = 0; l < kGvMaxLevels; l++)
                if (l < p) r = r - ((r + sig[l]) - sig[l]);
            mx = ref_max(mx, fabs(r));
        }
    }
    red[warp][lane] = mx;  // 0 for rows past m
    __syncthreads();
    if (warp == 0) {  // all 32 lanes: the shuffles below read every lane
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kGvWarps; w++) v = ref_max(v, red[w][lane]);
        if (row < m) atomic_max_nonneg(&M[(size_t)p * m + row], v);
        double g = v;  // warp max for the termination test
        for (int o = 16; o > 0; o >>= 1) g = ref_max(g, __shfl_xor_sync(0xffffffffu, g, o));
        if (lane == 0) atomic_max_nonneg(&gmax[p], g);
    }
}

// Products: P[(ia * nB + ib) * m + row] += sum_j slice_ia(A[row, j]) * xs[ib][j]
// for ia < nA (the row's nA levels), ib < NB.  P zeroed before.
template <int NB>
__global__ void __launch_bounds__(256) k_gemv_products(int m, int n, const double *__restrict__ A, int lda, int rho,
                                                       int nA, const double *__restrict__ M,
                                                       const double *__restrict__ xs, int ldx,
                                                       double *__restrict__ P) {
    __shared__ double ps[kGvMaxLevels * NB * 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = blockIdx.x * 32 + lane;
    const int col0 = (blockIdx.y * kGvWarps + warp) * kGvCols;
    for (int i = threadIdx.x; i < kGvMaxLevels * NB * 32; i += blockDim.x) ps[i] = 0.0;
    double sig[kGvMaxLevels];
#pragma unroll
    for (int l = 0; l < kGvMaxLevels; l++) sig[l] = (l < nA && row < m) ? dense_sigma(rho, M[(size_t)l * m + row], 1) : 0.0;
    double acc[kGvMaxLevels][NB];
#pragma unroll
    for (int a = 0; a < kGvMaxLevels; a++)
#pragma unroll
        for (int b = 0; b < NB; b++) acc[a][b] = 0.0;
    if (row < m) {
        const int cend = col0 + kGvCols < n ? col0 + kGvCols : n;
#pragma unroll 4
        for (int j = col0; j < cend; j++) {
            double r = A[(size_t)j * lda + row];
            double xv[NB];
#pragma unroll
            for (int b = 0; b < NB; b++) xv[b] = xs[(size_t)b * ldx + j];
#pragma unroll
            for (int l = 0; l < kGvMaxLevels; l++) {
                if (l < nA) {
                    const double s = (r + sig[l]) - sig[l];
                    r = r - s;
#pragma unroll
                    for (int b = 0; b < NB; b++) acc[l][b] = fma(s, xv[b], acc[l][b]);  // exact
                }
            }
        }
    }
    // the 8 warps hold the same 32 rows: add their partial products in turn
    for (int w = 0; w < kGvWarps; w++) {
        __syncthreads();
        if (warp == w) {
#pragma unroll
            for (int a = 0; a < kGvMaxLevels; a++)
                if (a < nA)
#pragma unroll
                    for (int b = 0; b < NB; b++) ps[(a * NB + b) * 32 + lane] += acc[a][b];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nA * NB * 32; i += blockDim.x) {
        const int pr = i >> 5, l = i & 31;
        const int rr = blockIdx.x * 32 + l;
        if (rr < m) atomicAdd(&P[(size_t)pr * m + rr], ps[i]);
    }
}

// ---------------------------------------------------------------------------
// Two reads of A on predicted chains.  A row's chain is predicted from its
// maximum alone: tau_0 = tau(max |a|), tau_l = tau_{l-1} + rho - 54 (the
// remainder after a level is at most half its grid 2^(rho + tau - 53), and a
// long row almost always holds one within a factor 2 of that).  The products
// pass cuts every element on the row's chain T and records the actual
// max |r_l| of each level; k_gemv_chain proves the chain: if T[0..l-1] are
// right, r_l is the reference's remainder, so max |r_l| is its maximum and
// tau(max |r_l|) its tau.  A row whose chain breaks at level l gets the true
// tau_l, a new prediction beyond it, zeroed products and another products
// pass (only rows still unproven take part), so each pass fixes at least one
// more level.
//
// Both passes stream A through shared memory with TMA: a block owns 32 rows
// and a column range, tiles of 32 rows x 64 columns (16 KB, one 256-byte
// segment per column) land in a 4-stage ring, and warp w takes columns
// 8w..8w+7 of every tile (lane = row, conflict-free reads).  The ring keeps
// 64 KB per block in flight without holding loads in registers.
// ---------------------------------------------------------------------------
constexpr int kGtCols = 64;
constexpr int kGtStages = 4;
constexpr int kGtTile = 32 * kGtCols;  // doubles per tile
constexpr uint32_t kGtTileBytes = kGtTile * sizeof(double);
constexpr int kGtSmem = kGtStages * kGtTileBytes + 1024;  // + room to align the ring to 1 KB
constexpr uint64_t kGtWaitNs = 2000000000ull;  // 2 s without progress
constexpr int kGtIters = 3;                     // products passes enqueued before the one host read

// PRED = false: Ma[row] = max |a| over the row (Ma zeroed before).
// PRED = true: for the rows with state != 0, P[(l * NB + b) * m + row] += sum_j
// slice_l(a) xs[b][j] on the chain T, and Ma[(l + 1) * m + row] = max |r_{l+1}|.
// A timed-out wait sets err[0] and ends the block after its loads in flight.
template <int NB, bool PRED>
__global__ void __launch_bounds__(256) k_gemv_tma(const __grid_constant__ CUtensorMap tmA, int m, int n, int rho, int cpb,
                                                  const int *__restrict__ T, const int *__restrict__ state,
                                                  const double *__restrict__ xs, int ldx, double *__restrict__ P,
                                                  double *__restrict__ Ma, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char gt_smem[];
    double *tiles = reinterpret_cast<double *>(gt_smem + ((1024 - (tc::smem_u32(gt_smem) & 1023)) & 1023));
    __shared__ __align__(8) uint64_t full[kGtStages], empty[kGtStages];
    __shared__ double ps[PRED ? kGvMaxLevels * NB * 32 : 1];
    __shared__ double red[kGvWarps][32];
    __shared__ int abort_flag, never;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row0 = blockIdx.x * 32, row = row0 + lane;
    const bool active = row < m && (!PRED || state[row] != 0);
    if (!__syncthreads_or(active)) return;  // block-uniform: no row of this block needs the pass
    const int c0 = blockIdx.y * cpb;
    const int cend = c0 + cpb < n ? c0 + cpb : n;
    const int nt = (cend - c0 + kGtCols - 1) / kGtCols;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kGtStages; q++) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], kGvWarps);
        }
        abort_flag = 0;
        never = 0;
        tc::fence_mbar_init();
    }
    if (PRED)
        for (int i = threadIdx.x; i < kGvMaxLevels * NB * 32; i += blockDim.x) ps[i] = 0.0;
    __syncthreads();
    int issued = 0;  // thread 0: tiles whose loads were issued
    if (threadIdx.x == 0) {
        tc::prefetch_tmap(&tmA);
        for (; issued < nt && issued < kGtStages; issued++) {
            tc::mbar_arrive_expect_tx(&full[issued], kGtTileBytes);
            tc::tma_load_2d(tiles + issued * kGtTile, &tmA, &full[issued], row0, c0 + issued * kGtCols);
        }
    }
    double sig[PRED ? kGvMaxLevels : 1];
    double acc[PRED ? kGvMaxLevels : 1][NB], mxl[PRED ? kGvMaxLevels : 1];
#pragma unroll
    for (int l = 0; l < (PRED ? kGvMaxLevels : 1); l++) {
        sig[l] = (PRED && active) ? 0.75 * pow2(rho + T[(size_t)l * m + row]) : 0.0;
        mxl[l] = 0.0;
#pragma unroll
        for (int b = 0; b < NB; b++) acc[l][b] = 0.0;
    }
    int consumed = 0;  // tiles this thread waited for
    for (int t = 0; t < nt; t++) {
        const int q = t % kGtStages;
        const uint32_t ph = (uint32_t)(t / kGtStages) & 1u;
        // every lane waits (and so sees the tile); the warp leaves together
        if (!__all_sync(0xffffffffu, tc::mbar_wait(&full[q], ph, &abort_flag, err, 1, kGtWaitNs))) break;
        consumed = t + 1;
        const double *tl = tiles + q * kGtTile + warp * 8 * 32;
        const int jb = c0 + t * kGtCols + warp * 8;
        if (active) {
#pragma unroll
            for (int c = 0; c < 8; c++) {
                if (jb + c < cend) {
                    double r = tl[c * 32 + lane];
                    if (!PRED) {
                        mxl[0] = ref_max(mxl[0], fabs(r));
                    } else {
                        double xv[NB];
                        bool xfin = true;  // a zero slice times Inf or NaN still makes NaN
#pragma unroll
                        for (int b = 0; b < NB; b++) {
                            xv[b] = xs[(size_t)b * ldx + jb + c];
                            // exponent field below all-ones (integer test, off the FP64 pipe)
                            xfin = xfin && (__double2hiint(xv[b]) & 0x7ff00000) != 0x7ff00000;
                        }
#pragma unroll
                        for (int l = 0; l < (PRED ? kGvMaxLevels : 1); l++) {
                            // a zero remainder cuts zero slices from here on (r = +-0: every bit
                            // but the sign clear)
                            if ((__double_as_longlong(r) << 1) != 0 || !xfin) {
                                const double sl = (r + sig[l]) - sig[l];
                                r = r - sl;
                                mxl[l] = ref_max(mxl[l], fabs(r));  // max |r_{l+1}|
#pragma unroll
                                for (int b = 0; b < NB; b++) acc[l][b] = fma(sl, xv[b], acc[l][b]);  // exact
                            }
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[q]);
        int rok = 1;
        if (threadIdx.x == 0 && issued < nt) {  // refill stage q once all warps are past tile t
            rok = tc::mbar_wait(&empty[q], ph, &abort_flag, err, 2, kGtWaitNs);
            if (rok) {
                tc::mbar_arrive_expect_tx(&full[q], kGtTileBytes);
                tc::tma_load_2d(tiles + q * kGtTile, &tmA, &full[q], row0, c0 + issued * kGtCols);
                issued++;
            }
        }
        if (!__shfl_sync(0xffffffffu, rok, 0)) break;  // warp 0 leaves together
    }
    if (threadIdx.x == 0) {  // after a timeout: let the loads in flight land before the block ends
        for (int t = consumed; t < issued; t++)
            if (!tc::mbar_wait(&full[t % kGtStages], (uint32_t)(t / kGtStages) & 1u, &never, err, 3, kGtWaitNs))
                break;
    }
    __syncthreads();
    if (abort_flag) return;
    if (PRED) {
        for (int w = 0; w < kGvWarps; w++) {  // the 8 warps hold the same 32 rows
            if (warp == w) {
#pragma unroll
                for (int a = 0; a < (PRED ? kGvMaxLevels : 1); a++)
#pragma unroll
                    for (int b = 0; b < NB; b++) ps[(a * NB + b) * 32 + lane] += acc[a][b];
            }
            __syncthreads();
        }
        for (int i = threadIdx.x; i < kGvMaxLevels * NB * 32; i += blockDim.x) {
            const int pr = i >> 5, rr = row0 + (i & 31);
            if (rr < m && state[rr] != 0) atomicAdd(&P[(size_t)pr * m + rr], ps[i]);
        }
    }
#pragma unroll
    for (int l = 0; l < (PRED ? kGvMaxLevels : 1); l++) {
        __syncthreads();
        red[warp][lane] = mxl[l];
        __syncthreads();
        if (warp == 0 && active) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < kGvWarps; w++) v = ref_max(v, red[w][lane]);
            atomic_max_nonneg(&Ma[(size_t)(PRED ? l + 1 : 0) * m + row], v);
        }
    }
}

// it < 0: the predicted chains T from the row maxima Ma[0..m), every row
// unproven.  it >= 0: the proof after products pass `it` (see above).  out[0]
// = max over proven rows of z - 1 (z = the first level with a zero remainder
// maximum), out[1] = 1 when a row has no zero level within the capacity,
// out[2] is the wait-error flag of the passes, out[4 + it] = rows whose
// chain broke in pass `it`.
__global__ void k_gemv_chain(int m, int rho, int it, double *__restrict__ Ma, int *__restrict__ T,
                             int *__restrict__ state, double *__restrict__ P, int np, int *__restrict__ out) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    if (it < 0) {
        int tau = tau_rule(Ma[row]);
        for (int l = 0; l < kGvMaxLevels; l++, tau += rho - 54) T[(size_t)l * m + row] = tau;
        state[row] = 1;
        return;
    }
    if (state[row] == 0) return;
    int z = -1, bad = -1;
    for (int l = 1; l < kGvMaxLevels + 1; l++) {
        const double v = Ma[(size_t)l * m + row];
        if (v == 0.0) {  // every later slice is zero whatever its tau
            z = l;
            break;
        }
        if (l < kGvMaxLevels && tau_rule(v) != T[(size_t)l * m + row]) {
            bad = l;
            break;
        }
    }
    if (bad > 0) {
        int tau = tau_rule(Ma[(size_t)bad * m + row]);
        for (int l = bad; l < kGvMaxLevels; l++, tau += rho - 54) T[(size_t)l * m + row] = tau;
        for (int l = 1; l < kGvMaxLevels + 1; l++) Ma[(size_t)l * m + row] = 0.0;
        for (int i = 0; i < np; i++) P[(size_t)i * m + row] = 0.0;
        atomicAdd(&out[4 + it], 1);
        return;
    }
    state[row] = 0;
    if (z < 0) atomicExch(&out[1], 1);
    else atomicMax(&out[0], z - 1);
}

template <int NB, bool PRED>
static int launch_gt(dim3 grid, cudaStream_t s, const CUtensorMap &tm, int m, int n, int rho, int cpb, const int *T,
                     const int *state, const double *xs, int ldx, double *P, double *Ma, int *err) {
    static std::atomic<uint64_t> attr{0};  // devices already opted in, per instantiation
    if (smem_optin((const void *)k_gemv_tma<NB, PRED>, kGtSmem, attr) != cudaSuccess)
        return CUOZBLAS_STATUS_CUDA_ERROR;
    k_gemv_tma<NB, PRED><<<grid, 256, kGtSmem, s>>>(tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

static int launch_gt_pred(int nB, dim3 grid, cudaStream_t s, const CUtensorMap &tm, int m, int n, int rho, int cpb,
                          const int *T, const int *state, const double *xs, int ldx, double *P, double *Ma, int *err) {
    switch (nB) {
    case 1: return launch_gt<1, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 2: return launch_gt<2, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 3: return launch_gt<3, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 4: return launch_gt<4, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 5: return launch_gt<5, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 6: return launch_gt<6, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    case 7: return launch_gt<7, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    default: return launch_gt<8, true>(grid, s, tm, m, n, rho, cpb, T, state, xs, ldx, P, Ma, err);
    }
}

// y = fma(alpha, t, beta y) for the 'n' GEMV with the plain form's split
// counts and sums; returns NOT_SUPPORTED (nothing launched) when a count
// exceeds the on-chip capacity, so the caller takes the materialised path.
int gemv_fused_n(cuozblasHandle_t *h, int m, int n, const double *A, int lda, const double *xs, int ldx, int nB,
                 int rho, int maxS, int fastMode, double alpha, double beta, double *y, int *nA_out) {
    if (nB < 1 || nB > kGvMaxLevels || m <= 0 || n <= 0 || maxS < 2) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    State *st = state(h);
    Arena ar(h);
    const uint64_t mk = ar.mark();
    double *M = ar.take<double>((uint64_t)(kGvMaxLevels + 1) * m);
    double *gmax = ar.take<double>(kGvMaxLevels + 2);
    double *P = ar.take<double>((uint64_t)kGvMaxLevels * nB * m);
    double *scratch = ar.take<double>((uint64_t)kGvMaxLevels * nB * m + 1);
    if (!ar.ok) {
        ar.release(mk);
        return CUOZBLAS_STATUS_NOT_SUPPORTED;
    }
    OZB_CHECK(cudaMemsetAsync(M, 0, sizeof(double) * (kGvMaxLevels + 1) * m, st->stream));
    OZB_CHECK(cudaMemsetAsync(gmax, 0, sizeof(double) * (kGvMaxLevels + 2), st->stream));
    const dim3 grid((m + 31) / 32, (n + kGvWarps * kGvCols - 1) / (kGvWarps * kGvCols));
    auto finish_sum = [&](int nA) -> int {
        int maxlevel = (nA - 1) + (nB - 1);
        const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
        maxlevel = (maxlevel - fastMode) > mn ? (maxlevel - fastMode) : mn;  // src/cpu/ozblas_gemm.cpp:163-164
        OZB_TRY(sum_rows_launch(h, m, nA, nB, maxlevel, P, m, alpha, beta, y, scratch));
        *nA_out = nA;
        return CUOZBLAS_STATUS_SUCCESS;
    };
    // two reads of A: the row maxima, then the products on the predicted chains
    // (repeated for the rows whose chain broke); the level passes below when
    // A does not suit a tensor map or a chain stays unproven
    CUtensorMap tm;
    if (!state(h)->env.gemv_levels && make_map_f64(&tm, A, m, n, lda, 32, kGtCols) == CUOZBLAS_STATUS_SUCCESS) {
        const uint64_t mk2 = ar.mark();
        double *Ma = ar.take<double>((uint64_t)(kGvMaxLevels + 1) * m);
        int *T = ar.take<int>((uint64_t)kGvMaxLevels * m);
        int *rstate = ar.take<int>((uint64_t)m);
        int *flags = ar.take<int>(4 + kGtIters);  // zmax, capacity, err, pad, failures per pass
        if (ar.ok) {
            const int rb = (m + 31) / 32, ctiles = (n + kGtCols - 1) / kGtCols;
            int gy = (sm_count() * 8 + rb - 1) / rb;  // about eight blocks per SM in all
            gy = gy < 1 ? 1 : (gy > ctiles ? ctiles : gy);
            const int cpb = (ctiles + gy - 1) / gy * kGtCols;
            const dim3 g2(rb, (n + cpb - 1) / cpb);
            int *err = flags + 2;
            OZB_CHECK(cudaMemsetAsync(Ma, 0, sizeof(double) * (kGvMaxLevels + 1) * m, st->stream));
            OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(double) * kGvMaxLevels * nB * m, st->stream));
            OZB_CHECK(cudaMemsetAsync(flags, 0, sizeof(int) * (4 + kGtIters), st->stream));
            counted(h);
            OZB_TRY((launch_gt<1, false>(g2, st->stream, tm, m, n, rho, cpb, nullptr, nullptr, nullptr, 0, nullptr, Ma,
                                         err)));
            counted(h);
            k_gemv_chain<<<(m + 255) / 256, 256, 0, st->stream>>>(m, rho, -1, Ma, T, rstate, P, kGvMaxLevels * nB,
                                                                  flags);
            OZB_CHECK(cudaGetLastError());
            for (int it = 0; it < kGtIters; it++) {
                counted(h);
                OZB_TRY(launch_gt_pred(nB, g2, st->stream, tm, m, n, rho, cpb, T, rstate, xs, ldx, P, Ma, err));
                counted(h);
                k_gemv_chain<<<(m + 255) / 256, 256, 0, st->stream>>>(m, rho, it, Ma, T, rstate, P,
                                                                      kGvMaxLevels * nB, flags);
                OZB_CHECK(cudaGetLastError());
            }
            OZB_CHECK(cudaMemcpyAsync(st->h_ints, flags, sizeof(int) * (4 + kGtIters), cudaMemcpyDeviceToHost,
                                      st->stream));
            OZB_CHECK(cudaStreamSynchronize(st->stream));
            if (st->h_ints[2] != 0) return CUOZBLAS_STATUS_DEVICE_TIMEOUT;
            if (st->h_ints[1] == 0 && st->h_ints[4 + kGtIters - 1] == 0) {  // every chain proven
                const int zmax = st->h_ints[0];
                const int c = (zmax < 1 ? 1 : zmax) + 1;  // the lines rule's count
                const int nA = c < maxS ? c : maxS;
                if (nA <= kGvMaxLevels) return finish_sum(nA);
            }
        }
        ar.release(mk2);
        ar.ok = true;
    }
    // level passes, all enqueued at once (a pass after the one that leaves every
    // remainder zero returns at once); then the count rule of split_lines_count
    // (level 0 always; the level that leaves every remainder zero counts; at
    // most maxS) from the passes' maxima
    const int last = maxS < kGvMaxLevels ? maxS : kGvMaxLevels;
    for (int p = 0; p <= last; p++) {
        counted(h);
        k_gemv_level<<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, p, M, gmax);
        OZB_CHECK(cudaGetLastError());
    }
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, gmax, sizeof(double) * (last + 1), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    int nA = -1;
    for (int p = 1; p <= last && nA < 0; p++) {
        if (st->h_dbl[p] == 0.0) {  // z = p - 1 for the last row to reach zero
            const int c = (p - 1 < 1 ? 1 : p - 1) + 1;
            nA = c < maxS ? c : maxS;
        } else if (p == maxS - 1) {  // no zero within the cap: z = maxS - 1
            nA = maxS;
        }
    }
    if (nA < 0 || nA > kGvMaxLevels) {  // more levels than the fused kernel holds
        ar.release(mk);
        return CUOZBLAS_STATUS_NOT_SUPPORTED;
    }
    OZB_CHECK(cudaMemsetAsync(P, 0, sizeof(double) * nA * nB * m, st->stream));
    counted(h);
    switch (nB) {
    case 1: k_gemv_products<1><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 2: k_gemv_products<2><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 3: k_gemv_products<3><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 4: k_gemv_products<4><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 5: k_gemv_products<5><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 6: k_gemv_products<6><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    case 7: k_gemv_products<7><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    default: k_gemv_products<8><<<grid, 256, 0, st->stream>>>(m, n, A, lda, rho, nA, M, xs, ldx, P); break;
    }
    OZB_CHECK(cudaGetLastError());
    return finish_sum(nA);
}

}  // namespace ozb
