// gemv_rn.cu — the NearSum GEMV 'n' as correctly rounded exact row dots.
//
// The reference's NearSum GEMV (src/cpu/ozblas_gemv.cpp:22-26 ->
// ozblas_gemm.cpp with n = 1) sums, per row, the products of the row's slices
// with x's slices (src/cpu/ozblas_sum.cpp:10-112).  Those products are exact
// (rho is chosen so that a length-n sum of slice products stays below 2^53 on
// its grid), so when the row's split and x's split are complete their sum is
// the exact row dot and NearSum returns its correct rounding.  Here:
//
//  k_gemv_rn_part   one thread per (row, chunk of columns): the exact dot of
//                   that chunk in fixed-grid bins (xbins.cuh), plus the chunk's
//                   statistics of the row (max, lowest set bit, Inf/NaN); A is
//                   read once, in its column-major order (lanes = rows).
//  k_gemv_rn_merge  one thread per row: the certified rounding of the row's
//                   chunks, the row's predicted split count and whether its
//                   split is complete (chain.cuh's argument: the actual chain
//                   descends no slower than the predicted one); the largest
//                   predicted count and one row holding it.
//  k_gemv_rn_count  the reference's own split of that one row (level by level)
//                   gives its actual count: equal to the predicted maximum, it
//                   is the maximum over all rows (every actual count is at
//                   most its prediction), which the exec info reports.
//  k_gemv_rn_write  y = fma(alpha, t, beta y) when every row is complete and
//                   certified, x's split is proven complete and the count
//                   holds; otherwise nothing is written and the caller runs
//                   the fused slice path.
#include "fused.h"
#include "ozb_internal.h"
#include "sum.cuh"
#include "xbins.cuh"

namespace ozb {

constexpr int kGrRows = 256;   // rows per block, one per thread
constexpr int kGrChunk = 512;  // columns per block

struct GRowPart {
    XPart p;
    double mx;
    int lsb, bad;
};

struct GemvRnStatus {
    unsigned long long best;  // (predicted count << 32) | row, the max over rows
    int incomplete;           // some row is incomplete, uncertified or flagged
    int count_ok;             // the proven row's count equals the predicted maximum
    int done;                 // y was written
    int nA;                   // the rows' split count (exec info)
};

__global__ void __launch_bounds__(kGrRows) k_gemv_rn_part(int m, int n, const double *__restrict__ A, int lda,
                                                          const double *__restrict__ x, GRowPart *__restrict__ parts) {
    __shared__ double xs[kGrChunk];
    const int row = blockIdx.x * kGrRows + threadIdx.x;
    const int c0 = blockIdx.y * kGrChunk;
    const int len = n - c0 < kGrChunk ? n - c0 : kGrChunk;
    for (int j = threadIdx.x; j < len; j += kGrRows) xs[j] = x[c0 + j];
    __syncthreads();
    if (row >= m) return;
    XAcc acc;
    xacc_init(acc);
    double mx = 0.0;
    int lsb = 0, bad = 0;
    const double *a = A + row + (size_t)c0 * lda;
    int j = 0;
    for (int blk = 0; j + 8 <= len; j += 8, blk++) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = __ldg(a + (size_t)(j + u) * lda);
        unsigned hi = 0u;
#pragma unroll
        for (int u = 0; u < 8; u++) {
            scan_elem(v[u], mx, lsb, bad);
            hi = max(hi, abs_hiword(__dmul_rn(v[u], xs[j + u])));
        }
        xacc_fit1(acc, hi);
#pragma unroll
        for (int u = 0; u < 8; u++) xacc_product(acc, v[u], xs[j + u]);
        if ((blk & 7) == 7) xacc_normalize1(acc);  // every 64 products
    }
    for (; j < len; j++) {
        const double v = a[(size_t)j * lda];
        scan_elem(v, mx, lsb, bad);
        xacc_fit1(acc, abs_hiword(__dmul_rn(v, xs[j])));
        xacc_product(acc, v, xs[j]);
    }
    xacc_normalize1(acc);
    GRowPart g;
    g.p.B = (double)acc.B;
#pragma unroll
    for (int k = 0; k < kXK; k++) g.p.a[k] = acc.a[k];
    g.p.drop = acc.drop;
    g.p.es = acc.es;
    g.p.ea = acc.ea;
    g.p.flags = (double)acc.flags;
    g.mx = mx;
    g.lsb = lsb;
    g.bad = bad;
    parts[(size_t)blockIdx.y * m + row] = g;
}

__global__ void __launch_bounds__(256) k_gemv_rn_merge(int m, int nchunks, const GRowPart *__restrict__ parts, int rho,
                                                       int maxS, double *__restrict__ t, GemvRnStatus *st) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    VecStats vs{};
    for (int c = 0; c < nchunks; c++) {
        const GRowPart &g = parts[(size_t)c * m + row];
        vs.mx[0] = ref_max(vs.mx[0], g.mx);
        vs.lsb[0] = max(vs.lsb[0], g.lsb);
        vs.bad[0] |= g.bad;
    }
    double out = 0.0;
    const bool ok = xparts_round1(nchunks, [&](int c) -> const XPart & { return parts[(size_t)c * m + row].p; }, out) &&
                    split_complete(vs, 0, rho, maxS);
    if (!ok) {
        atomicOr(&st->incomplete, 1);
        return;
    }
    t[row] = out;
    // the predicted split count of the row (src/cpu/ozblas_split.cpp:272-289)
    int z = 0;
    if (vs.lsb[0] != 0) {
        const int d = 54 - rho, G0 = rho + tau_rule(vs.mx[0]) - 53;
        const int num = G0 - (kLsbBias - vs.lsb[0]);
        z = num <= 0 ? 0 : (num + d - 1) / d;
    }
    int ns = (z < 1 ? 1 : z) + 1;
    if (ns > maxS) ns = maxS;
    atomicMax(&st->best, ((unsigned long long)ns << 32) | (unsigned)row);
}

// The reference's dense split of one row (src/cpu/ozblas_split.cpp:36-289 on
// the transposed operand: one line of length n), level by level, for its
// count.  One block; the row's elements stay in registers.
constexpr int kGrCountPer = 32;  // elements per thread: rows up to 256 * 32 = 8192 entries
__global__ void __launch_bounds__(256) k_gemv_rn_count(int m, int n, const double *__restrict__ A, int lda, int rho,
                                                       int maxS, GemvRnStatus *st) {
    __shared__ double red[8];
    if (st->incomplete) return;  // uniform
    const int row = (int)(st->best & 0xffffffffu), pred = (int)(st->best >> 32);
    double r[kGrCountPer];
#pragma unroll
    for (int e = 0; e < kGrCountPer; e++) {
        const int j = threadIdx.x + e * 256;
        r[e] = j < n ? A[row + (size_t)j * lda] : 0.0;
    }
    double mx = 0.0;
#pragma unroll
    for (int e = 0; e < kGrCountPer; e++) mx = ref_max(mx, fabs(r[e]));
    mx = block_max_nonneg(mx, red);
    int z = 0, s = 0;
    for (s = 0; s < maxS; s++) {
        if (mx == 0.0) break;  // uniform
        const double sig = dense_sigma(rho, mx, 1);
        double nm = 0.0;
#pragma unroll
        for (int e = 0; e < kGrCountPer; e++) {
            r[e] = r[e] - ((r[e] + sig) - sig);
            nm = ref_max(nm, fabs(r[e]));
        }
        mx = block_max_nonneg(nm, red);
        if (mx == 0.0) {
            z = s;
            break;
        }
    }
    int ns = s >= maxS ? maxS : (z < 1 ? 1 : z) + 1;
    if (ns > maxS) ns = maxS;
    if (threadIdx.x == 0) {
        st->count_ok = ns == pred;
        st->nA = ns;
    }
}

__global__ void __launch_bounds__(256) k_gemv_rn_write(int m, const double *__restrict__ t, double alpha, double beta,
                                                       double *__restrict__ y, const GemvRnStatus *st,
                                                       const CsrScratch *xs) {
    if (st->incomplete || !st->count_ok || !xs->valid || !xs->xcomplete) return;  // uniform
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        y[i] = fma(alpha, t[i], beta * y[i]);
}

__global__ void k_gemv_rn_done(GemvRnStatus *st, const CsrScratch *xs) {
    st->done = !st->incomplete && st->count_ok && xs->valid && xs->xcomplete;
}

// NearSum GEMV 'n' (fastMode 0) through the exact row dots.  *done = false:
// nothing was written, the caller runs the slice path.  *nA / *nB: the
// reference's split counts of A's rows and of x.
int gemv_rn_n(cuozblasHandle_t *h, int m, int n, const double *A, int lda, const double *x, double alpha, double beta,
              double *y, bool *done, int *nA, int *nB) {
    *done = false;
    if (m <= 0 || n <= 0 || n > 256 * kGrCountPer) return CUOZBLAS_STATUS_SUCCESS;
    State *st = state(h);
    cudaStream_t s = st->stream;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    const int nchunks = (n + kGrChunk - 1) / kGrChunk;
    GRowPart *parts = ar.take<GRowPart>((uint64_t)nchunks * m);
    double *t = ar.take<double>((uint64_t)m);
    GemvRnStatus *gs = ar.take<GemvRnStatus>(1);
    CsrScratch *xs = ar.take<CsrScratch>(1);
    if (!ar.ok) {
        ar.release(mk);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    OZB_CHECK(cudaMemsetAsync(gs, 0, sizeof(GemvRnStatus), s));
    OZB_CHECK(cudaMemsetAsync(xs, 0, sizeof(CsrScratch), s));
    const int nsm = sm_count();
    span_begin(h);
    // x: statistics, then the proof of its predicted chain (count and completeness)
    counted(h);
    OZB_TRY(vec_stats_launch(s, nsm, n, x, &xs->vs, 0));
    counted(h);
    OZB_TRY(csr_proof_launch(s, n, x, rho, maxS, xs, nullptr));
    counted(h);
    k_gemv_rn_part<<<dim3((m + kGrRows - 1) / kGrRows, nchunks), kGrRows, 0, s>>>(m, n, A, lda, x, parts);
    counted(h);
    k_gemv_rn_merge<<<(m + 255) / 256, 256, 0, s>>>(m, nchunks, parts, rho, maxS, t, gs);
    counted(h);
    k_gemv_rn_count<<<1, 256, 0, s>>>(m, n, A, lda, rho, maxS, gs);
    int wb = (m + 255) / 256;
    if (wb > nsm * 8) wb = nsm * 8;
    counted(h);
    k_gemv_rn_write<<<wb, 256, 0, s>>>(m, t, alpha, beta, y, gs, xs);
    counted(h);
    k_gemv_rn_done<<<1, 1, 0, s>>>(gs, xs);
    OZB_CHECK(cudaGetLastError());
    span_end(h);
    int res[5];  // done, nA (from the status), nB
    OZB_CHECK(cudaMemcpyAsync(&res[0], &gs->done, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaMemcpyAsync(&res[2], &xs->nB, sizeof(int), cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaStreamSynchronize(s));
    ar.release(mk);
    if (res[0]) {
        *done = true;
        *nA = res[1];
        *nB = res[2];
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
