// gemv_rn.cu — the NearSum GEMV 'n' as correctly rounded exact row dots.
//
// The reference's NearSum GEMV (src/cpu/ozblas_gemv.cpp:22-26 ->
// ozblas_gemm.cpp with n = 1) sums, per row, the products of the row's slices
// with x's slices (src/cpu/ozblas_sum.cpp:10-112).  Those products are exact
// (rho is chosen so that a length-n sum of slice products stays below 2^53 on
// its grid), so when the row's split and x's split are complete their sum is
// the exact row dot and NearSum returns its correct rounding.  Here:
//
//  k_gemv_rn_part   one thread per (row, range of columns): the exact dot of
//                   that range in fixed-grid bins (xbins.cuh), plus the range's
//                   statistics of the row (max, lowest set bit, Inf/NaN); A is
//                   read once, in its column-major order (lanes = rows), through
//                   a per-thread cp.async ring; rows x ranges fill one wave.
//  k_gemv_rn_merge  one thread per row: the certified rounding of the row's
//                   ranges, the row's predicted split count and whether its
//                   split is complete (chain.cuh's argument: the actual chain
//                   descends no slower than the predicted one); the largest
//                   predicted count and one row holding it.
//  k_gemv_rn_write  y = fma(alpha, t, beta y) when every row is complete and
//                   certified and x's split is proven complete (otherwise
//                   nothing is written and the caller runs the fused slice
//                   path).  Its last block splits the row with the largest
//                   predicted count the reference's way: equal to the
//                   prediction, that count is the maximum over all rows (every
//                   actual count is at most its prediction), which the exec
//                   info reports; otherwise every row's count is taken
//                   (k_gemv_rn_count_rows, rare).
#include "fused.h"
#include "ozb_internal.h"
#include "sum.cuh"
#include "xbins.cuh"

namespace ozb {

constexpr int kGrRows = 256;  // rows per block, one per thread
constexpr int kGrGroup = 8;   // columns per group: one cp.async stage, one bin fit
constexpr int kGrStages = 3;  // cp.async ring depth (48 KB per block: groups in flight per thread)
constexpr int kGrKD = 3;      // bins a product is cut onto (the window below is bounded per group)

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

// One thread per (row, range of `cols` columns): each thread streams its own
// row segment through a private cp.async ring in shared memory (a warp's 32
// rows are 256 contiguous bytes of a column, so the copies coalesce; a
// thread reads back only what it copied, so no block barrier is needed),
// and cuts 8 products per group onto its bins with one fit and one bound.
__global__ void __launch_bounds__(kGrRows, 3) k_gemv_rn_part(int m, int n, const double *__restrict__ A, int lda,
                                                          const double *__restrict__ x, int cols,
                                                          GRowPart *__restrict__ parts) {
    __shared__ __align__(16) double ring[kGrStages][kGrGroup][kGrRows];
    const int t = threadIdx.x;
    const int row = blockIdx.x * kGrRows + t;
    const int c0 = blockIdx.y * cols;
    const int len = n - c0 < cols ? n - c0 : cols;
    if (len <= 0) return;  // uniform
    // lanes past the last row read that row again (warp votes need every
    // lane) and write nothing
    const bool live = row < m;
    const double *a = A + (live ? row : m - 1) + (size_t)c0 * lda;
    const double *xc = x + c0;
    const int ng = len / kGrGroup;
    auto issue = [&](int g) {
        if (g < ng) {
            double(*st)[kGrRows] = ring[g % kGrStages];
#pragma unroll
            for (int u = 0; u < kGrGroup; u++) cp_async8(&st[u][t], a + (size_t)(g * kGrGroup + u) * lda);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int g = 0; g < kGrStages - 1; g++) issue(g);
    XAcc acc;
    xacc_init(acc);
    LazyStats rs;  // the row's statistics (per lane)
    for (int g = 0; g < ng; g++) {
        cp_async_wait<kGrStages - 2>();
        double v[kGrGroup], w[kGrGroup];
#pragma unroll
        for (int u = 0; u < kGrGroup; u++) {
            v[u] = ring[g % kGrStages][u][t];
            w[u] = __ldg(xc + g * kGrGroup + u);
        }
        issue(g + kGrStages - 1);  // into the slot read in the previous group (this thread's own)
        unsigned hi = 0u;
#pragma unroll
        for (int u = 0; u < kGrGroup; u++) {
            lazy_elem1(rs, v[u]);
            hi = max(hi, abs_hiword(__dmul_rn(v[u], w[u])));
        }
        xacc_fit1(acc, hi);
#pragma unroll
        for (int u = 0; u < kGrGroup; u++) xacc_product_lean<kGrKD>(acc, v[u], w[u]);
        xacc_lean_bounds<kGrKD>(acc, hi, kGrGroup);
        if ((g & 7) == 7) xacc_normalize1(acc);  // every 64 products
    }
    cp_async_wait<0>();
    for (int j = ng * kGrGroup; j < len; j++) {
        const double v = a[(size_t)j * lda];
        lazy_elem1(rs, v);
        xacc_fit1(acc, abs_hiword(__dmul_rn(v, xc[j])));
        xacc_product(acc, v, xc[j]);
    }
    xacc_normalize1(acc);
    GRowPart gp;
    gp.p.B = (double)acc.B;
#pragma unroll
    for (int k = 0; k < kXK; k++) gp.p.a[k] = acc.a[k];
    gp.p.drop = acc.drop;
    gp.p.es = acc.es;
    gp.p.ea = acc.ea;
    gp.p.flags = (double)acc.flags;
    gp.mx = rs.mx;
    gp.lsb = lazy_key(rs);
    gp.bad = lazy_bad(rs);
    if (live) parts[(size_t)blockIdx.y * m + row] = gp;
}

__global__ void __launch_bounds__(64) k_gemv_rn_merge(int m, int nchunks, const GRowPart *__restrict__ parts, int rho,
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
// count.  One block of 256 threads; the row's elements stay in registers.
constexpr int kGrCountPer = 32;  // elements per thread: rows up to 256 * 32 = 8192 entries
__device__ int gemv_row_count(int row, int n, const double *__restrict__ A, int lda, int rho, int maxS) {
    __shared__ double red[8];
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
    return ns > maxS ? maxS : ns;
}

// y = fma(alpha, t, beta y) when every row is complete and certified and x's
// split is proven complete (otherwise nothing is written and the caller runs
// the fused slice path).  The last block instead splits the row that holds
// the largest predicted count: equal to the prediction, that count is the
// maximum over all rows (each actual count is at most its prediction).
__global__ void __launch_bounds__(256) k_gemv_rn_write(int m, int n, const double *__restrict__ A, int lda, int rho,
                                                       int maxS, const double *__restrict__ t, double alpha,
                                                       double beta, double *__restrict__ y, GemvRnStatus *st,
                                                       const CsrScratch *xs) {
    if (st->incomplete || !xs->valid || !xs->xcomplete) return;  // uniform
    if (blockIdx.x == gridDim.x - 1) {
        const int row = (int)(st->best & 0xffffffffu), pred = (int)(st->best >> 32);
        const int ns = gemv_row_count(row, n, A, lda, rho, maxS);
        if (threadIdx.x == 0) {
            st->count_ok = ns == pred;
            st->nA = ns;
        }
        return;
    }
    const int nb = gridDim.x - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += nb * blockDim.x)
        y[i] = fma(alpha, t[i], beta * y[i]);
}

// The rare case of a row whose split has fewer levels than predicted: the
// actual count of every row (one block per row), the maximum into st->nA.
__global__ void __launch_bounds__(256) k_gemv_rn_count_rows(int n, const double *__restrict__ A, int lda, int rho,
                                                            int maxS, GemvRnStatus *st) {
    const int ns = gemv_row_count(blockIdx.x, n, A, lda, rho, maxS);
    if (threadIdx.x == 0) atomicMax(&st->nA, ns);
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
    // one wave: row blocks x column ranges ~ the resident blocks of the device
    // (a range of at least 64 columns, at most 512 ranges: the merge's exact bin sum)
    const int nsm = sm_count();
    static std::atomic<int> occ_cached{0};
    int occ = occ_cached.load();
    if (occ == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gemv_rn_part, kGrRows, 0) != cudaSuccess || occ < 1)
            occ = 1;
        occ_cached.store(occ);
    }
    const int rblocks = (m + kGrRows - 1) / kGrRows;
    int nsplit = nsm * occ / rblocks;
    const int max_split = (n + 63) / 64 < 512 ? (n + 63) / 64 : 512;
    if (nsplit > max_split) nsplit = max_split;
    if (nsplit < 1) nsplit = 1;
    int cols = (n + nsplit - 1) / nsplit;
    cols = (cols + kGrGroup - 1) / kGrGroup * kGrGroup;
    const int nchunks = (n + cols - 1) / cols;
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
    span_begin(h);
    // x: statistics, then the proof of its predicted chain (count and completeness)
    counted(h);
    OZB_TRY(vec_stats_launch(s, nsm, n, x, &xs->vs, 0));
    counted(h);
    OZB_TRY(csr_proof_launch(s, n, x, rho, maxS, xs, nullptr));
    counted(h);
    k_gemv_rn_part<<<dim3(rblocks, nchunks), kGrRows, 0, s>>>(m, n, A, lda, x, cols, parts);
    counted(h);
    k_gemv_rn_merge<<<(m + 63) / 64, 64, 0, s>>>(m, nchunks, parts, rho, maxS, t, gs);
    int wb = (m + 255) / 256;
    if (wb > nsm * 8) wb = nsm * 8;
    counted(h);
    k_gemv_rn_write<<<wb + 1, 256, 0, s>>>(m, n, A, lda, rho, maxS, t, alpha, beta, y, gs, xs);
    OZB_CHECK(cudaGetLastError());
    span_end(h);
    GemvRnStatus gst;
    CsrScratch xst;
    OZB_CHECK(cudaMemcpyAsync(&gst, gs, sizeof(gst), cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaMemcpyAsync(&xst, xs, sizeof(xst), cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaStreamSynchronize(s));
    int res[3] = {!gst.incomplete && xst.valid && xst.xcomplete, gst.nA, xst.nB};
    if (res[0] && !gst.count_ok) {  // y is written; the exec info needs every row's actual count
        OZB_CHECK(cudaMemsetAsync(&gs->nA, 0, sizeof(int), s));
        counted(h);
        k_gemv_rn_count_rows<<<m, 256, 0, s>>>(n, A, lda, rho, maxS, gs);
        OZB_CHECK(cudaGetLastError());
        OZB_CHECK(cudaMemcpyAsync(&res[1], &gs->nA, sizeof(int), cudaMemcpyDeviceToHost, s));
        OZB_CHECK(cudaStreamSynchronize(s));
    }
    ar.release(mk);
    if (res[0]) {
        *done = true;
        *nA = res[1];
        *nB = res[2];
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
