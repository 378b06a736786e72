// gemm_q.cu — the quad I/O form <__float128, double, double>: binary128 data,
// FP64 slices and exact FP64 slice products, binary128 ordered sum
// (src/cpu/ozblas_gemm.cpp:3-316 with TYPE1 = __float128; the reference runs
// this form on the CPU only).
//
// Split (src/cpu/ozblas_split.cpp:181-221): rho = ceil(113 - (53 - log2 k)/2),
// tau = ceil((double)log2q(max)) (tau_rule_q), slice = (x + sigma) - sigma in
// binary128 (q_split: x rounded to the grid 2^(rho + tau - 113), ties to
// even), stored as the double scalbnq(slice, -tau) with tau per line and
// level.  A slice then has at most 113 - rho + 1 <= 27 bits, so the products
// of two slices over k terms are exact in FP64 and run on the plain form's
// DMMA / skinny kernels.  Sum (src/cpu/ozblas_sum.cpp:382-432): t starts at
// +0 and adds scalbnq(product, tauA + tauB) in pair order, in binary128; the
// output is fmaq(alpha, t, beta * C).  Binary128 arithmetic is q128.cuh.
// FSum only: the reference has no NearSum for mixed types.
#include <math.h>
#include <string.h>
#include <stdlib.h>

#include <vector>

#include "ozb_internal.h"
#include "q128.cuh"
#include "sum.cuh"

namespace ozb {

// getRho<__float128, double> with the reference's own expression (epse 113 and 53).
static int rho_rule_q(int dim, int splitEpsMode) {
    const double d = dim < 1 ? 1.0 : (double)dim;
    if (splitEpsMode == 9) return (int)ceil((113 - (53 - log2(2. * sqrt(d))) / 2));
    return (int)ceil((113 - (53 - log2(d)) / 2));
}

__device__ __forceinline__ Q128 q_ld(const Q128 *p) { return q_make(p->hi, p->lo); }
__device__ __forceinline__ void q_st(Q128 *p, Q128 v) {
    p->lo = v.lo;
    p->hi = v.hi;
}

// Largest magnitude over the block (non-NaN magnitudes order as unsigned bits).
__device__ Q128 block_max_q(Q128 v, Q128 *red) {
    for (int o = 16; o > 0; o >>= 1) {
        Q128 w;
        w.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
        w.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
        if (q_mag_less(v, w)) v = w;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    Q128 r = q_zero(0);
    for (int i = 0; i < nw; i++)
        if (q_mag_less(r, red[i])) r = red[i];
    return r;
}

// One CTA per line; element i of line l at X[l * ls + i * es] (es = 1:
// contiguous lines; ls = 1, es = ld: the rows of a column-major matrix).
// The remainders live in rem (k per line).  COUNT: atomicMax(*zmax, first
// level leaving a zero line).  WRITE: ns FP64 slices [s][line][ldo] and
// exps[s * nl + line] = tau.
template <bool WRITE>
__global__ void __launch_bounds__(256) k_split_lines_q(int k, int nl, const Q128 *__restrict__ X, int64_t ls,
                                                       int64_t es, int rho, int levels, double *__restrict__ out,
                                                       int ldo, short *__restrict__ exps, Q128 *__restrict__ rem,
                                                       int *__restrict__ zmax) {
    __shared__ Q128 red[8];
    const int line = blockIdx.x;
    if (line >= nl) return;
    const Q128 *x = X + (size_t)line * ls;
    Q128 *r = rem + (size_t)line * k;
    Q128 mx = q_zero(0);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const Q128 v = q_ld(x + (size_t)i * es);
        q_st(r + i, v);
        const Q128 a = q_abs(v);
        if (q_mag_less(mx, a)) mx = a;
    }
    mx = block_max_q(mx, red);
    int z = levels;
    for (int s = 0; s < levels; s++) {
        const int tau = tau_rule_q(mx);
        if (WRITE && threadIdx.x == 0) exps[(size_t)s * nl + line] = (short)tau;
        double *o = WRITE ? out + ((size_t)s * nl + line) * ldo : nullptr;
        Q128 nm = q_zero(0);
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            Q128 v = q_ld(r + i);
            const double sl = q_split(v, rho, tau);
            q_st(r + i, v);
            const Q128 a = q_abs(v);
            if (q_mag_less(nm, a)) nm = a;
            if (WRITE) o[i] = sl;
        }
        if (WRITE)
            for (int i = k + threadIdx.x; i < ldo; i += blockDim.x) o[i] = 0.0;
        mx = block_max_q(nm, red);
        if (!WRITE && q_is_zero(mx)) {
            z = s;
            break;
        }
    }
    if (!WRITE && threadIdx.x == 0) atomicMax(zmax, z);
}

// The WRITE pass of k_split_lines_q with the slices cut into D int8 digit
// planes instead of FP64 slices: slice = q 2^(rho - 113) with |q| < 2^(7 D),
// digit d of level s = sign(q) ((|q| >> 7 (D - 1 - d)) & 127) at
// dig[((s D + d) lines_pad + line) k_pad + i] (the buffer is zeroed before).
__global__ void __launch_bounds__(256) k_split_lines_q_digits(int k, int nl, const Q128 *__restrict__ X, int64_t ls,
                                                              int64_t es, int rho, int ns, int D, int lines_pad,
                                                              int k_pad, int8_t *__restrict__ dig,
                                                              short *__restrict__ exps, Q128 *__restrict__ rem) {
    __shared__ Q128 red[8];
    const int line = blockIdx.x;
    if (line >= nl) return;
    const Q128 *x = X + (size_t)line * ls;
    Q128 *r = rem + (size_t)line * k;
    Q128 mx = q_zero(0);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const Q128 v = q_ld(x + (size_t)i * es);
        q_st(r + i, v);
        const Q128 a = q_abs(v);
        if (q_mag_less(mx, a)) mx = a;
    }
    mx = block_max_q(mx, red);
    for (int s = 0; s < ns; s++) {
        const int tau = tau_rule_q(mx);
        if (threadIdx.x == 0) exps[(size_t)s * nl + line] = (short)tau;
        Q128 nm = q_zero(0);
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            Q128 v = q_ld(r + i);
            const double sl = q_split(v, rho, tau);
            q_st(r + i, v);
            const Q128 a = q_abs(v);
            if (q_mag_less(nm, a)) nm = a;
            const long long q = (long long)scale2(sl, 113 - rho);  // exact integer
            const unsigned long long aq = (unsigned long long)(q < 0 ? -q : q);
            for (int d = 0; d < D; d++) {
                const int dv = (int)((aq >> (7 * (D - 1 - d))) & 127);
                dig[(((size_t)s * D + d) * lines_pad + line) * k_pad + i] = (int8_t)(q < 0 ? -dv : dv);
            }
        }
        mx = block_max_q(nm, red);
    }
}

// General GEMM sum: element e = col * m + row of a block of nc columns from
// c0; pbuf[p * count + e] exact FP64 products of pair dp[p].
__global__ void k_sum_pairs_q(int m, int n, int64_t count, int c0, int np, const double *__restrict__ pbuf,
                              const int2 *__restrict__ dp, const short *__restrict__ Ea,
                              const short *__restrict__ Eb, Q128 alpha, Q128 beta, Q128 *__restrict__ C, int ldc) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const int row = (int)(e % m), col = c0 + (int)(e / m);
    Q128 t = q_zero(0);
    for (int p = 0; p < np; p++) {
        const int2 pr = dp[p];
        const int sc = Ea[(size_t)pr.x * m + row] + Eb[(size_t)pr.y * n + col];
        t = q_add(t, q_from_double_scaled(pbuf[(size_t)p * count + e], sc));
    }
    Q128 *cp = C + (size_t)col * ldc + row;
    q_st(cp, q_fma(alpha, t, q_mul(beta, q_ld(cp))));
}

// Skinny sum: P[(ia * nB + ib) * ldp + row]; A's exponents at Ea[ia * ldea + row], the vector's at Eb[ib].
__global__ void k_sum_rows_q(int m, int nA, int nB, int maxlevel, const double *__restrict__ P, int64_t ldp,
                             const short *__restrict__ Ea, int ldea, const short *__restrict__ Eb, Q128 alpha,
                             Q128 beta, Q128 *__restrict__ y) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    Q128 t = q_zero(0);
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) {
        const int sc = Ea[(size_t)ia * ldea + row] + Eb[ib];
        t = q_add(t, q_from_double_scaled(P[(size_t)(ia * nB + ib) * ldp + row], sc));
    });
    q_st(y + row, q_fma(alpha, t, q_mul(beta, q_ld(y + row))));
}

static int ceil_to(int v, int q) { return (v + q - 1) / q * q; }

// Split op(X): nl lines of length k (strided: element i of line l at X[i*ldx + l]).
static int split_operand_q(cuozblasHandle_t *h, bool lines_strided, int nl, int k, const Q128 *X, int ldx, int rho,
                           int maxS, int ldk, double **slices, short **exps, int *ns, Arena &ar) {
    State *st = state(h);
    const int64_t ls = lines_strided ? 1 : ldx, es = lines_strided ? ldx : 1;
    const uint64_t mk = ar.mark();
    Q128 *rem = ar.take<Q128>((uint64_t)nl * (k > 0 ? k : 1));
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    // count (as split_lines_count: level 0 always, then until a level leaves every line zero)
    if (maxS <= 1 || nl == 0) {
        *ns = 1;
    } else {
        OZB_CHECK(cudaMemsetAsync(st->d_ints, 0, sizeof(int), st->stream));
        counted(h);
        k_split_lines_q<false><<<nl, 256, 0, st->stream>>>(k, nl, X, ls, es, rho, maxS - 1, nullptr, 0, nullptr, rem,
                                                            st->d_ints);
        OZB_CHECK(cudaGetLastError());
        OZB_CHECK(cudaMemcpyAsync(st->h_ints, st->d_ints, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
        OZB_CHECK(cudaStreamSynchronize(st->stream));
        const int zmax = st->h_ints[0];
        const int c = (zmax < 1 ? 1 : zmax) + 1;
        *ns = c < maxS ? c : maxS;
    }
    ar.release(mk);
    *slices = ar.take<double>((uint64_t)(*ns) * nl * ldk);
    *exps = ar.take<short>((uint64_t)(*ns) * nl);
    const uint64_t mk2 = ar.mark();
    rem = ar.take<Q128>((uint64_t)nl * (k > 0 ? k : 1));
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    if (nl > 0) {
        counted(h);
        k_split_lines_q<true><<<nl, 256, 0, st->stream>>>(k, nl, X, ls, es, rho, *ns, *slices, ldk, *exps, rem,
                                                           nullptr);
        OZB_CHECK(cudaGetLastError());
    }
    ar.release(mk2);
    return CUOZBLAS_STATUS_SUCCESS;
}

int gemm_q_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, const void *alpha_h, const void *Av,
                int lda, const void *Bv, int ldb, const void *beta_h, void *Cv, int ldc, int fastMode) {
    State *st = state(h);
    const Q128 *A = reinterpret_cast<const Q128 *>(Av), *B = reinterpret_cast<const Q128 *>(Bv);
    Q128 *C = reinterpret_cast<Q128 *>(Cv);
    Q128 alpha, beta;
    memcpy(&alpha, alpha_h, 16);
    memcpy(&beta, beta_h, 16);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule_q(k, h->splitEpsMode);
    Arena ar(h);
    const bool dot = (m == 1 && n == 1);
    const bool skinny_n = (n == 1);
    const int ldk = dot || skinny_n ? ceil_to(k > 0 ? k : 1, 2) : ceil_to(k > 0 ? k : 1, 16);

    ev_record(h, 0);
    st->plain_timers = true;
    double *Sa = nullptr, *Sb = nullptr;
    short *Ea = nullptr, *Eb = nullptr;
    int nA = 0, nB = 0;
    // lines of op(A): rows of A ('n': strided by lda); op(B): columns of B ('t': strided)
    OZB_TRY(split_operand_q(h, dot ? false : !is_trans(ta), m, k, A, dot ? k : lda, rho, maxS, ldk, &Sa, &Ea, &nA,
                            ar));
    ev_record(h, 1);
    OZB_TRY(split_operand_q(h, skinny_n ? false : is_trans(tb), n, k, B, skinny_n ? k : ldb, rho, maxS, ldk, &Sb,
                            &Eb, &nB, ar));
    ev_record(h, 2);
    const int fast = dot ? 0 : fastMode;
    int maxlevel = (nA - 1) + (nB - 1);
    {
        const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
        maxlevel = (maxlevel - fast) > mn ? (maxlevel - fast) : mn;  // src/cpu/ozblas_gemm.cpp:163-164
    }
    int np = 0;
    for_each_pair(nA, nB, maxlevel, [&](int, int) { np++; });
    h->nSplitA = (float)nA;
    h->nSplitB = (float)nB;
    h->nSplitC = dot ? 1.f : (skinny_n && fast == 0 ? (float)(maxlevel + 1 < nA ? maxlevel + 1 : nA) : (float)np);
    h->mbk = m;
    h->nbk = n;

    if (dot || skinny_n) {
        const int rows = dot ? 1 : m;
        double *P = ar.take<double>((uint64_t)nA * nB * rows);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(pair_products_skinny(h, dot, m, k, nA, nB, Sa, Sb, ldk, P));
        ev_record(h, 3);
        counted(h);
        k_sum_rows_q<<<(rows + 127) / 128, 128, 0, st->stream>>>(rows, nA, nB, maxlevel, P, rows, Ea, rows, Eb, alpha,
                                                                 beta, C);
        OZB_CHECK(cudaGetLastError());
        ev_record(h, 4);
        return CUOZBLAS_STATUS_SUCCESS;
    }

    // Pair products on the INT8 tensor cores when every slice is D <= 4 int8
    // digits (|q| <= 2^(113 - rho) < 2^(7 D)), an INT32 group of D digit pairs
    // over k stays exact, and the products of all pairs fit the arena at once.
    {
        const int D = (113 - rho + 1 + 6) / 7;
        const int k_pad = (k + 127) / 128 * 128;
        const int lpadA = (m + 127) / 128 * 128, lpadB = (n + 127) / 128 * 128;
        const uint64_t need = (uint64_t)nA * D * lpadA * k_pad + (uint64_t)nB * D * lpadB * k_pad +
                              sizeof(double) * (uint64_t)np * m * n + (uint64_t)16 * (m > n ? m : n) * k + (1u << 20);
        const uint64_t avail = h->workSizeBytes - ((ar.mark() + 255) / 256 * 256);
        if (D <= 4 && (double)D * k * 127.0 * 127.0 < 2147483647.0 && need < avail && !state(h)->env.q_dmma) {
            std::vector<int2> pl;
            for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { pl.push_back(make_int2(ia, ib)); });
            int8_t *dg[2];
            for (int o = 0; o < 2; o++) {
                const int nl = o == 0 ? m : n, ns = o == 0 ? nA : nB, lpad = o == 0 ? lpadA : lpadB;
                const bool strided = o == 0 ? !is_trans(ta) : is_trans(tb);
                const Q128 *X = o == 0 ? A : B;
                const int ldx = o == 0 ? lda : ldb;
                dg[o] = ar.take<int8_t>((uint64_t)ns * D * lpad * k_pad);
                short *ex = o == 0 ? Ea : Eb;  // the FP64 split's exponents are the same taus
                const uint64_t mk2 = ar.mark();
                Q128 *rem = ar.take<Q128>((uint64_t)nl * (k > 0 ? k : 1));
                if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
                OZB_CHECK(cudaMemsetAsync(dg[o], 0, (size_t)ns * D * lpad * k_pad, st->stream));
                counted(h);
                k_split_lines_q_digits<<<nl, 256, 0, st->stream>>>(k, nl, X, strided ? 1 : ldx, strided ? ldx : 1, rho,
                                                                   ns, D, lpad, k_pad, dg[o], ex, rem);
                OZB_CHECK(cudaGetLastError());
                ar.release(mk2);
            }
            double *pbuf = ar.take<double>((uint64_t)np * m * n);
            int2 *dp = ar.take<int2>(np > 0 ? np : 1);
            if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
            OZB_CHECK(cudaMemcpyAsync(dp, pl.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, st->stream));
            OZB_TRY(i8_exact_pairs(h, m, n, k_pad, dg[0], lpadA, nA * D, dg[1], lpadB, nB * D, D, pl,
                                   2 * (rho - 113), nullptr, nullptr, pbuf));
            const int64_t count = (int64_t)m * n;
            counted(h);
            k_sum_pairs_q<<<(unsigned)((count + 255) / 256), 256, 0, st->stream>>>(m, n, count, 0, np, pbuf, dp, Ea,
                                                                                  Eb, alpha, beta, C, ldc);
            OZB_CHECK(cudaGetLastError());
            ev_record(h, 3);
            ev_record(h, 4);
            return CUOZBLAS_STATUS_SUCCESS;
        }
    }

    int2 *hp = new int2[np > 0 ? np : 1];
    int q = 0;
    for_each_pair(nA, nB, maxlevel, [&](int ia, int ib) { hp[q++] = make_int2(ia, ib); });
    int2 *dp = ar.take<int2>(np > 0 ? np : 1);
    if (!ar.ok) {
        delete[] hp;
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    cudaError_t ce = cudaMemcpyAsync(dp, hp, sizeof(int2) * np, cudaMemcpyHostToDevice, st->stream);
    cudaError_t ce2 = cudaStreamSynchronize(st->stream);
    delete[] hp;
    OZB_CHECK(ce);
    OZB_CHECK(ce2);
    // pair products to a buffer, blocked over columns when the arena is short
    const uint64_t avail = h->workSizeBytes - ((ar.mark() + 255) / 256 * 256);
    int64_t ncols = (int64_t)(avail / (sizeof(double) * (uint64_t)np * (uint64_t)m));
    if (ncols >= n) {
        ncols = n;
    } else {
        ncols = ncols / 64 * 64;
        if (ncols == 0) return CUOZBLAS_STATUS_WORKSPACE;
    }
    double *pbuf = ar.take<double>((uint64_t)np * m * ncols);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    for (int64_t c0 = 0; c0 < n; c0 += ncols) {
        const int nc = (int)((n - c0) < ncols ? (n - c0) : ncols);
        OZB_TRY(gemm_pairs_store(h, m, nc, n, ldk, Sa, Sb + (size_t)c0 * ldk, dp, np, pbuf));
        const int64_t count = (int64_t)m * nc;
        counted(h);
        k_sum_pairs_q<<<(unsigned)((count + 255) / 256), 256, 0, st->stream>>>(m, n, count, (int)c0, np, pbuf, dp, Ea,
                                                                              Eb, alpha, beta, C, ldc);
        OZB_CHECK(cudaGetLastError());
    }
    ev_record(h, 3);  // products and sum interleave per column block here
    ev_record(h, 4);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
