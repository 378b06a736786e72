// csrmv_fused.cu — the plain-form CSRMV without materialised slices.
//
// The reference splits A row by row (src/cpu/ozblas_split.cpp:779-815), x with
// one global tau chain (:62-103), forms one CSRMM per A slice with a
// sequential fma chain per row (src/cpu/ozblas_blas_wrapper.cpp:231-255) and
// sums the pair products per row (src/cpu/ozblas_csrmv.cpp:100-160).  Here:
//
//  1. max|x| (and the longest row);
//  2. x's chain is predicted (tau_{s+1} = tau_s + rho - 54) and proven by
//     per-level flags over all of x (as in dot_fused.cu); if it does not hold,
//     or x needs more than 8 levels, the caller uses the general path before
//     anything is written;
//  3. one thread per row: the row's own tau chain (rho from its nnz, sigma
//     divided by the CG's splitShift) is exact per row, so it is computed in
//     place; x's slices at the gathered columns come from the proven chain;
//     every pair product is the CPU's sequential fma chain in storage order,
//     summed in (ik, ia) order (FSum) or NearSum-ed.  Rows longer than 8 or
//     needing more than 6 levels are deferred to a per-row general kernel.
//
// Pairs whose A slice is beyond a row's own exact split are zero slices in
// the reference; they add +0 to the ordered sum and nothing to NearSum, so
// skipping them leaves the bits unchanged.  fastMode must be 0 (the caller
// uses the general path otherwise).
#include "ozb_device.cuh"
#include "ozb_internal.h"
#include "sum.cuh"

namespace ozb {

constexpr int kCsrLv = 8;           // levels of x computed / checked
constexpr int kCsrRowMax = 8;       // entries per row held on chip
constexpr int kCsrAlv = 6;          // levels of a row held on chip
constexpr int kCsrThreads = 128;

struct CsrScratch {
    double xmax;
    unsigned int nz, hi;
    int valid, nB, maxlen, nslow, zmax;  // zmax: first zero-remainder level, max over rows
    double sigma[kCsrLv];
};

__global__ void __launch_bounds__(256) k_csr_prep(int m, int n, const double *__restrict__ x,
                                                  const int *__restrict__ rowptr, CsrScratch *sc) {
    __shared__ double red[8];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double mx = 0.0;
    int ml = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride)
        mx = ref_max(mx, fabs(x[i]));
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)m; i += stride) {
        const int l = rowptr[i + 1] - rowptr[i];
        ml = ml > l ? ml : l;
    }
    mx = block_max_nonneg(mx, red);
    for (int o = 16; o > 0; o >>= 1) {
        const int t = __shfl_xor_sync(0xffffffffu, ml, o);
        ml = ml > t ? ml : t;
    }
    if (threadIdx.x == 0) atomic_max_nonneg(&sc->xmax, mx);
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->maxlen, ml);
}

__device__ __forceinline__ double csr_tau_threshold(int t) {
    const int e = t - 1;
    if (e < -1022 || e > 1023) return -1.0;
    const int ae = e < 0 ? -e : e;
    int p = (ae == 0) ? -1 : (31 - clz32((uint32_t)ae));
    if (e < 0 && (ae & (ae - 1)) == 0) p -= 1;
    int J;
    switch (p) {
        case 2: J = 1; break;
        case 3: J = 2; break;
        case 4: J = 5; break;
        case 5: J = 11; break;
        case 6: J = 22; break;
        case 7: J = 44; break;
        case 8: J = 88; break;
        case 9: J = 177; break;
        case 10: J = 354; break;
        default: J = 0; break;
    }
    return from_bits(dbits(pow2(e)) + (uint64_t)J);
}

// Per-level flags of x's predicted chain.
__global__ void __launch_bounds__(256) k_vec_chain_flags(int n, const double *__restrict__ x, int rho,
                                                         CsrScratch *sc) {
    __shared__ double sig[kCsrLv], thr[kCsrLv];
    if (threadIdx.x == 0) {
        int tau = tau_rule(sc->xmax);
        for (int s = 0; s < kCsrLv; s++) {
            sig[s] = 0.75 * pow2(rho + tau);
            tau = tau + rho - 54;
            thr[s] = csr_tau_threshold(tau);
        }
    }
    __syncthreads();
    unsigned nz = 0, hi = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        double r = x[i];
#pragma unroll
        for (int s = 0; s < kCsrLv; s++) {
            const double sl = (r + sig[s]) - sig[s];
            r = r - sl;
            const uint64_t rb = dbits(r) & 0x7fffffffffffffffULL;
            nz |= (rb != 0) ? (1u << s) : 0u;
            hi |= (rb > dbits(thr[s])) ? (1u << s) : 0u;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nz |= __shfl_xor_sync(0xffffffffu, nz, o);
        hi |= __shfl_xor_sync(0xffffffffu, hi, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicOr(&sc->nz, nz);
        atomicOr(&sc->hi, hi);
    }
}

__global__ void k_vec_chain_finish(CsrScratch *sc, int rho, int maxS) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int tau = tau_rule(sc->xmax);
    double thr[kCsrLv];
    for (int s = 0; s < kCsrLv; s++) {
        sc->sigma[s] = 0.75 * pow2(rho + tau);
        tau = tau + rho - 54;
        thr[s] = csr_tau_threshold(tau);
    }
    const unsigned nz = sc->nz, hi = sc->hi;
    int z = kCsrLv;
    for (int s = 0; s < kCsrLv; s++)
        if (!(nz & (1u << s))) {
            z = s;
            break;
        }
    int ns;
    bool ok = true;
    if (z >= kCsrLv) {
        if (maxS > kCsrLv) ok = false;
        ns = maxS;
    } else {
        ns = (z < 1 ? 1 : z) + 1;
        if (ns > maxS) ns = maxS;
    }
    for (int s = 0; ok && s + 1 < ns; s++)
        if ((nz & (1u << s)) && (!(hi & (1u << s)) || thr[s] < 0.0)) ok = false;
    sc->nB = ns;
    sc->valid = ok ? 1 : 0;
}

// One thread per row; per-thread slices in shared memory laid out
// [index][thread] so a warp's accesses hit distinct banks.
template <int SUM_MODE>
__global__ void __launch_bounds__(kCsrThreads) k_csrmv_fast(int m, const double *__restrict__ val,
                                                            const int *__restrict__ colind,
                                                            const int *__restrict__ rowptr,
                                                            const double *__restrict__ x, int shift, int epsmode,
                                                            int maxS, double alpha, double beta,
                                                            double *__restrict__ y, CsrScratch *__restrict__ sc,
                                                            int *__restrict__ slow_rows) {
    extern __shared__ double sh[];
    __shared__ double xs_sigma[kCsrLv];
    if (!sc->valid) return;
    const int nB = sc->nB;
    if (threadIdx.x < kCsrLv) xs_sigma[threadIdx.x] = sc->sigma[threadIdx.x];
    __syncthreads();
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int T = blockDim.x, t = threadIdx.x;
    double *A = sh;                                  // [kCsrAlv * kCsrRowMax][T]
    double *X = sh + kCsrAlv * kCsrRowMax * T;      // [kCsrLv * kCsrRowMax][T]
    double *Tm = X + kCsrLv * kCsrRowMax * T;       // [kCsrAlv * kCsrLv][T] (NearSum terms)
    const int lo = rowptr[row], len = rowptr[row + 1] - lo;
    if (len > kCsrRowMax) {
        slow_rows[atomicAdd(&sc->nslow, 1)] = row;
        return;
    }
    double r[kCsrRowMax];
    int c[kCsrRowMax];
    double mx = 0.0;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        r[e] = e < len ? val[lo + e] : 0.0;
        c[e] = e < len ? colind[lo + e] : 0;
        mx = ref_max(mx, fabs(r[e]));
    }
    // the row's own split (src/cpu/ozblas_split.cpp:779-815, sigma / shift)
    int na = 0, z = 0;
    if (len > 0) {
        const int rho = rho_rule(len, epsmode);
        z = maxS;
        for (int s = 0; s < kCsrAlv && s < maxS; s++) {
            const double sigma = 0.75 * pow2(rho + tau_rule(mx)) / (double)shift;
            double nm = 0.0;
#pragma unroll
            for (int e = 0; e < kCsrRowMax; e++) {
                const double sl = (r[e] + sigma) - sigma;
                r[e] = r[e] - sl;
                A[(s * kCsrRowMax + e) * T + t] = sl;
                nm = ref_max(nm, fabs(r[e]));
            }
            na = s + 1;
            mx = nm;
            if (nm == 0.0) {
                z = s;
                break;
            }
        }
        if (mx != 0.0 && na < maxS) {  // needs more levels than held on chip
            slow_rows[atomicAdd(&sc->nslow, 1)] = row;
            return;
        }
    }
    atomicMax(&sc->zmax, z);
    // x's slices at this row's columns
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        double xr = e < len ? x[c[e]] : 0.0;
        for (int s = 0; s < nB; s++) {
            const double sl = (xr + xs_sigma[s]) - xs_sigma[s];
            xr = xr - sl;
            X[(s * kCsrRowMax + e) * T + t] = sl;
        }
    }
    double tsum = 0.0;
    int np = 0;
    const int maxlevel = na + nB - 2;
    for (int ik = 0; ik <= maxlevel; ik++) {
        const int ia0 = ik - (nB - 1) > 0 ? ik - (nB - 1) : 0, ia1 = ik < na - 1 ? ik : na - 1;
        for (int ia = ia0; ia <= ia1; ia++) {
            const int ib = ik - ia;
            double p = 0.0;
            for (int e = 0; e < len; e++)
                p = fma(A[(ia * kCsrRowMax + e) * T + t], X[(ib * kCsrRowMax + e) * T + t], p);
            if (SUM_MODE == 1)
                Tm[np * T + t] = p;
            else
                tsum += p;
            np++;
        }
    }
    if (SUM_MODE == 1) tsum = nearsum(np, Tm + t, T);
    y[row] = fma(alpha, tsum, beta * y[row]);
}

// Recompute slice `lv` of v from scratch along the chain sig[0..lv].
__device__ __forceinline__ double slice_at(double v, const double *sig, int lv) {
    double sl = 0.0;
    for (int s = 0; s <= lv; s++) {
        sl = (v + sig[s]) - sig[s];
        v = v - sl;
    }
    return sl;
}

// General per-row kernel for the deferred rows: any length, any level count;
// slices recomputed on the fly; NearSum terms in `terms` (slot x maxS*kCsrLv).
template <int SUM_MODE>
__global__ void __launch_bounds__(128) k_csrmv_slow(int nrows, const int *__restrict__ rows,
                                                    const double *__restrict__ val, const int *__restrict__ colind,
                                                    const int *__restrict__ rowptr, const double *__restrict__ x,
                                                    int shift, int epsmode, int maxS, double alpha, double beta,
                                                    double *__restrict__ y, CsrScratch *__restrict__ sc,
                                                    double *__restrict__ terms) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nrows) return;
    const int row = rows[slot];
    const int lo = rowptr[row], hi = rowptr[row + 1], len = hi - lo;
    const int nB = sc->nB;
    double sa[kMaxSplitDefault];
    int na = 0, z = 0;
    if (len > 0) {
        z = maxS;
        const int rho = rho_rule(len, epsmode);
        double mx = 0.0;
        for (int i = lo; i < hi; i++) mx = ref_max(mx, fabs(val[i]));
        for (int s = 0; s < maxS; s++) {
            sa[s] = 0.75 * pow2(rho + tau_rule(mx)) / (double)shift;
            na = s + 1;
            double nm = 0.0;
            for (int i = lo; i < hi; i++) {
                double v = val[i];
                for (int q = 0; q <= s; q++) {
                    const double sl = (v + sa[q]) - sa[q];
                    v = v - sl;
                }
                nm = ref_max(nm, fabs(v));
            }
            mx = nm;
            if (nm == 0.0) {
                z = s;
                break;
            }
        }
    }
    atomicMax((int *)&sc->zmax, z);
    double tsum = 0.0;
    int np = 0;
    double *tm = terms + (size_t)slot * kMaxSplitDefault * kCsrLv;
    const int maxlevel = na + nB - 2;
    for (int ik = 0; ik <= maxlevel; ik++) {
        const int ia0 = ik - (nB - 1) > 0 ? ik - (nB - 1) : 0, ia1 = ik < na - 1 ? ik : na - 1;
        for (int ia = ia0; ia <= ia1; ia++) {
            const int ib = ik - ia;
            double p = 0.0;
            for (int i = lo; i < hi; i++)
                p = fma(slice_at(val[i], sa, ia), slice_at(x[colind[i]], sc->sigma, ib), p);
            if (SUM_MODE == 1)
                tm[np] = p;
            else
                tsum += p;
            np++;
        }
    }
    if (SUM_MODE == 1) tsum = nearsum(np, tm, 1);
    y[row] = fma(alpha, tsum, beta * y[row]);
}

// Fused CSRMV.  *done = false (and y untouched) when x's chain is not proven
// or needs more than 8 levels: the caller then runs the general path.
int csrmv_fused(cuozblasHandle_t *h, int m, int n, double alpha, const double *val, const int *colind,
                const int *rowptr, const double *x, double beta, double *y, int shift, bool *done, int *nA_out,
                int *nB_out) {
    State *st = state(h);
    *done = false;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    CsrScratch *sc = ar.take<CsrScratch>(1);
    int *slow = ar.take<int>(m > 0 ? m : 1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    OZB_CHECK(cudaMemsetAsync(sc, 0, sizeof(CsrScratch), st->stream));
    int dev = 0, nsm = 0;
    OZB_CHECK(cudaGetDevice(&dev));
    OZB_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t span = m > n ? m : n;
    int blocks = (int)((span + 255) / 256);
    if (blocks > nsm * 8) blocks = nsm * 8;
    if (blocks < 1) blocks = 1;
    counted(h);
    k_csr_prep<<<blocks, 256, 0, st->stream>>>(m, n, x, rowptr, sc);
    int fb = (int)(((int64_t)n + 255) / 256);
    if (fb > nsm * 8) fb = nsm * 8;
    if (fb < 1) fb = 1;
    counted(h);
    k_vec_chain_flags<<<fb, 256, 0, st->stream>>>(n, x, rho, sc);
    counted(h);
    k_vec_chain_finish<<<1, 32, 0, st->stream>>>(sc, rho, maxS);
    const size_t sm_fsum = sizeof(double) * (kCsrAlv + kCsrLv) * kCsrRowMax * kCsrThreads;
    const size_t sm_near = sm_fsum + sizeof(double) * kCsrAlv * kCsrLv * kCsrThreads;
    const int rb = (m + kCsrThreads - 1) / kCsrThreads;
    if (m > 0) {
        counted(h);
        if (h->sumMode == 1) {
            OZB_CHECK(cudaFuncSetAttribute(k_csrmv_fast<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_near));
            k_csrmv_fast<1><<<rb, kCsrThreads, sm_near, st->stream>>>(m, val, colind, rowptr, x, shift,
                                                                       h->splitEpsMode, maxS, alpha, beta, y, sc, slow);
        } else {
            OZB_CHECK(cudaFuncSetAttribute(k_csrmv_fast<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_fsum));
            k_csrmv_fast<0><<<rb, kCsrThreads, sm_fsum, st->stream>>>(m, val, colind, rowptr, x, shift,
                                                                       h->splitEpsMode, maxS, alpha, beta, y, sc, slow);
        }
    }
    OZB_CHECK(cudaGetLastError());
    int res[5];  // valid, nB, maxlen, nslow, zmax (partial until the deferred rows ran)
    OZB_CHECK(cudaMemcpyAsync(res, &sc->valid, sizeof(res), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    if (!res[0]) {
        ar.release(mk);
        return CUOZBLAS_STATUS_SUCCESS;  // y untouched: general path
    }
    const int nslow = res[3];
    if (nslow > 0) {
        const int chunk = 8192;
        double *terms = ar.take<double>((uint64_t)chunk * kMaxSplitDefault * kCsrLv);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        for (int c0 = 0; c0 < nslow; c0 += chunk) {
            const int nr = nslow - c0 < chunk ? nslow - c0 : chunk;
            counted(h);
            if (h->sumMode == 1)
                k_csrmv_slow<1><<<(nr + 127) / 128, 128, 0, st->stream>>>(nr, slow + c0, val, colind, rowptr, x,
                                                                          shift, h->splitEpsMode, maxS, alpha, beta,
                                                                          y, sc, terms);
            else
                k_csrmv_slow<0><<<(nr + 127) / 128, 128, 0, st->stream>>>(nr, slow + c0, val, colind, rowptr, x,
                                                                          shift, h->splitEpsMode, maxS, alpha, beta,
                                                                          y, sc, terms);
            OZB_CHECK(cudaGetLastError());
        }
    }
    if (nslow > 0) {
        OZB_CHECK(cudaMemcpyAsync(&res[4], &sc->zmax, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
        OZB_CHECK(cudaStreamSynchronize(st->stream));
    }
    ar.release(mk);
    *done = true;
    *nB_out = res[1];
    const int c = (res[4] < 1 ? 1 : res[4]) + 1;  // count rule, src/cpu/ozblas_split.cpp:272-289
    *nA_out = m > 0 ? (c < maxS ? c : maxS) : (maxS < 2 ? maxS : 2);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
