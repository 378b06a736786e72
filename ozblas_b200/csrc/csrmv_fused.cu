// csrmv_fused.cu — the plain-form CSRMV without materialised slices.
//
// The reference splits A row by row (src/cpu/ozblas_split.cpp:779-815), x with
// one global tau chain (:62-103), forms one CSRMM per A slice with a
// sequential fma chain per row (src/cpu/ozblas_blas_wrapper.cpp:231-255) and
// sums the pair products per row (src/cpu/ozblas_csrmv.cpp:100-160).  Here:
//
//  1. one pass over x: max, lowest set bit, Inf/NaN (chain.cuh);
//  2. x's chain is predicted (tau_{s+1} = tau_s + rho - 54) and its slice
//     count follows from the lowest set bit; a second pass over x proves the
//     prediction level by level.  If it does not hold, or x needs more than
//     8 levels, the main kernel writes nothing and the caller runs the
//     general path;
//  3. one thread per row: the row's own tau chain (rho from its nnz, sigma
//     divided by the CG's splitShift) is exact per row, so it is computed in
//     place; x's slices at the gathered columns come from the proven chain;
//     every pair product is the CPU's sequential fma chain in storage order,
//     summed in (ik, ia) order (FSum) or NearSum-ed.  A block stages its
//     val/colind range in shared memory with coalesced loads and issues all
//     gathers of x before using them.  Rows longer than 8 or needing more
//     levels than the kernel holds are deferred to a per-row general kernel.
//
// Pairs whose A slice is beyond a row's own exact split are zero slices in
// the reference; they add +0 to the ordered sum and nothing to NearSum, so
// skipping them leaves the bits unchanged.  fastMode must be 0 (the caller
// uses the general path otherwise).
#include "fused.h"
#include "sum.cuh"

namespace ozb {

// Max, lowest set bit and Inf/NaN of v into vs[index] (the first pass of a
// vector's predicted chain).
template <bool ALIGNED>
__global__ void __launch_bounds__(256) k_vec_stats(int n, const double *__restrict__ x, VecStats *vs, int index) {
    __shared__ double red[8];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double mx = 0.0;
    int lx = 0, bx = 0;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ALIGNED) {
        const int64_t np = (int64_t)n >> 1;
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        for (; i < np; i += stride) {
            const double2 a = x2[i];
            scan_elem(a.x, mx, lx, bx);
            scan_elem(a.y, mx, lx, bx);
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) scan_elem(x[n - 1], mx, lx, bx);
    } else {
        for (; i < n; i += stride) scan_elem(x[i], mx, lx, bx);
    }
    scan_commit(vs, index, mx, lx, bx, red);
}

template <int G, int T>
__device__ __forceinline__ unsigned proof_body(double v, const TreePlan &pl) {
    double q[T + 1];
    cut_tree<G, T>(v, pl.sig[0], q);
    unsigned hw[kCsrLv];
#pragma unroll
    for (int s = 0; s < T; s++) hw[s] = abs_hiword(q[s + 1]);
    return prove_levels<T>(hw, pl.hb[0], pl.need[0]);
}

// Proof of x's predicted chain.  One witness per level suffices, so a warp
// stops as soon as it has proven every level the plan needs (and all warps stop
// once any warp has); only an unproven chain reads the whole vector.  The last
// block publishes validity, slice count and sigmas.
template <int G>
__global__ void __launch_bounds__(256) k_csr_proof(int n, const double *__restrict__ x, int rho, int maxS,
                                                   CsrScratch *sc, const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    __shared__ TreePlan pl;
    __shared__ int last;
    const int t = threadIdx.x;
    plan_in_block(&sc->vs, rho, maxS, true, pl);
    __syncthreads();
    const unsigned need = pl.need[0];
    if (pl.valid && need) {  // uniform
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        const int64_t iw = (int64_t)blockIdx.x * blockDim.x + (t & ~31);  // the warp's first element
        const int64_t K = iw < n ? ((int64_t)n - iw + stride - 1) / stride : 0;
        int64_t i = (int64_t)blockIdx.x * blockDim.x + t;
        unsigned got = 0u;
        for (int64_t k = 0; k < K; k++, i += stride) {
            if ((got & need) == need || (k & 7) == 7 && __ldcg(&sc->proven) == need) break;  // uniform per warp
            const double v = i < n ? x[i] : 0.0;
            int T = plan_depth(pl, 0, __reduce_min_sync(0xffffffffu, exp_key(v)));
            if (T > pl.L - 1) T = pl.L - 1;
            switch (T) {
                case 0: break;
                case 1: got |= proof_body<G, 1>(v, pl); break;
                case 2: got |= proof_body<G, 2>(v, pl); break;
                case 3: got |= proof_body<G, 3>(v, pl); break;
                case 4: got |= proof_body<G, 4>(v, pl); break;
                case 5: got |= proof_body<G, 5>(v, pl); break;
                case 6: got |= proof_body<G, 6>(v, pl); break;
                default: got |= proof_body<G, 7>(v, pl); break;
            }
        }
        if ((t & 31) == 0 && got) atomicOr(&sc->proven, got & need);
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || t != 0) return;
    __threadfence();
    const int valid = pl.valid && (__ldcg(&sc->proven) & need) == need;
    for (int s = 0; s < kCsrLv; s++) sc->sigma[s] = pl.sig[0][s];
    sc->nB = pl.ns[0];
    sc->xcomplete = valid && pl.z[0] <= pl.ns[0] - 1;
    sc->rn_declined = 0;
    sc->valid = valid;
    // leave the proof and the statistics zeroed for the next use (every block
    // has read the statistics: the ticket comes after)
    sc->proven = 0u;
    sc->ticket = 0u;
    sc->vs = VecStats{};
}

// Visit the pairs (ia < na, ib < nb) of a row in summation order: ik
// ascending, ia ascending (compile-time indices, so P stays in registers).
template <int NA, typename F>
__device__ __forceinline__ void for_row_pairs(int na, int nb, F f) {
#pragma unroll
    for (int ik = 0; ik < NA + kCsrLv - 1; ik++)
#pragma unroll
        for (int ia = 0; ia < NA; ia++) {
            const int ib = ik - ia;
            if (ib >= 0 && ib < kCsrLv)
                if (ia < na && ib < nb) f(ia, ib);
        }
}

// NearSum (src/cpu/ozblas_sum.cpp:10-112, as in sum.cuh) over the row's pair
// products held in registers; same term order as sum.cuh's callers.
template <int NA>
__device__ __forceinline__ void ns_transform_row(double (&v)[NA][kCsrLv], int na, int nb, int n, double rho,
                                                 double &tau1, double &tau2) {
    const int emin = -1022, epse = 53;
    double mu = 0.0;
    for_row_pairs<NA>(na, nb, [&](int a, int b) {
        const double t = fabs(v[a][b]);
        mu = (mu > t) ? mu : t;
    });
    if (n == 0 || mu == 0.) {
        tau1 = rho;
        tau2 = 0.;
        return;
    }
    const int M = ceil_log2_int((uint32_t)(n + 2));
    double sigma = pow2(M + tau_rule(mu));
    double t = rho;
    for (;;) {
        double tau = 0.;
        for_row_pairs<NA>(na, nb, [&](int a, int b) {
            const double tmp = (sigma + v[a][b]) - sigma;
            v[a][b] -= tmp;
            tau += tmp;
        });
        tau1 = t + tau;
        if ((sigma <= pow2(emin)) || (fabs(tau1) >= pow2(2 * M + 1 - epse) * sigma)) {
            tau2 = tau - (tau1 - t);
            return;
        }
        sigma = pow2(M - epse) * sigma;
        t = tau1;
    }
}

template <int NA>
__device__ __forceinline__ void ns_transformk_row(double (&v)[NA][kCsrLv], int na, int nb, int n, double rho,
                                                  double &res, double &r) {
    double tmp = 0., tau1, tau2;
    ns_transform_row<NA>(v, na, nb, n, rho, tau1, tau2);
    for_row_pairs<NA>(na, nb, [&](int a, int b) { tmp += v[a][b]; });
    res = tau1 + (tau2 + tmp);
    r = tau2 - (res - tau1);
}

template <int NA>
__device__ __forceinline__ double nearsum_row(double (&v)[NA][kCsrLv], int na, int nb) {
    {
        CrSum cs;
        for_row_pairs<NA>(na, nb, [&](int a, int b) { cs.add(v[a][b]); });
        double out;
        if (cs.finish(out)) return out;
    }
    const int n = na * nb;
    const double eps = pow2(-53);
    double res, r, delta, r2, res2, mu, delta2, tmp;
    ns_transformk_row<NA>(v, na, nb, n, 0., res, r);
    ns_transformk_row<NA>(v, na, nb, n, r, delta, r2);
    if (delta == 0) return res;
    res2 = res + sign1(delta) * eps * fabs(res);
    if (res2 == res) {
        mu = sign1(delta) * eps * fabs(res);
        res2 = res + 2. * sign1(delta) * eps * fabs(res);
    } else {
        mu = (res2 - res) / 2.;
    }
    if (fabs(delta) < fabs(mu)) return res;
    if (fabs(delta) > fabs(mu)) return res2;
    ns_transformk_row<NA>(v, na, nb, n, r2, delta2, tmp);
    if (delta2 == 0) return res + mu;
    if (sign1(delta2) == sign1(mu)) return res2;
    return res;
}

// The row's own chain (src/cpu/ozblas_split.cpp:779-815, sigma / shift) over
// its entries a[] (zero padded to kCsrRowMax), at most NA levels: the sigmas,
// the level count na and the first zero-remainder level z.  Returns false
// when the row needs more than NA levels (and nSplitMax allows more).
template <int NA>
__device__ __forceinline__ bool row_chain(const double (&a)[kCsrRowMax], int len, int shift, int epsmode, int maxS,
                                          double (&sigA)[NA], int &na, int &z) {
    na = 0;
    z = 0;
#pragma unroll
    for (int s = 0; s < NA; s++) sigA[s] = 0.0;
    if (len <= 0) return true;
    const int rho = rho_rule(len, epsmode);
    double rr[kCsrRowMax];
    double mx = 0.0;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        rr[e] = a[e];
        mx = ref_max(mx, fabs(a[e]));
    }
    z = maxS;
    bool fin = false;
#pragma unroll
    for (int s = 0; s < NA; s++) {
        if (!fin && s < maxS) {
            const double sg = shift_sigma(0.75 * pow2(rho + tau_rule(mx)), shift);
            sigA[s] = sg;
            double nm = 0.0;
#pragma unroll
            for (int e = 0; e < kCsrRowMax; e++) {
                const double sl = (rr[e] + sg) - sg;
                rr[e] = rr[e] - sl;
                nm = ref_max(nm, fabs(rr[e]));
            }
            na = s + 1;
            mx = nm;
            if (nm == 0.0) {
                z = s;
                fin = true;
            }
        }
    }
    return !(mx != 0.0 && na < maxS);
}

// The rows the row kernel defers (more than kCsrRowMax entries, or more than
// NA levels), listed once for a matrix that is multiplied many times.
template <int NA>
__global__ void __launch_bounds__(128) k_csr_slow_rows(int m, const double *__restrict__ val,
                                                       const int *__restrict__ rowptr, int shift, int epsmode,
                                                       int maxS, int *__restrict__ list, int *__restrict__ count) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int lo = rowptr[row], len = rowptr[row + 1] - lo;
    bool defer = len > kCsrRowMax;
    if (!defer) {
        double a[kCsrRowMax];
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) a[e] = e < len ? val[lo + e] : 0.0;
        double sigA[NA];
        int na, z;
        defer = !row_chain<NA>(a, len, shift, epsmode, maxS, sigA, na, z);
    }
    if (defer) list[atomicAdd(count, 1)] = row;
}

int csr_slow_rows_launch(cudaStream_t s, int m, const double *val, const int *rowptr, int shift, int epsmode,
                         int maxS, int na_hint, int *list, int *count) {
    if (m <= 0) return CUOZBLAS_STATUS_SUCCESS;
    if (na_hint > 0 && na_hint <= 2)
        k_csr_slow_rows<2><<<(m + 127) / 128, 128, 0, s>>>(m, val, rowptr, shift, epsmode, maxS, list, count);
    else if (na_hint > 4)
        k_csr_slow_rows<6><<<(m + 127) / 128, 128, 0, s>>>(m, val, rowptr, shift, epsmode, maxS, list, count);
    else
        k_csr_slow_rows<4><<<(m + 127) / 128, 128, 0, s>>>(m, val, rowptr, shift, epsmode, maxS, list, count);
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

// One thread per row, everything in registers: each row's tau chain runs
// over its (at most kCsrRowMax) entries, keeping only the sigmas, then every
// entry is re-cut with them while x's slices at its column come from the
// proven chain; the pair products P[ia][ib] are the CPU's sequential fma
// chains in storage order.  Rows with more entries, or needing more than NA
// levels, go to the slow list.
template <int NA, int NB, int GX>
__device__ __forceinline__ void row_products(const double (&a)[kCsrRowMax], const double (&xv)[kCsrRowMax], int len,
                                             int na, const double (&sigA)[NA], const double *xsig,
                                             double (&P)[NA][kCsrLv]) {
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        if (e < len) {
            double sa[NA];
            double r = a[e];
#pragma unroll
            for (int s = 0; s < NA; s++) {
                sa[s] = 0.0;
                if (s < na) {
                    const double sl = (r + sigA[s]) - sigA[s];
                    r = r - sl;
                    sa[s] = sl;
                }
            }
            double sx[NB];
            cut_tree<GX, NB - 1>(xv[e], xsig, sx);
#pragma unroll
            for (int ia = 0; ia < NA; ia++)
                if (ia < na)
#pragma unroll
                    for (int ib = 0; ib < NB; ib++) P[ia][ib] = fma(sa[ia], sx[ib], P[ia][ib]);
        }
    }
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
                                                    double *__restrict__ terms, VecStats *__restrict__ ystats,
                                                    int ystats_index, const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform
    if (!sc->valid) return;          // uniform: x's chain is not proven
    __shared__ double red[4];
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    double ynew = 0.0;
    const bool wrote = slot < nrows;
    if (wrote) {
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
                sa[s] = shift_sigma(0.75 * pow2(rho + tau_rule(mx)), shift);
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
        ynew = fma(alpha, tsum, beta * y[row]);
        y[row] = ynew;
    }
    if (ystats) {
        double mx = 0.0;
        int lsb = 0, bad = 0;
        if (wrote) scan_elem(ynew, mx, lsb, bad);
        scan_commit(ystats, ystats_index, mx, lsb, bad, red);
    }
}

// Persistent, software-pipelined form of the row kernel (same arithmetic per
// row).  A CTA walks tiles of kCsrThreads rows; while it computes tile j from
// one shared-memory slot, cp.async fills the other with tile j+1: its val and
// colind ranges and old y during the row chains, then the gathers of x at its
// columns during the products, and the row pointers of tile j+2.  Tiles whose
// entries do not fit the slot are read from global memory directly.
struct CsrSlot {
    int rp[kCsrThreads + 4];
    double yold[kCsrThreads];
    double val[kCsrThreads * kCsrRowMax];
    double xg[kCsrThreads * kCsrRowMax];
    int col[kCsrThreads * kCsrRowMax];
};

template <int SUM_MODE, int NA, int GX>
__global__ void __launch_bounds__(kCsrThreads, NA > 4 ? 2 : 4)
    k_csrmv_pipe(int m, int n, const double *__restrict__ val, const int *__restrict__ colind,
                 const int *__restrict__ rowptr, const double *__restrict__ x, int shift, int epsmode, int maxS,
                 double alpha, double beta, double *__restrict__ y, CsrScratch *__restrict__ sc,
                 int *__restrict__ slow_rows, int append_slow, VecStats *__restrict__ ystats, int ystats_index,
                 const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    constexpr int kStage = kCsrThreads * kCsrRowMax;
    __shared__ CsrSlot slot[2];
    __shared__ double xs_sigma[kCsrLv];
    __shared__ double red[kCsrThreads / 32];
    const int t = threadIdx.x;
    const int ntiles = (m + kCsrThreads - 1) / kCsrThreads;
    if (t < kCsrLv) xs_sigma[t] = sc->sigma[t];
    const int valid = sc->valid;
    const int nB = sc->nB;
    __syncthreads();
    if (!valid) return;  // uniform: the caller runs the general path
    int tile = blockIdx.x;
    if (tile >= ntiles) return;  // uniform

    auto rows_of = [&](int tl) { return (m - tl * kCsrThreads < kCsrThreads) ? m - tl * kCsrThreads : kCsrThreads; };
    auto issue_rp = [&](int tl, CsrSlot &S) {
        const int r0 = tl * kCsrThreads, nrow = rows_of(tl);
        if (t < nrow) cp_async4(&S.rp[t], rowptr + r0 + t);
        if (t == 0) cp_async4(&S.rp[nrow], rowptr + r0 + nrow);
    };
    auto issue_vals = [&](int tl, CsrSlot &S) {  // needs S.rp
        const int r0 = tl * kCsrThreads, nrow = rows_of(tl);
        const int p0 = S.rp[0], cnt = S.rp[nrow] - p0;
        if (t < nrow) cp_async8(&S.yold[t], y + r0 + t);
        if (cnt <= kStage)
            for (int i = t; i < cnt; i += kCsrThreads) {
                cp_async8(&S.val[i], val + p0 + i);
                cp_async4(&S.col[i], colind + p0 + i);
            }
    };
    auto issue_gathers = [&](int tl, CsrSlot &S) {  // needs S.col
        const int nrow = rows_of(tl);
        const int cnt = S.rp[nrow] - S.rp[0];
        if (cnt <= kStage && n > 0)
            for (int i = t; i < cnt; i += kCsrThreads) cp_async8(&S.xg[i], x + S.col[i]);
    };

    // prologue: the first tile complete in slot 0, the next tile's row pointers in slot 1
    issue_rp(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_vals(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_gathers(tile, slot[0]);
    if (tile + (int)gridDim.x < ntiles) issue_rp(tile + gridDim.x, slot[1]);
    cp_async_commit();

    double smx = 0.0;  // statistics of the written y, folded once at the end
    int slsb = 0, sbad = 0, zmax = 0;
    for (int j = 0; tile < ntiles; j++, tile += gridDim.x) {
        CsrSlot &S = slot[j & 1], &N = slot[(j & 1) ^ 1];
        const int nxt = tile + gridDim.x;
        cp_async_wait_all();  // this tile's gathers and the next tile's row pointers
        __syncthreads();
        if (nxt < ntiles) issue_vals(nxt, N);
        cp_async_commit();
        // ---- phase 1: this tile's entries and row chains
        const int r0 = tile * kCsrThreads, nrow = rows_of(tile);
        const int row = r0 + t;
        const bool active = t < nrow;
        const int p0 = S.rp[0], cnt = S.rp[nrow] - p0;
        const bool staged = cnt <= kStage;
        int lo = p0, len = 0;
        if (active) {
            lo = S.rp[t];
            len = S.rp[t + 1] - lo;
        }
        bool defer = active && len > kCsrRowMax;
        const bool work = active && !defer;
        const double yold = active ? S.yold[t] : 0.0;
        double a[kCsrRowMax];
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) {
            const bool in = work && e < len;
            double v = 0.0;
            if (staged)
                v = S.val[min(lo - p0 + e, kStage - 1)];
            else if (in)
                v = val[lo + e];
            a[e] = in ? v : 0.0;
        }
        double sigA[NA];
        int na = 0, z = 0;
        if (work && !row_chain<NA>(a, len, shift, epsmode, maxS, sigA, na, z)) defer = true;
        if (defer && append_slow) slow_rows[atomicAdd(&sc->nslow, 1)] = row;
        if (work && !defer) zmax = z > zmax ? z : zmax;
        cp_async_wait_all();  // the next tile's val and colind
        __syncthreads();
        if (nxt < ntiles) issue_gathers(nxt, N);
        if (nxt + (int)gridDim.x < ntiles) issue_rp(nxt + gridDim.x, S);  // S.rp is no longer read
        cp_async_commit();
        // ---- phase 2: products and sums
        if (work && !defer) {
            double xv[kCsrRowMax];
#pragma unroll
            for (int e = 0; e < kCsrRowMax; e++) {
                double v = 0.0;
                if (e < len && n > 0) v = staged ? S.xg[lo - p0 + e] : x[colind[lo + e]];
                xv[e] = v;
            }
            double P[NA][kCsrLv];
#pragma unroll
            for (int i = 0; i < NA; i++)
#pragma unroll
                for (int jj = 0; jj < kCsrLv; jj++) P[i][jj] = 0.0;
            switch (nB) {  // uniform
                case 1: row_products<NA, 1, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 2: row_products<NA, 2, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 3: row_products<NA, 3, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 4: row_products<NA, 4, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 5: row_products<NA, 5, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 6: row_products<NA, 6, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                case 7: row_products<NA, 7, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
                default: row_products<NA, 8, GX>(a, xv, len, na, sigA, xs_sigma, P); break;
            }
            double tsum = 0.0;
            if (SUM_MODE == 1)
                tsum = nearsum_row<NA>(P, na, nB);
            else
                for_row_pairs<NA>(na, nB, [&](int ia, int ib) { tsum += P[ia][ib]; });
            const double ynew = fma(alpha, tsum, beta * yold);
            y[row] = ynew;
            if (ystats) scan_elem(ynew, smx, slsb, sbad);
        }
    }
    cp_async_wait_all();
    {
        const int zw = __reduce_max_sync(0xffffffffu, zmax);
        if ((t & 31) == 0 && zw > 0) atomicMax(&sc->zmax, zw);
    }
    if (ystats) scan_commit(ystats, ystats_index, smx, slsb, sbad, red);
}

// ---------------------------------------------------------------------------
// Lean row kernel (rows of at most NA <= 4 levels).  Same arithmetic per row
// as k_csrmv_pipe, with less work around it:
//  * each row is staged zero padded into kCsrRowMax slots (cp.async with zero
//    fill), so a thread reads its entries and gathered x values with 16-byte
//    shared loads and needs no masks;
//  * the row chain keeps its slices (the products use them directly instead
//    of cutting every entry again);
//  * the row max is taken over the high words of |r| (one integer max per
//    entry); the full value is looked at only when the high word leaves tau
//    open (an exact power of two, zero, subnormal) — rows with Inf or NaN
//    entries go to the general per-row kernel;
//  * the pair products are held for exactly NA x nB pairs, so FSum and the
//    certified correctly rounded sum run without guards (pairs beyond a
//    row's own levels are +0 and change neither sum).
struct LeanSlot {
    int rp[kCsrThreads + 4];
    double yold[kCsrThreads];
    double val[kCsrThreads * kCsrRowMax];  // entry e of row t at lean_pos(t, e); zero padded
    double xg[kCsrThreads * kCsrRowMax];   // x at the entry's column, same positions
    int col[kCsrThreads * kCsrRowMax];     // row t's columns at t * kCsrRowMax + e
};
static_assert(kCsrRowMax == 8, "lean rows hold 8 entries as four 16-byte pairs");

// Entry e of row t: the row's four 16-byte pairs are rotated by (t >> 1) & 3
// so that the 16-byte reads of eight consecutive rows hit distinct banks.
__device__ __forceinline__ int lean_pos(int t, int e) {
    return t * kCsrRowMax + ((((e >> 1) ^ (t >> 1)) & 3) << 1) + (e & 1);
}

__device__ __forceinline__ void lean_read(const double *base, int t, double (&v)[kCsrRowMax]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const double2 p = *reinterpret_cast<const double2 *>(base + t * kCsrRowMax + (((i ^ (t >> 1)) & 3) << 1));
        v[2 * i] = p.x;
        v[2 * i + 1] = p.y;
    }
}

__device__ __forceinline__ unsigned hi_abs(double v) { return (unsigned)__double2hiint(v) & 0x7fffffffu; }

// tau_rule(max_e |r_e|) given mh, the max of the entries' |high words| (all
// entries finite): a normal max whose high word has mantissa bits set lies
// above every tau threshold of its binade, so tau = exponent + 1.
__device__ __forceinline__ int lean_tau(unsigned mh, const double (&r)[kCsrRowMax]) {
    if ((mh & 0xfffffu) != 0u && mh >= 0x00100000u) return (int)(mh >> 20) - 1022;
    double mx = 0.0;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) mx = fmax(mx, fabs(r[e]));
    return tau_rule(mx);
}

// The row's own chain (src/cpu/ozblas_split.cpp:779-815) as row_chain
// computes it, keeping the slices.  Returns false when the row needs more
// than NA levels (and nSplitMax allows more) or holds Inf / NaN.
template <int NA>
__device__ __forceinline__ bool lean_chain(double (&r)[kCsrRowMax], int len, int shift, int epsmode, int maxS,
                                           double (&sa)[kCsrRowMax][NA], int &na, int &z) {
    na = 0;
    z = 0;
    unsigned mh = 0u;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) mh = max(mh, hi_abs(r[e]));
    if (mh >= 0x7ff00000u) return false;  // Inf or NaN: the general kernel
    const int rho = rho_rule(len > 0 ? len : 1, epsmode);
    z = len > 0 ? maxS : 0;
    bool fin = len <= 0;
    double sg = 1.0;
    // Levels after the first zero remainder cut zeros into +0 slices (with the
    // last sigma), which is what the products need there; only levels beyond
    // nSplitMax are set to zero explicitly.
#pragma unroll
    for (int s = 0; s < NA; s++) {
        if (s < maxS) {  // uniform
            if (!fin) sg = shift_sigma(0.75 * pow2(rho + lean_tau(mh, r)), shift);
            unsigned nh = 0u;
#pragma unroll
            for (int e = 0; e < kCsrRowMax; e++) {
                const double sl = (r[e] + sg) - sg;
                r[e] = r[e] - sl;
                sa[e][s] = sl;
                nh = max(nh, hi_abs(r[e]));
            }
            if (!fin) {
                na = s + 1;
                bool zero = false;
                if (nh == 0u) {
                    unsigned lo = 0u;
#pragma unroll
                    for (int e = 0; e < kCsrRowMax; e++) lo |= (unsigned)__double2loint(r[e]);
                    zero = lo == 0u;
                }
                if (zero) {
                    z = s;
                    fin = true;
                }
            }
            mh = nh;
        } else {
#pragma unroll
            for (int e = 0; e < kCsrRowMax; e++) sa[e][s] = 0.0;
        }
    }
    return fin || na >= maxS;
}

template <int SUM_MODE, int NA, int NB, int GX>
__device__ __forceinline__ double lean_products(const double (&sa)[kCsrRowMax][NA], const double (&xv)[kCsrRowMax],
                                                int len, int na, const double *xsig) {
    double P[NA][NB];
#pragma unroll
    for (int i = 0; i < NA; i++)
#pragma unroll
        for (int j = 0; j < NB; j++) P[i][j] = 0.0;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        if (e < len) {
            double sx[NB];
            cut_tree<GX, NB - 1>(xv[e], xsig, sx);
#pragma unroll
            for (int ia = 0; ia < NA; ia++)
#pragma unroll
                for (int ib = 0; ib < NB; ib++) P[ia][ib] = fma(sa[e][ia], sx[ib], P[ia][ib]);
        }
    }
    if (SUM_MODE == 0) {
        double t = 0.0;
#pragma unroll
        for (int ik = 0; ik < NA + NB - 1; ik++)
#pragma unroll
            for (int ia = 0; ia < NA; ia++)
                if (ik - ia >= 0 && ik - ia < NB) t += P[ia][ik - ia];
        return t;
    } else {
        CrSum cs;
#pragma unroll
        for (int ik = 0; ik < NA + NB - 1; ik++)
#pragma unroll
            for (int ia = 0; ia < NA; ia++)
                if (ik - ia >= 0 && ik - ia < NB) cs.add(P[ia][ik - ia]);
        double out;
        if (cs.finish(out)) return out;
        double Q[NA][kCsrLv];
#pragma unroll
        for (int i = 0; i < NA; i++)
#pragma unroll
            for (int j = 0; j < kCsrLv; j++) Q[i][j] = j < NB ? P[i][j] : 0.0;
        return nearsum_row<NA>(Q, na, NB);
    }
}

template <int SUM_MODE, int NA, int GX>
__global__ void __launch_bounds__(kCsrThreads, NA >= 4 ? 3 : 4)
    k_csrmv_lean(int m, int n, const double *__restrict__ val, const int *__restrict__ colind,
                 const int *__restrict__ rowptr, const double *__restrict__ x, int shift, int epsmode, int maxS,
                 double alpha, double beta, double *__restrict__ y, CsrScratch *__restrict__ sc,
                 int *__restrict__ slow_rows, int append_slow, VecStats *__restrict__ ystats, int ystats_index,
                 const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    __shared__ __align__(16) LeanSlot slot[2];
    __shared__ double xs_sigma[kCsrLv];
    __shared__ double red[kCsrThreads / 32];
    const int t = threadIdx.x;
    const int ntiles = (m + kCsrThreads - 1) / kCsrThreads;
    if (t < kCsrLv) xs_sigma[t] = sc->sigma[t];
    const int valid = sc->valid;
    const int nB = sc->nB;
    __syncthreads();
    if (!valid) return;  // uniform: the caller runs the general path
    int tile = blockIdx.x;
    if (tile >= ntiles) return;  // uniform

    auto rows_of = [&](int tl) { return (m - tl * kCsrThreads < kCsrThreads) ? m - tl * kCsrThreads : kCsrThreads; };
    auto issue_rp = [&](int tl, LeanSlot &S) {
        const int r0 = tl * kCsrThreads, nrow = rows_of(tl);
        if (t < nrow) cp_async4(&S.rp[t], rowptr + r0 + t);
        if (t == 0) cp_async4(&S.rp[nrow], rowptr + r0 + nrow);
    };
    auto issue_vals = [&](int tl, LeanSlot &S) {  // needs S.rp
        const int r0 = tl * kCsrThreads;
        if (t >= rows_of(tl)) return;
        const double *dummy = y + r0 + t;  // a valid address for copies that read nothing
        cp_async8(&S.yold[t], dummy);
        const int lo = S.rp[t], len = S.rp[t + 1] - lo;
        if (len > kCsrRowMax) return;
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) {
            const bool in = e < len;
            cp_async8_zfill(&S.val[lean_pos(t, e)], in ? (const void *)(val + lo + e) : (const void *)dummy,
                            in ? 8u : 0u);
            cp_async4_zfill(&S.col[t * kCsrRowMax + e], in ? (const void *)(colind + lo + e) : (const void *)dummy,
                            in ? 4u : 0u);
        }
    };
    auto issue_gathers = [&](int tl, LeanSlot &S) {  // needs S.rp and S.col
        const int r0 = tl * kCsrThreads;
        if (t >= rows_of(tl)) return;
        const double *dummy = y + r0 + t;
        const int lo = S.rp[t], len = S.rp[t + 1] - lo;
        if (len > kCsrRowMax) return;
        const int4 c0 = *reinterpret_cast<const int4 *>(&S.col[t * kCsrRowMax]);
        const int4 c1 = *reinterpret_cast<const int4 *>(&S.col[t * kCsrRowMax + 4]);
        const int cc[kCsrRowMax] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) {
            const bool in = e < len && n > 0;
            cp_async8_zfill(&S.xg[lean_pos(t, e)], in ? (const void *)(x + cc[e]) : (const void *)dummy,
                            in ? 8u : 0u);
        }
    };

    // prologue: the first tile complete in slot 0, the next tile's row pointers in slot 1
    issue_rp(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_vals(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_gathers(tile, slot[0]);
    if (tile + (int)gridDim.x < ntiles) issue_rp(tile + gridDim.x, slot[1]);
    cp_async_commit();

    double smx = 0.0;  // statistics of the written y, folded once at the end
    int slsb = 0, sbad = 0, zmax = 0;
    for (int j = 0; tile < ntiles; j++, tile += gridDim.x) {
        LeanSlot &S = slot[j & 1], &N = slot[(j & 1) ^ 1];
        const int nxt = tile + gridDim.x;
        cp_async_wait_all();  // this tile's gathers and the next tile's row pointers
        __syncthreads();
        if (nxt < ntiles) issue_vals(nxt, N);
        cp_async_commit();
        // ---- phase 1: this tile's row chains
        const int r0 = tile * kCsrThreads, nrow = rows_of(tile);
        const int row = r0 + t;
        const bool active = t < nrow;
        int len = 0;
        if (active) len = S.rp[t + 1] - S.rp[t];
        bool defer = active && len > kCsrRowMax;
        const bool work = active && !defer;
        const double yold = active ? S.yold[t] : 0.0;
        double sa[kCsrRowMax][NA];
        int na = 0, z = 0;
        if (work) {
            double r[kCsrRowMax];
            lean_read(S.val, t, r);
            if (!lean_chain<NA>(r, len, shift, epsmode, maxS, sa, na, z)) defer = true;
        }
        if (defer && append_slow) slow_rows[atomicAdd(&sc->nslow, 1)] = row;
        if (work && !defer) zmax = z > zmax ? z : zmax;
        cp_async_wait_all();  // the next tile's val and colind
        __syncthreads();
        if (nxt < ntiles) issue_gathers(nxt, N);
        if (nxt + (int)gridDim.x < ntiles) issue_rp(nxt + gridDim.x, S);  // S.rp is no longer read
        cp_async_commit();
        // ---- phase 2: products and sums
        if (work && !defer) {
            double xv[kCsrRowMax];
            lean_read(S.xg, t, xv);
            double tsum;
            switch (nB) {  // uniform
                case 1: tsum = lean_products<SUM_MODE, NA, 1, GX>(sa, xv, len, na, xs_sigma); break;
                case 2: tsum = lean_products<SUM_MODE, NA, 2, GX>(sa, xv, len, na, xs_sigma); break;
                case 3: tsum = lean_products<SUM_MODE, NA, 3, GX>(sa, xv, len, na, xs_sigma); break;
                case 4: tsum = lean_products<SUM_MODE, NA, 4, GX>(sa, xv, len, na, xs_sigma); break;
                case 5: tsum = lean_products<SUM_MODE, NA, 5, GX>(sa, xv, len, na, xs_sigma); break;
                case 6: tsum = lean_products<SUM_MODE, NA, 6, GX>(sa, xv, len, na, xs_sigma); break;
                case 7: tsum = lean_products<SUM_MODE, NA, 7, GX>(sa, xv, len, na, xs_sigma); break;
                default: tsum = lean_products<SUM_MODE, NA, 8, GX>(sa, xv, len, na, xs_sigma); break;
            }
            const double ynew = fma(alpha, tsum, beta * yold);
            y[row] = ynew;
            if (ystats) scan_elem(ynew, smx, slsb, sbad);
        }
    }
    cp_async_wait_all();
    {
        const int zw = __reduce_max_sync(0xffffffffu, zmax);
        if ((t & 31) == 0 && zw > 0) atomicMax(&sc->zmax, zw);
    }
    if (ystats) scan_commit(ystats, ystats_index, smx, slsb, sbad, red);
}

// ---------------------------------------------------------------------------
// NearSum rows, correctly rounded.  With sumMode 1 the reference's row result
// is NearSum over the row's slice-pair products (src/cpu/ozblas_csrmv.cpp:
// 100-160, src/cpu/ozblas_sum.cpp:10-112).  Each pair product is exact when
// its slices' bits fit: an A slice is at most 2^(53 - rho_A) grid units
// (times the shift), an x slice at most 2^(53 - rho_x), so a row of len
// entries sums to at most len 2^(106 - rho_A - rho_x + log2 shift) units of
// the product grid, exact below 2^53.  With both splits complete the pair
// products then add up to the exact row dot product, and NearSum returns its
// correct rounding.  So a row that meets both conditions is computed as
// RN(sum_j a_j x_j) directly: TwoProd of each entry gives exact terms, the
// certified TwoSum cascade (crsum.h) rounds them, NearSum when it cannot
// certify.  Rows that do not meet them (or whose products leave the range
// TwoProd keeps exact) are deferred to the per-row general kernel.
// ---------------------------------------------------------------------------
constexpr int kCsrSlowChunk = 8192;  // rows per launch of the per-row general kernel

__device__ __forceinline__ bool rn_row_dot(const double (&v)[kCsrRowMax], const double (&xv)[kCsrRowMax], int len,
                                           double &out) {
    double t[2 * kCsrRowMax];
    CrSum cs;
    bool ok = true;
#pragma unroll
    for (int e = 0; e < kCsrRowMax; e++) {
        const double p = e < len ? __dmul_rn(v[e], xv[e]) : 0.0;
        const double er = e < len ? __fma_rn(v[e], xv[e], -p) : 0.0;
        const double ap = fabs(p);
        if (e < len && ((ap < 0x1p-969 && v[e] != 0.0 && xv[e] != 0.0) || !(ap < 0x1p1023))) ok = false;
        t[2 * e] = p;
        t[2 * e + 1] = er;
        cs.add(p);
        cs.add(er);
    }
    if (!ok) return false;
    if (cs.finish(out)) return true;
    out = nearsum(2 * kCsrRowMax, t, 1);
    return true;
}

__host__ __device__ __forceinline__ int ceil_log2_small(int v) {
    int c = 0;
    while ((1 << c) < v) c++;
    return c;
}

template <int NA>
__global__ void __launch_bounds__(kCsrThreads, 4)
    k_csrmv_rn(int m, int n, const double *__restrict__ val, const int *__restrict__ colind,
               const int *__restrict__ rowptr, const double *__restrict__ x, int shift, int lg_shift, int rho_x,
               int epsmode, int maxS, double alpha, double beta, double *__restrict__ y, CsrScratch *__restrict__ sc,
               int *__restrict__ slow_rows, int append_slow, VecStats *__restrict__ ystats, int ystats_index,
               const VecStats *__restrict__ xstats, const int *__restrict__ gate) {
    if (gate && *gate == 0) return;  // uniform: a captured solver step that is switched off
    __shared__ __align__(16) LeanSlot slot[2];
    __shared__ double red[kCsrThreads / 32];
    __shared__ int xok;
    const int t = threadIdx.x;
    const int ntiles = (m + kCsrThreads - 1) / kCsrThreads;
    // x's split must be complete: from the proof kernel (sc), or with `xstats`
    // (no proof ran) straight from x's statistics
    if (t == 0) {
        if (xstats) {
            VecStats vs;
            vs.mx[0] = __ldcg(&xstats->mx[0]);
            vs.lsb[0] = __ldcg(&xstats->lsb[0]);
            vs.bad[0] = __ldcg(&xstats->bad[0]);
            xok = split_complete(vs, 0, rho_x, maxS) ? 1 : 0;
        } else {
            xok = !sc->valid ? -1 : (sc->xcomplete ? 1 : 0);
        }
    }
    __syncthreads();
    if (xok < 0) return;  // uniform: the caller runs the general path
    if (xok == 0) {       // uniform: the lean kernel computes the slices instead
        if (blockIdx.x == 0 && t == 0) sc->rn_declined = 1;
        return;
    }
    int tile = blockIdx.x;
    if (tile >= ntiles) return;  // uniform

    auto rows_of = [&](int tl) { return (m - tl * kCsrThreads < kCsrThreads) ? m - tl * kCsrThreads : kCsrThreads; };
    auto issue_rp = [&](int tl, LeanSlot &S) {
        const int r0 = tl * kCsrThreads, nrow = rows_of(tl);
        if (t < nrow) cp_async4(&S.rp[t], rowptr + r0 + t);
        if (t == 0) cp_async4(&S.rp[nrow], rowptr + r0 + nrow);
    };
    auto issue_vals = [&](int tl, LeanSlot &S) {  // needs S.rp
        const int r0 = tl * kCsrThreads;
        if (t >= rows_of(tl)) return;
        const double *dummy = y + r0 + t;  // a valid address for copies that read nothing
        cp_async8(&S.yold[t], dummy);
        const int lo = S.rp[t], len = S.rp[t + 1] - lo;
        if (len > kCsrRowMax) return;
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) {
            const bool in = e < len;
            cp_async8_zfill(&S.val[lean_pos(t, e)], in ? (const void *)(val + lo + e) : (const void *)dummy,
                            in ? 8u : 0u);
            cp_async4_zfill(&S.col[t * kCsrRowMax + e], in ? (const void *)(colind + lo + e) : (const void *)dummy,
                            in ? 4u : 0u);
        }
    };
    auto issue_gathers = [&](int tl, LeanSlot &S) {  // needs S.rp and S.col
        const int r0 = tl * kCsrThreads;
        if (t >= rows_of(tl)) return;
        const double *dummy = y + r0 + t;
        const int lo = S.rp[t], len = S.rp[t + 1] - lo;
        if (len > kCsrRowMax) return;
        const int4 c0 = *reinterpret_cast<const int4 *>(&S.col[t * kCsrRowMax]);
        const int4 c1 = *reinterpret_cast<const int4 *>(&S.col[t * kCsrRowMax + 4]);
        const int cc[kCsrRowMax] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
        for (int e = 0; e < kCsrRowMax; e++) {
            const bool in = e < len && n > 0;
            cp_async8_zfill(&S.xg[lean_pos(t, e)], in ? (const void *)(x + cc[e]) : (const void *)dummy,
                            in ? 8u : 0u);
        }
    };

    issue_rp(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_vals(tile, slot[0]);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_gathers(tile, slot[0]);
    if (tile + (int)gridDim.x < ntiles) issue_rp(tile + gridDim.x, slot[1]);
    cp_async_commit();

    double smx = 0.0;
    int slsb = 0, sbad = 0, zmax = 0;
    for (int j = 0; tile < ntiles; j++, tile += gridDim.x) {
        LeanSlot &S = slot[j & 1], &N = slot[(j & 1) ^ 1];
        const int nxt = tile + gridDim.x;
        cp_async_wait_all();
        __syncthreads();
        if (nxt < ntiles) issue_vals(nxt, N);
        cp_async_commit();
        // ---- phase 1: the row's own split: complete, and exact slice products
        const int r0 = tile * kCsrThreads, nrow = rows_of(tile);
        const int row = r0 + t;
        const bool active = t < nrow;
        int len = 0;
        if (active) len = S.rp[t + 1] - S.rp[t];
        // `listed`: a row the slice kernel defers too (longer than 8, more than NA
        // levels, Inf / NaN); with a fixed list (append_slow = 0) its caller
        // computes it.  `defer`: a row this kernel cannot give the reference's
        // bits (incomplete split, possibly inexact slice products, TwoProd out of
        // range): appended, or with a fixed list the whole product is declined.
        bool listed = active && len > kCsrRowMax, defer = false;
        bool work = active && !listed;
        const double yold = active ? S.yold[t] : 0.0;
        if (work) {
            // len 2^(106 - rho_A - rho_x + log2 shift) < 2^53 in product-grid units
            if (len > 0 && ceil_log2_small(len) + 106 - rho_rule(len, epsmode) - rho_x + lg_shift > 53) defer = true;
            double r[kCsrRowMax], sa[kCsrRowMax][NA];
            lean_read(S.val, t, r);
            int na = 0, z = 0;
            if (!lean_chain<NA>(r, len, shift, epsmode, maxS, sa, na, z))
                listed = true;  // more levels than held, or Inf / NaN
            else if (len > 0 && z >= maxS)
                defer = true;   // an incomplete split
            if (!listed && !defer) zmax = z > zmax ? z : zmax;
        }
        cp_async_wait_all();
        __syncthreads();
        if (nxt < ntiles) issue_gathers(nxt, N);
        if (nxt + (int)gridDim.x < ntiles) issue_rp(nxt + gridDim.x, S);
        cp_async_commit();
        // ---- phase 2: the correctly rounded row dot
        work = work && !listed && !defer;
        if (work) {
            double v[kCsrRowMax], xv[kCsrRowMax], tsum = 0.0;
            lean_read(S.val, t, v);
            lean_read(S.xg, t, xv);
            if (rn_row_dot(v, xv, len, tsum)) {
                const double ynew = fma(alpha, tsum, beta * yold);
                y[row] = ynew;
                if (ystats) scan_elem(ynew, smx, slsb, sbad);
            } else {
                defer = true;
            }
        }
        if (append_slow) {
            if (listed || defer) slow_rows[atomicAdd(&sc->nslow, 1)] = row;
        } else if (defer) {
            sc->rn_declined = 1;
        }
    }
    cp_async_wait_all();
    {
        const int zw = __reduce_max_sync(0xffffffffu, zmax);
        if ((t & 31) == 0 && zw > 0) atomicMax(&sc->zmax, zw);
    }
    if (ystats) scan_commit(ystats, ystats_index, smx, slsb, sbad, red);
}

bool csr_rn_applies(const CsrmvArgs &a) {
    return a.sum_mode == 1 && a.epsmode == 0 && a.shift > 0 && (a.shift & (a.shift - 1)) == 0;
}

template <int NA>
static void launch_rn(const CsrmvArgs &a, cudaStream_t s, CsrScratch *sc, int *slow, int append, VecStats *ystats,
                      int ystats_index, const VecStats *xstats, const int *gate) {
    static std::atomic<int> per_sm{0};  // resident CTAs per SM (once per instantiation)
    int ps = per_sm.load();
    if (ps == 0) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_csrmv_rn<NA>, kCsrThreads, 0);
        ps = v > 0 ? v : 1;
        per_sm.store(ps);
    }
    const int rb = (a.m + kCsrThreads - 1) / kCsrThreads;
    const int cap = sm_count() * ps;
    const int grid = rb < cap ? rb : cap;
    const int lg_shift = 31 - __builtin_clz((unsigned)a.shift);
    const int rho_x = rho_rule(a.n > 0 ? a.n : 1, a.epsmode);
    k_csrmv_rn<NA><<<grid, kCsrThreads, 0, s>>>(a.m, a.n, a.val, a.colind, a.rowptr, a.x, a.shift, lg_shift, rho_x,
                                                 a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, slow, append, ystats,
                                                 ystats_index, xstats, gate);
}

int csr_rn_launch(cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int fixed_slow, VecStats *ystats,
                  int ystats_index, double *terms, const int *gate, const VecStats *xstats) {
    if (a.m <= 0) return CUOZBLAS_STATUS_SUCCESS;
    const int append = fixed_slow < 0 ? 1 : 0;
    // the levels per row held on chip match the slow-row list's (csr_slow_rows_launch)
    if (a.na_hint > 0 && a.na_hint <= 2)
        launch_rn<2>(a, s, sc, slow, append, ystats, ystats_index, xstats, gate);
    else if (a.na_hint > 4)
        launch_rn<6>(a, s, sc, slow, append, ystats, ystats_index, xstats, gate);
    else
        launch_rn<4>(a, s, sc, slow, append, ystats, ystats_index, xstats, gate);
    for (int c0 = 0; c0 < fixed_slow; c0 += kCsrSlowChunk) {  // the listed rows (general per-row kernel)
        const int nr = fixed_slow - c0 < kCsrSlowChunk ? fixed_slow - c0 : kCsrSlowChunk;
        k_csrmv_slow<1><<<(nr + 127) / 128, 128, 0, s>>>(nr, slow + c0, a.val, a.colind, a.rowptr, a.x, a.shift,
                                                        a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, terms, ystats,
                                                        ystats_index, gate);
    }
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

template <int SUM_MODE, int NA, int GX>
static void launch_lean_g(int ntiles, cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int append,
                          VecStats *ys, int yi, const int *gate) {
    static int per_sm = 0;  // resident CTAs per SM (once per instantiation)
    if (per_sm == 0) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_csrmv_lean<SUM_MODE, NA, GX>, kCsrThreads, 0);
        per_sm = v > 0 ? v : 1;
    }
    const int cap = sm_count() * per_sm;
    const int grid = ntiles < cap ? ntiles : cap;
    k_csrmv_lean<SUM_MODE, NA, GX><<<grid, kCsrThreads, 0, s>>>(a.m, a.n, a.val, a.colind, a.rowptr, a.x, a.shift,
                                                                  a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, slow,
                                                                  append, ys, yi, gate);
}

template <int SUM_MODE, int NA>
static void launch_lean(int gx, int ntiles, cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow,
                        int append, VecStats *ys, int yi, const int *gate) {
    if (gx >= 3)
        launch_lean_g<SUM_MODE, NA, 3>(ntiles, s, a, sc, slow, append, ys, yi, gate);
    else if (gx == 2)
        launch_lean_g<SUM_MODE, NA, 2>(ntiles, s, a, sc, slow, append, ys, yi, gate);
    else
        launch_lean_g<SUM_MODE, NA, 1>(ntiles, s, a, sc, slow, append, ys, yi, gate);
}

template <int SUM_MODE, int NA, int GX>
static void launch_pipe_g(int ntiles, cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int append,
                          VecStats *ys, int yi, const int *gate) {
    static int per_sm = 0;  // resident CTAs per SM (once per instantiation)
    if (per_sm == 0) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_csrmv_pipe<SUM_MODE, NA, GX>, kCsrThreads, 0);
        per_sm = v > 0 ? v : 1;
    }
    const int cap = sm_count() * per_sm;
    const int grid = ntiles < cap ? ntiles : cap;
    k_csrmv_pipe<SUM_MODE, NA, GX><<<grid, kCsrThreads, 0, s>>>(a.m, a.n, a.val, a.colind, a.rowptr, a.x, a.shift,
                                                                  a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, slow,
                                                                  append, ys, yi, gate);
}

template <int SUM_MODE, int NA>
static void launch_reg(int gx, int ntiles, cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int append,
                       VecStats *ys, int yi, const int *gate) {
    if (gx >= 3)
        launch_pipe_g<SUM_MODE, NA, 3>(ntiles, s, a, sc, slow, append, ys, yi, gate);
    else if (gx == 2)
        launch_pipe_g<SUM_MODE, NA, 2>(ntiles, s, a, sc, slow, append, ys, yi, gate);
    else
        launch_pipe_g<SUM_MODE, NA, 1>(ntiles, s, a, sc, slow, append, ys, yi, gate);
}

int vec_stats_launch(cudaStream_t s, int nsm, int n, const double *x, VecStats *vs, int index) {
    int blocks = (int)(((int64_t)n + 511) / 512);
    if (blocks > nsm * 8) blocks = nsm * 8;
    if (blocks < 1) blocks = 1;
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0)
        k_vec_stats<true><<<blocks, 256, 0, s>>>(n, x, vs, index);
    else
        k_vec_stats<false><<<blocks, 256, 0, s>>>(n, x, vs, index);
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

int csr_proof_launch(cudaStream_t s, int n, const double *x, int rho, int maxS, CsrScratch *sc, const int *gate) {
    const int gx = chain_group(rho, 3);
    int pb = n > 0 ? (int)(((int64_t)n + 255) / 256) : 1;
    const int pcap = sm_count() * 4;
    if (pb > pcap) pb = pcap;
    if (gx >= 3)
        k_csr_proof<3><<<pb, 256, 0, s>>>(n, x, rho, maxS, sc, gate);
    else if (gx == 2)
        k_csr_proof<2><<<pb, 256, 0, s>>>(n, x, rho, maxS, sc, gate);
    else
        k_csr_proof<1><<<pb, 256, 0, s>>>(n, x, rho, maxS, sc, gate);
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

// The row kernel, and with fixed_slow > 0 the deferred rows of that list
// (terms: NearSum workspace of kCsrSlowChunk rows).
int csr_rows_launch(cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int fixed_slow, VecStats *ystats,
                    int ystats_index, double *terms, const int *gate) {
    if (a.m <= 0) return CUOZBLAS_STATUS_SUCCESS;
    const int rho = rho_rule(a.n, a.epsmode);
    const int gx = chain_group(rho, 3);
    const int rb = (a.m + kCsrThreads - 1) / kCsrThreads;
    // levels per row held on chip: 2 when the caller knows the rows need at
    // most 2 (the CG's pre-split count), 6 when they need more than 4, else 4
    const int na = (a.na_hint > 0 && a.na_hint <= 2) ? 2 : a.na_hint == 3 ? 3 : (a.na_hint > 4 ? 6 : 4);
    const int append = fixed_slow < 0 ? 1 : 0;
    if (a.sum_mode == 1) {
        if (na == 2)
            launch_lean<1, 2>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else if (na == 3)
            launch_lean<1, 3>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else if (na == 6)
            launch_reg<1, 6>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else
            launch_lean<1, 4>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
    } else {
        if (na == 2)
            launch_lean<0, 2>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else if (na == 3)
            launch_lean<0, 3>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else if (na == 6)
            launch_reg<0, 6>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
        else
            launch_lean<0, 4>(gx, rb, s, a, sc, slow, append, ystats, ystats_index, gate);
    }
    for (int c0 = 0; c0 < fixed_slow; c0 += kCsrSlowChunk) {
        const int nr = fixed_slow - c0 < kCsrSlowChunk ? fixed_slow - c0 : kCsrSlowChunk;
        if (a.sum_mode == 1)
            k_csrmv_slow<1><<<(nr + 127) / 128, 128, 0, s>>>(nr, slow + c0, a.val, a.colind, a.rowptr, a.x, a.shift,
                                                            a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, terms,
                                                            ystats, ystats_index, gate);
        else
            k_csrmv_slow<0><<<(nr + 127) / 128, 128, 0, s>>>(nr, slow + c0, a.val, a.colind, a.rowptr, a.x, a.shift,
                                                            a.epsmode, a.maxS, a.alpha, a.beta, a.y, sc, terms,
                                                            ystats, ystats_index, gate);
    }
    return cudaGetLastError() == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

// Fused CSRMV.  *done = false (and y untouched) when x's chain is not proven
// or needs more than 8 levels: the caller then runs the general path.
// `na_hint` (levels of the rows, when the caller knows them) selects how many
// levels per row the main kernel holds.
int csrmv_fused(cuozblasHandle_t *h, int m, int n, double alpha, const double *val, const int *colind,
                const int *rowptr, const double *x, double beta, double *y, int shift, int na_hint, bool *done,
                int *nA_out, int *nB_out) {
    State *st = state(h);
    *done = false;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    CsrScratch *sc = ar.take<CsrScratch>(1);
    int *slow = ar.take<int>(m > 0 ? m : 1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    cudaStream_t s = st->stream;
    OZB_CHECK(cudaMemsetAsync(sc, 0, sizeof(CsrScratch), s));
    const int nsm = sm_count();
    span_begin(h);
    counted(h);
    OZB_TRY(vec_stats_launch(s, nsm, n, x, &sc->vs, 0));
    counted(h);
    OZB_TRY(csr_proof_launch(s, n, x, rho, maxS, sc, nullptr));
    const CsrmvArgs args{m, n, alpha, beta, val, colind, rowptr, x, y, shift, h->splitEpsMode, maxS, h->sumMode,
                         na_hint};
    // NearSum: correctly rounded exact row dots where the splits allow (the
    // slices otherwise, and when x's split turns out incomplete)
    const bool rn = csr_rn_applies(args) && !st->env.csr_slices;
    if (m > 0) counted(h);
    if (rn)
        OZB_TRY(csr_rn_launch(s, args, sc, slow, -1, nullptr, 0, nullptr, nullptr));
    else
        OZB_TRY(csr_rows_launch(s, args, sc, slow, -1, nullptr, 0, nullptr, nullptr));
    span_end(h);
    int res[6];  // valid, nB, nslow, zmax (partial until the deferred rows ran), xcomplete, rn_declined
    OZB_CHECK(cudaMemcpyAsync(res, &sc->valid, sizeof(res), cudaMemcpyDeviceToHost, s));
    OZB_CHECK(cudaStreamSynchronize(s));
    if (!res[0]) {
        ar.release(mk);
        return CUOZBLAS_STATUS_SUCCESS;  // y untouched: general path
    }
    if (rn && res[5]) {  // the row kernel declined: the slice kernel computes every row
        if (m > 0) counted(h);
        OZB_TRY(csr_rows_launch(s, args, sc, slow, -1, nullptr, 0, nullptr, nullptr));
        span_end(h);
        OZB_CHECK(cudaMemcpyAsync(res, &sc->valid, sizeof(res), cudaMemcpyDeviceToHost, s));
        OZB_CHECK(cudaStreamSynchronize(s));
    }
    const int nslow = res[2];
    if (nslow > 0) {
        double *terms = ar.take<double>((uint64_t)kCsrSlowChunk * kMaxSplitDefault * kCsrLv);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        for (int c0 = 0; c0 < nslow; c0 += kCsrSlowChunk) {
            const int nr = nslow - c0 < kCsrSlowChunk ? nslow - c0 : kCsrSlowChunk;
            counted(h);
            if (h->sumMode == 1)
                k_csrmv_slow<1><<<(nr + 127) / 128, 128, 0, s>>>(nr, slow + c0, val, colind, rowptr, x, shift,
                                                                h->splitEpsMode, maxS, alpha, beta, y, sc, terms,
                                                                nullptr, 0, nullptr);
            else
                k_csrmv_slow<0><<<(nr + 127) / 128, 128, 0, s>>>(nr, slow + c0, val, colind, rowptr, x, shift,
                                                                h->splitEpsMode, maxS, alpha, beta, y, sc, terms,
                                                                nullptr, 0, nullptr);
            OZB_CHECK(cudaGetLastError());
        }
        OZB_CHECK(cudaMemcpyAsync(&res[3], &sc->zmax, sizeof(int), cudaMemcpyDeviceToHost, s));
        OZB_CHECK(cudaStreamSynchronize(s));
    }
    ar.release(mk);
    *done = true;
    *nB_out = res[1];
    const int c = (res[3] < 1 ? 1 : res[3]) + 1;  // count rule, src/cpu/ozblas_split.cpp:272-289
    *nA_out = m > 0 ? (c < maxS ? c : maxS) : (maxS < 2 ? maxS : 2);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
