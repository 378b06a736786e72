// cg.cu — the unpreconditioned CG iterations as captured CUDA graphs.
//
// One iteration of the reference CG (src/cpu/ozblas_cg.cpp:61-114) is
//   q = A p (Ozaki CSRMV), tmp = <p, q>, alpha = dold / tmp,
//   x = fma(alpha, p, x), r = fma(-alpha, q, r), dnew = <r, r>,
//   resi = sqrt(dnew), beta = dnew / dold, dold = dnew,
//   p = beta * p, p = fma(1, r, p), history, stop if resi / nrmb < tol.
// Here the scalars live on the device (IEEE division and square root give
// the host's bits), every DOT's first pass (max and lowest set bit of its
// vectors) is folded into the kernel that writes the vector (the p and r
// updates, the SpMV's epilogue), and the scratch areas clean themselves, so
// an iteration is eight kernels (five with NearSum, below) with no host round
// trip.  K iterations are captured once into a graph and replayed.
//
// Every kernel reads a device gate: the iterations after convergence or
// maxiter do nothing.  A fused step whose predicted chain is not proven
// stops the batch where it is: before the x and r updates (the SpMV or
// <p, q>) or after them (<r, r>).  The host finishes that iteration from
// there with the level-by-level path and resumes the graphs, so the
// iterates are the reference's in every case.
#include <stdio.h>
#include <stdlib.h>

#include <functional>
#include <vector>

#include "fused.h"
#include "tc05.cuh"
#include "xbins.cuh"

namespace ozb {

struct CgDev {
    double dold, alpha, beta, nrmb, tol;
    int iter, maxiter;  // completed iterations
    int gate;           // the next iteration's steps run
    int ran;            // this iteration reached its beta (the p update runs)
    int stop;           // converged
    int broken;         // a fused step was not proven
};

__global__ void k_cg_alpha(CgDev *d, const DotScratch *dpq, const CsrScratch *cs) {
    if (!d->gate) return;
    if (dpq->out.status != 1 || !cs->valid) {
        d->broken = cs->valid ? 1 : 2;  // 1: <p, q> not proven, 2: the SpMV's x chain not proven
        d->gate = 0;
        return;
    }
    d->alpha = d->dold / dpq->out.result;
}

__global__ void __launch_bounds__(256) k_cg_update_xr(int n, double *__restrict__ x, double *__restrict__ r,
                                                      const double *__restrict__ p, const double *__restrict__ q,
                                                      const CgDev *d, VecStats *rs) {
    __shared__ double red[8];
    if (!d->gate) return;  // uniform
    const double al = d->alpha;
    double mx = 0.0;
    int lsb = 0, bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = fma(al, p[i], x[i]);
        const double ri = fma(-al, q[i], r[i]);
        r[i] = ri;
        scan_elem(ri, mx, lsb, bad);
    }
    scan_commit(rs, 0, mx, lsb, bad, red);
}

__global__ void k_cg_beta(CgDev *d, const DotScratch *drr, double *res, unsigned long long *stamp) {
    if (!d->gate) {
        d->ran = 0;
        return;
    }
    if (drr->out.status != 1) {
        d->broken = 3;  // <r, r> not proven
        d->gate = 0;
        d->ran = 0;
        return;
    }
    const double dnew = drr->out.result;
    const double resi = sqrt(dnew);
    d->beta = dnew / d->dold;
    d->dold = dnew;
    d->iter += 1;
    const double rel = resi / d->nrmb;
    res[d->iter] = rel;
    stamp[d->iter] = tc::globaltimer();
    d->ran = 1;
    if (rel < d->tol) d->stop = 1;
    d->gate = (!d->stop && d->iter < d->maxiter) ? 1 : 0;
}

__global__ void __launch_bounds__(256) k_cg_update_p(int n, double *__restrict__ p, const double *__restrict__ r,
                                                     const CgDev *d, VecStats *ps_a, VecStats *ps_b) {
    __shared__ double red[8];
    if (!d->ran) return;  // uniform
    const double be = d->beta;
    double mx = 0.0;
    int lsb = 0, bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        // p = beta p, then p = fma(1, r, p): two roundings, never contracted into one fma
        const double pi = fma(1.0, r[i], __dmul_rn(be, p[i]));
        p[i] = pi;
        scan_elem(pi, mx, lsb, bad);
    }
    scan_commit(ps_a, 0, mx, lsb, bad, red);
    scan_commit(ps_b, 0, mx, lsb, bad, red);
}

__global__ void k_cg_stamp(unsigned long long *t) { *t = tc::globaltimer(); }

// ---- NearSum: the dots fused into their producers ----------------------------
// With sumMode 1 each DOT of the iteration is RN of the exact dot product
// whenever the reference's split of both vectors is complete
// (split_complete, from the statistics the producers already gather), so
// <p, q> is one exact pass over p and q that ends in alpha, and <r, r> rides
// in the x / r update, whose last block computes beta, the history and the
// gate: five kernels per iteration (proof, SpMV, <p, q> + alpha,
// x / r + <r, r> + beta, p update) and no separate DOT passes.  The SpMV's
// rows are then correctly rounded exact row dots (csrmv_fused.cu), which need
// only p's split to be complete, not its proven chain: without listed rows
// the proof kernel is left out too (four kernels).

// Exact p . q of n elements into bins, U double2 pairs per lane per step.
template <bool ALIGNED>
__device__ __forceinline__ void cg_dot_stream(int n, const double *__restrict__ a, const double *__restrict__ b,
                                              XAcc &acc) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t iw = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    if (ALIGNED) {
        constexpr int U = 2;
        const int64_t np = (int64_t)n >> 1;
        const double2 *a2 = reinterpret_cast<const double2 *>(a);
        const double2 *b2 = reinterpret_cast<const double2 *>(b);
        const int64_t steps = iw < np ? (np - iw + U * stride - 1) / (U * stride) : 0;
        int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (int64_t s = 0; s < steps; s++, i += U * stride) {
            double2 u[U], v[U];
#pragma unroll
            for (int k = 0; k < U; k++) {
                const int64_t e = i + k * stride;
                u[k] = e < np ? a2[e] : make_double2(0.0, 0.0);
                v[k] = e < np ? b2[e] : make_double2(0.0, 0.0);
            }
            unsigned hi = 0u;
#pragma unroll
            for (int k = 0; k < U; k++) {
                hi = max(hi, abs_hiword(__dmul_rn(u[k].x, v[k].x)));
                hi = max(hi, abs_hiword(__dmul_rn(u[k].y, v[k].y)));
            }
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, hi));
#pragma unroll
            for (int k = 0; k < U; k++) {
                xacc_product(acc, u[k].x, v[k].x);
                xacc_product(acc, u[k].y, v[k].y);
            }
            if ((s & 15) == 15) xacc_normalize(acc);  // every 64 products per lane
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x < 32) {  // the odd last element, one warp
            const double ae = threadIdx.x == 0 ? a[n - 1] : 0.0, be = threadIdx.x == 0 ? b[n - 1] : 0.0;
            xacc_normalize(acc);
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(ae, be))));
            xacc_product(acc, ae, be);
        }
    } else {
        const int64_t steps = iw < n ? ((int64_t)n - iw + stride - 1) / stride : 0;
        int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (int64_t s = 0; s < steps; s++, i += stride) {
            const double ae = i < n ? a[i] : 0.0, be = i < n ? b[i] : 0.0;
            xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(ae, be))));
            xacc_product(acc, ae, be);
            if ((s & 63) == 63) xacc_normalize(acc);
        }
    }
}

__device__ __forceinline__ VecStats load_stats(const VecStats *g) {
    VecStats v;
    for (int i = 0; i < 2; i++) {
        v.mx[i] = __ldcg(&g->mx[i]);
        v.lsb[i] = __ldcg(&g->lsb[i]);
        v.bad[i] = __ldcg(&g->bad[i]);
    }
    return v;
}

// tmp = <p, q> and alpha = dold / tmp.  The statistics of p (from the p
// update) and of q (from the SpMV) are in dpq->vs; they are consumed here.
template <bool ALIGNED>
__global__ void __launch_bounds__(256) k_cg_pq(int n, const double *__restrict__ p, const double *__restrict__ q,
                                               CgDev *d, DotScratch *dpq, CsrScratch *cs, XReduce *xr, int rho,
                                               int maxS, int proof_ran) {
    __shared__ double res_sh;
    __shared__ int cert_sh;
    if (!d->gate) return;  // uniform
    if ((proof_ran && !cs->valid) || cs->rn_declined) {  // the SpMV did not run: the host path takes this iteration
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            d->broken = 2;
            d->gate = 0;
        }
        return;
    }
    XAcc acc;
    xacc_init(acc);
    cg_dot_stream<ALIGNED>(n, p, q, acc);
    if (!xreduce_finish(acc, xr, &res_sh, &cert_sh)) return;
    if (threadIdx.x == 0) {
        const VecStats vs = load_stats(&dpq->vs);
        if (cert_sh && split_complete(vs, 0, rho, maxS) && split_complete(vs, 1, rho, maxS)) {
            d->alpha = d->dold / fma(1.0, res_sh, 0.0 * 0.0);
        } else {
            d->broken = 1;
            d->gate = 0;
        }
        dpq->vs = VecStats{};
        cs->rn_declined = 0;  // every block has read it (the ticket comes after)
    }
}

// x = fma(alpha, p, x), r = fma(-alpha, q, r), dnew = <r, r> (exact, in the
// same pass), then k_cg_beta's step in the last block.
__global__ void __launch_bounds__(256) k_cg_xr_rr(int n, double *__restrict__ x, double *__restrict__ r,
                                                  const double *__restrict__ p, const double *__restrict__ q,
                                                  CgDev *d, VecStats *rs, XReduce *xr, int rho, int maxS,
                                                  double *res, unsigned long long *stamp) {
    __shared__ double red[8];
    __shared__ double res_sh;
    __shared__ int cert_sh;
    if (!d->gate) {  // uniform
        if (blockIdx.x == 0 && threadIdx.x == 0) d->ran = 0;
        return;
    }
    const double al = d->alpha;
    double mx = 0.0;
    int lsb = 0, bad = 0;
    XAcc acc;
    xacc_init(acc);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t iw = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    const int64_t steps = iw < n ? ((int64_t)n - iw + stride - 1) / stride : 0;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t s = 0; s < steps; s++, i += stride) {
        double ri = 0.0;
        if (i < n) {
            x[i] = fma(al, p[i], x[i]);
            ri = fma(-al, q[i], r[i]);
            r[i] = ri;
            scan_elem(ri, mx, lsb, bad);
        }
        xacc_fit(acc, __reduce_max_sync(0xffffffffu, abs_hiword(__dmul_rn(ri, ri))));
        xacc_product(acc, ri, ri);
        if ((s & 63) == 63) xacc_normalize(acc);
    }
    scan_commit(rs, 0, mx, lsb, bad, red);
    if (!xreduce_finish(acc, xr, &res_sh, &cert_sh)) return;
    if (threadIdx.x == 0) {
        const VecStats vs = load_stats(rs);
        *rs = VecStats{};
        if (!(cert_sh && split_complete(vs, 0, rho, maxS))) {
            d->broken = 3;  // <r, r> not certified
            d->gate = 0;
            d->ran = 0;
            return;
        }
        const double dnew = fma(1.0, res_sh, 0.0 * 0.0);
        const double resi = sqrt(dnew);
        d->beta = dnew / d->dold;
        d->dold = dnew;
        d->iter += 1;
        const double rel = resi / d->nrmb;
        res[d->iter] = rel;
        stamp[d->iter] = tc::globaltimer();
        d->ran = 1;
        if (rel < d->tol) d->stop = 1;
        d->gate = (!d->stop && d->iter < d->maxiter) ? 1 : 0;
    }
}

// Run the CG iterations from the state (x, r, p, dold) after `iter`
// iterations.  `host_head` runs an iteration's SpMV, <p, q> and x, r updates
// through the host path, `host_tail` the rest (it reports convergence);
// `res`/`when` (host, maxiter + 1 entries) receive resi / nrmb and the
// elapsed seconds of each iteration.
int cg_graph(cuozblasHandle_t *h, int n, const double *val, const int *colind, const int *rowptr, double *x,
             double *r, double *p, double *q, double nrmb, double tol, int maxiter, int shift, int na_hint,
             double &dold, int &iter, bool &stop, double t1, double *res, double *when,
             const std::function<int()> &host_head, const std::function<int(bool &)> &host_tail,
             const std::function<double()> &wall_now) {
    State *st = state(h);
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const int rho = rho_rule(n, h->splitEpsMode);
    const int nsm = sm_count();
    const int K = maxiter - iter < 32 ? maxiter - iter : 32;  // iterations per graph
    if (K <= 0) return CUOZBLAS_STATUS_SUCCESS;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    const uint64_t nn = (uint64_t)n;
    CgDev *d = ar.take<CgDev>(1);
    DotScratch *dpq = ar.take<DotScratch>(1), *drr = ar.take<DotScratch>(1);
    CsrScratch *cs = ar.take<CsrScratch>(1);
    const bool fused_dots = h->sumMode == 1 && !st->env.dot_two_pass;
    XReduce *xpq = fused_dots ? ar.take<XReduce>(1) : nullptr, *xrr = fused_dots ? ar.take<XReduce>(1) : nullptr;
    int *slow = ar.take<int>(nn + 1);
    double *res_dev = ar.take<double>((uint64_t)maxiter + 1);
    unsigned long long *stamp_dev = ar.take<unsigned long long>((uint64_t)maxiter + 2);
    if (!ar.ok) {
        ar.release(mk);
        return CUOZBLAS_STATUS_WORKSPACE;
    }
    // the host path (fallback batches) allocates above these buffers
    const uint64_t mask0 = h->memMaskSplitA;
    h->memMaskSplitA = st->off;
    cudaStream_t s = nullptr;
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    OZB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int status = CUOZBLAS_STATUS_SUCCESS;
    auto cleanup = [&]() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        h->memMaskSplitA = mask0;
        ar.release(mk);
    };
#define CG_CHECK(call)                                      \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) {                            \
            fprintf(stderr, "cuozblas: CUDA error %s in CG graph\n", cudaGetErrorString(_e)); \
            cleanup();                                      \
            return CUOZBLAS_STATUS_CUDA_ERROR;              \
        }                                                   \
    } while (0)
    // rows the row kernel defers: a property of A, listed once
    int nslow = 0;
    CG_CHECK(cudaMemsetAsync(slow + nn, 0, sizeof(int), s));
    if ((status = csr_slow_rows_launch(s, n, val, rowptr, shift, h->splitEpsMode, maxS, na_hint, slow,
                                       reinterpret_cast<int *>(slow + nn)))) {
        cleanup();
        return status;
    }
    CG_CHECK(cudaMemcpyAsync(&nslow, slow + nn, sizeof(int), cudaMemcpyDeviceToHost, s));
    CG_CHECK(cudaStreamSynchronize(s));
    double *terms = nullptr;
    if (nslow > 0) {
        terms = ar.take<double>((uint64_t)8192 * kMaxSplitDefault * kCsrLv);
        if (!ar.ok) {
            cleanup();
            return CUOZBLAS_STATUS_WORKSPACE;
        }
        h->memMaskSplitA = st->off;
    }
    if ((status = dot_tree_prepare())) {
        cleanup();
        return status;
    }
    const CsrmvArgs spmv{n, n, 1.0, 0.0, val, colind, rowptr, p, q, shift, h->splitEpsMode, maxS, h->sumMode,
                         na_hint};
    // seed the device state from the host's
    auto seed = [&]() -> int {
        CgDev hd{};
        hd.dold = dold;
        hd.nrmb = nrmb;
        hd.tol = tol;
        hd.iter = iter;
        hd.maxiter = maxiter;
        hd.gate = (!stop && iter < maxiter) ? 1 : 0;
        OZB_CHECK(cudaMemcpyAsync(d, &hd, sizeof(hd), cudaMemcpyHostToDevice, s));
        OZB_CHECK(cudaMemsetAsync(dpq, 0, sizeof(DotScratch), s));
        OZB_CHECK(cudaMemsetAsync(drr, 0, sizeof(DotScratch), s));
        OZB_CHECK(cudaMemsetAsync(cs, 0, sizeof(CsrScratch), s));
        if (fused_dots) {
            OZB_CHECK(cudaMemsetAsync(xpq, 0, sizeof(XReduce), s));
            OZB_CHECK(cudaMemsetAsync(xrr, 0, sizeof(XReduce), s));
        }
        OZB_TRY(vec_stats_launch(s, nsm, n, p, &cs->vs, 0));
        OZB_TRY(vec_stats_launch(s, nsm, n, p, &dpq->vs, 0));
        OZB_CHECK(cudaStreamSynchronize(s));
        return CUOZBLAS_STATUS_SUCCESS;
    };
    if ((status = seed())) {
        cleanup();
        return status;
    }
    // capture K iterations
    const int ub = (int)((nn + 255) / 256) < nsm * 8 ? (int)((nn + 255) / 256) : nsm * 8;
    CG_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int cap = CUOZBLAS_STATUS_SUCCESS;
    const bool aligned_pq = ((reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(q)) & 15u) == 0;
    int xb = ub < nsm * 4 ? ub : nsm * 4;  // blocks of the fused dot kernels (one part each)
    if (xb > kXMaxBlocks) xb = kXMaxBlocks;
    const bool rn_rows = fused_dots && csr_rn_applies(spmv) && !st->env.csr_slices;
    // correctly rounded rows need only p's completeness (its statistics from the p
    // update, dpq->vs[0]), not its proven chain: no proof kernel unless listed rows
    // (computed through p's slices) need one
    const bool no_proof = rn_rows && nslow == 0;
    for (int k = 0; k < K && !cap; k++) {
        if (!no_proof) cap = csr_proof_launch(s, n, p, rho, maxS, cs, &d->gate);
        if (!cap)
            cap = rn_rows ? csr_rn_launch(s, spmv, cs, slow, nslow, &dpq->vs, 1, terms, &d->gate,
                                          no_proof ? &dpq->vs : nullptr)
                          : csr_rows_launch(s, spmv, cs, slow, nslow, &dpq->vs, 1, terms, &d->gate);
        if (fused_dots) {
            if (aligned_pq)
                k_cg_pq<true><<<xb, 256, 0, s>>>(n, p, q, d, dpq, cs, xpq, rho, maxS, no_proof ? 0 : 1);
            else
                k_cg_pq<false><<<xb, 256, 0, s>>>(n, p, q, d, dpq, cs, xpq, rho, maxS, no_proof ? 0 : 1);
            k_cg_xr_rr<<<xb, 256, 0, s>>>(n, x, r, p, q, d, &drr->vs, xrr, rho, maxS, res_dev, stamp_dev);
        } else {
            if (!cap)
                cap = dot_tree_launch(s, nsm, n, p, q, rho, maxS, h->sumMode, dpq, &d->gate, state(h)->env.dot_tree);
            k_cg_alpha<<<1, 1, 0, s>>>(d, dpq, cs);
            k_cg_update_xr<<<ub, 256, 0, s>>>(n, x, r, p, q, d, &drr->vs);
            if (!cap)
                cap = dot_tree_launch(s, nsm, n, r, r, rho, maxS, h->sumMode, drr, &d->gate, state(h)->env.dot_tree);
            k_cg_beta<<<1, 1, 0, s>>>(d, drr, res_dev, stamp_dev);
        }
        k_cg_update_p<<<ub, 256, 0, s>>>(n, p, r, d, &cs->vs, &dpq->vs);
    }
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (cap) {
        cleanup();
        return cap;
    }
    CG_CHECK(ce);
    CG_CHECK(cudaGraphInstantiate(&exec, graph, 0));
    const int per_iter = (fused_dots ? (no_proof ? 4 : 5) : 8) + (nslow > 0 ? (nslow + 8191) / 8192 : 0);
    // device clock against the host's, for the elapsed-time history
    k_cg_stamp<<<1, 1, 0, s>>>(stamp_dev + maxiter + 1);
    unsigned long long dev0 = 0;
    CG_CHECK(cudaMemcpyAsync(&dev0, stamp_dev + maxiter + 1, sizeof(dev0), cudaMemcpyDeviceToHost, s));
    CG_CHECK(cudaStreamSynchronize(s));
    const double host0 = wall_now();
    int batches = 0, reruns = 0;
    while (!stop && iter < maxiter) {
        const int before = iter;
        batches++;
        CG_CHECK(cudaGraphLaunch(exec, s));
        CgDev hd;
        CG_CHECK(cudaMemcpyAsync(&hd, d, sizeof(hd), cudaMemcpyDeviceToHost, s));
        CG_CHECK(cudaStreamSynchronize(s));
        st->launches += (uint64_t)per_iter * (uint64_t)(hd.iter - before);
        const int got = hd.iter - before;  // iterations the graph completed
        if (got > 0) {
            std::vector<unsigned long long> ts((size_t)got);
            CG_CHECK(cudaMemcpyAsync(res + before + 1, res_dev + before + 1, sizeof(double) * got,
                                     cudaMemcpyDeviceToHost, s));
            CG_CHECK(cudaMemcpyAsync(ts.data(), stamp_dev + before + 1, sizeof(unsigned long long) * got,
                                     cudaMemcpyDeviceToHost, s));
            CG_CHECK(cudaStreamSynchronize(s));
            for (int i = 0; i < got; i++)
                when[before + 1 + i] = host0 - t1 + (double)(long long)(ts[(size_t)i] - dev0) * 1e-9;
        }
        if (!hd.broken) {
            iter = hd.iter;
            dold = hd.dold;
            stop = hd.stop != 0;
            continue;
        }
        // a step was not proven: the host path finishes this iteration
        iter = hd.iter;
        dold = hd.dold;
        if (state(h)->env.cg_trace)
            fprintf(stderr, "cuozblas: CG iteration %d finished on the host (step %d)\n", iter + 1, hd.broken);
        if (hd.broken != 3 && (status = host_head())) {
            cleanup();
            return status;
        }
        if ((status = host_tail(stop))) {
            cleanup();
            return status;
        }
        reruns++;
        CG_CHECK(cudaStreamSynchronize(st->stream));  // the host path's last updates of p, r, x
        if ((status = seed())) {
            cleanup();
            return status;
        }
    }
    if (state(h)->env.cg_trace)
        fprintf(stderr, "cuozblas: CG %d iterations in %d graph batches of %d, %d finished on the host path\n",
                iter, batches, K, reruns);
    cleanup();
    return CUOZBLAS_STATUS_SUCCESS;
#undef CG_CHECK
}

}  // namespace ozb
