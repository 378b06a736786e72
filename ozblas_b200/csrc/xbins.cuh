// xbins.cuh — exact accumulation of a stream of doubles in one pass, in bins
// of fixed absolute grids, for the correctly rounded (NearSum) reductions.
//
// With a complete split the reference's NearSum DOT returns RN of the exact
// dot product (its slice-pair products are exact and NearSum rounds their
// exact sum once), so any exact method gives its bits.  Here every product
// x*y is the exact pair (p, e) of TwoProd (p = RN(x y), e = fma(x, y, -p)).
// The e are at most 2^-53 |p|: they are added in plain FP64 (es) next to a
// rounded-up sum of their magnitudes (ea), and es's error is bounded by
// 2^-28 ea (at most 2^22 additions on any path).  Each p is cut onto the
// grids of K consecutive bins:
//   bin j holds multiples of g_j = 2^((B - j) W),
//   q_j = (r + sigma_j) - sigma_j with sigma_j = 1.5 * 2^((B - j) W + 52)
// is r rounded to g_j (exact while |r| < 2^((B - j) W + 51)), r -= q_j is
// exact, and the bin adds q_j exactly while it stays below 2^53 g_j.  B is
// warp-uniform: it rises when a product reaches 2^((B + 1) W) or when a
// lane's top bin fills (the top bin's content is then cut onto the next grid
// up and the lowest bin leaves the window).  What a deposit leaves below the
// lowest bin, and every bin that leaves the window, is added with upward
// rounding to `drop`, an upper bound of everything not held exactly; the
// final value is certified by rounding the held sum (bins and es) minus and
// plus the total bound (equal results: the rounding of the true sum is
// determined).
#pragma once
#include "chain.cuh"
#include "ozb_device.cuh"
#include "sum.cuh"

namespace ozb {

constexpr int kXK = 4;      // bins per lane
constexpr int kXW = 44;     // bits per bin (a bin takes 2^(52 - 44) = 256 deposits between renormalisations)
constexpr int kXBmin = -20; // lowest top bin: the lowest grid stays >= 2^-1012 (sigmas normal)
constexpr int kXBmax = 21;  // highest top bin: sigmas of the next bin up stay finite

struct XAcc {
    int B;              // top bin (warp-uniform)
    double a[kXK];      // bins, exact
    double sig[kXK];    // sigma_j of the current B
    double drop;        // upper bound of |everything not held| (rounded up)
    double es, ea;      // sum of the TwoProd error terms, sum of their magnitudes (rounded up)
    int flags;          // 1: a product outside the range TwoProd keeps exact (tiny or huge)
};

__device__ __forceinline__ void xacc_sigmas(XAcc &x) {
#pragma unroll
    for (int j = 0; j < kXK; j++) x.sig[j] = 1.5 * pow2((x.B - j) * kXW + 52);
}

__device__ __forceinline__ void xacc_init(XAcc &x) {
    x.B = kXBmin;
#pragma unroll
    for (int j = 0; j < kXK; j++) x.a[j] = 0.0;
    x.drop = 0.0;
    x.es = x.ea = 0.0;
    x.flags = 0;
    xacc_sigmas(x);
}

// Cut v onto bins j0..K-1 (v below the top of bin j0's range).
template <int J0>
__device__ __forceinline__ void xacc_deposit(XAcc &x, double v) {
    double r = v;
#pragma unroll
    for (int j = J0; j < kXK; j++) {
        const double q = __dsub_rn(__dadd_rn(r, x.sig[j]), x.sig[j]);
        r = __dsub_rn(r, q);
        x.a[j] = __dadd_rn(x.a[j], q);
    }
    x.drop = __dadd_ru(x.drop, fabs(r));
}

// The product x * y: p into the bins, its exact error term into es / ea.
__device__ __forceinline__ void xacc_product(XAcc &x, double a, double b) {
    const double p = __dmul_rn(a, b);
    const double e = __fma_rn(a, b, -p);
    const double ap = fabs(p);
    // TwoProd is exact unless the product is tiny (its error term underflows)
    // or beyond the window's top (kXBmax)
    if ((ap < 0x1p-969 && a != 0.0 && b != 0.0) || ap >= 0x1p1012) x.flags |= 1;
    xacc_deposit<0>(x, p);
    x.es = __dadd_rn(x.es, e);
    x.ea = __dadd_ru(x.ea, fabs(e));
}

// Lean form for a group of products fitted together (xacc_fit / xacc_fit1 on
// their largest high word): p goes into bins 0..KD-1 only, and neither the
// remainder below bin KD-1 nor |e| is accumulated per product; instead
// xacc_lean_bounds adds, once per group, bounds that hold for every member:
// the remainder after bin KD-1 is at most g_{KD-1} / 2 and |e| <= ulp(p) / 2.
// The flags collect the products TwoProd cannot keep exact (xacc_product):
// tiny ones here, huge ones in xacc_lean_bounds.
constexpr unsigned kXTinyHi = (unsigned)(-969 + 1023) << 20;  // high word of 2^-969
constexpr unsigned kXHugeHi = (unsigned)(1012 + 1023) << 20;  // high word of 2^1012

template <int KD>
__device__ __forceinline__ void xacc_product_lean(XAcc &x, double a, double b) {
    const double p = __dmul_rn(a, b);
    const double e = __fma_rn(a, b, -p);
    if (abs_hiword(p) < kXTinyHi)  // p tiny or zero: an issue only when both factors are nonzero
        if (a != 0.0 && b != 0.0) x.flags |= 1;
    double r = p;
#pragma unroll
    for (int j = 0; j < KD; j++) {
        const double q = __dsub_rn(__dadd_rn(r, x.sig[j]), x.sig[j]);
        if (j + 1 < KD) r = __dsub_rn(r, q);
        x.a[j] = __dadd_rn(x.a[j], q);
    }
    x.es = __dadd_rn(x.es, e);
}

// Bounds of a group of `cnt` lean products whose largest |p| has the high
// word `hi`: drop += cnt g_{KD-1} / 2, ea += cnt 2^(E - 53) (E the exponent of
// the largest |p|; smaller products have smaller error terms).  Call after
// the group's deposits with the B they used.
template <int KD>
__device__ __forceinline__ void xacc_lean_bounds(XAcc &x, unsigned hi, int cnt) {
    if (hi >= kXHugeHi) x.flags |= 1;
    x.drop = __dadd_ru(x.drop, (double)cnt * pow2((x.B - (KD - 1)) * kXW - 1));
    const int E = (int)(hi >> 20) - 1023;
    if (hi >= kXTinyHi) x.ea = __dadd_ru(x.ea, (double)cnt * pow2(E - 53));
}

// Raise B by one: the top bin is cut onto the new top grid, the rest move
// down one bin, the lowest leaves the window (into drop).  Every lane of the
// warp calls this together.
__device__ __forceinline__ void xacc_raise(XAcc &x) {
    if (x.B >= kXBmax) {
        x.flags |= 1;
        return;
    }
    const double s = 1.5 * pow2((x.B + 1) * kXW + 52);
    const double c = __dsub_rn(__dadd_rn(x.a[0], s), s);
    x.drop = __dadd_ru(x.drop, fabs(x.a[kXK - 1]));
#pragma unroll
    for (int j = kXK - 1; j >= 2; j--) x.a[j] = x.a[j - 1];
    x.a[1] = __dsub_rn(x.a[0], c);
    x.a[0] = c;
    x.B += 1;
    xacc_sigmas(x);
}

// Before depositing products whose largest magnitude (over the warp) has the
// high word `hi_max` (sign cleared): raise B until they lie below 2^((B+1)W).
__device__ __forceinline__ void xacc_fit(XAcc &x, unsigned hi_max) {
    while (x.B < kXBmax && hi_max >= (unsigned)((x.B + 1) * kXW + 1023) << 20) xacc_raise(x);
}

// Carry every bin's part above the next bin's grid into it (exact), then keep
// the top bin below 2^(W-1) g_0 by raising B (warp-uniform).  Afterwards
// |a_j| <= 2^(W-1) g_j for every bin, so 2^(54 - W) such values add exactly.
__device__ __forceinline__ void xacc_normalize(XAcc &x) {
#pragma unroll
    for (int j = kXK - 1; j >= 1; j--) {
        const double c = __dsub_rn(__dadd_rn(x.a[j], x.sig[j - 1]), x.sig[j - 1]);
        x.a[j] = __dsub_rn(x.a[j], c);
        x.a[j - 1] = __dadd_rn(x.a[j - 1], c);
    }
    for (int guard = 0; guard < 4; guard++) {
        const double lim = pow2((x.B + 1) * kXW - 1);
        if (!__any_sync(0xffffffffu, fabs(x.a[0]) > lim)) break;
        xacc_raise(x);
        const double c = __dsub_rn(__dadd_rn(x.a[1], x.sig[0]), x.sig[0]);
        x.a[1] = __dsub_rn(x.a[1], c);
        x.a[0] = __dadd_rn(x.a[0], c);
    }
}

// Per-lane forms, for lanes that accumulate different reductions (the rows of
// a matrix): every lane keeps its own B, and the decisions diverge.
__device__ __forceinline__ void xacc_fit1(XAcc &x, unsigned hi) {
    while (x.B < kXBmax && hi >= (unsigned)((x.B + 1) * kXW + 1023) << 20) xacc_raise(x);
}

__device__ __forceinline__ void xacc_normalize1(XAcc &x) {
#pragma unroll
    for (int j = kXK - 1; j >= 1; j--) {
        const double c = __dsub_rn(__dadd_rn(x.a[j], x.sig[j - 1]), x.sig[j - 1]);
        x.a[j] = __dsub_rn(x.a[j], c);
        x.a[j - 1] = __dadd_rn(x.a[j - 1], c);
    }
    for (int guard = 0; guard < 4 && fabs(x.a[0]) > pow2((x.B + 1) * kXW - 1); guard++) {
        xacc_raise(x);
        const double c = __dsub_rn(__dadd_rn(x.a[1], x.sig[0]), x.sig[0]);
        x.a[1] = __dsub_rn(x.a[1], c);
        x.a[0] = __dadd_rn(x.a[0], c);
    }
}

// One bin set of a block or of the whole reduction: top bin B, K bins,
// the drop bound and the flags.
struct XPart {
    double B, a[kXK], drop, es, ea, flags;
};

// Bound of |es - (exact sum of the error terms)| for a total magnitude ea.
__device__ __forceinline__ double xes_bound(double ea) { return __dmul_ru(ea, 0x1p-28); }

// The certified correct rounding of the exact sum of `np` normalised bin
// sets, part(i) returning the i-th (one thread; np <= 2^(54 - W) / 2 so the
// bins add exactly).
template <typename Get>
__device__ inline bool xparts_round1(int np, Get part, double &out) {
    int Bg = kXBmin, f = 0;
    for (int i = 0; i < np; i++) {
        Bg = max(Bg, (int)part(i).B);
        f |= (int)part(i).flags;
    }
    if (f) return false;
    double c[kXK + 1], drop = 0.0, es = 0.0, ea = 0.0;
#pragma unroll
    for (int j = 0; j < kXK; j++) c[j] = 0.0;
    for (int i = 0; i < np; i++) {
        const XPart &q = part(i);
        const int d = Bg - (int)q.B;
#pragma unroll
        for (int j = 0; j < kXK; j++) {
            if (j + d < kXK)
                c[j + d] = __dadd_rn(c[j + d], q.a[j]);
            else
                drop = __dadd_ru(drop, fabs(q.a[j]));
        }
        drop = __dadd_ru(drop, q.drop);
        es = __dadd_rn(es, q.es);
        ea = __dadd_ru(ea, q.ea);
    }
    c[kXK] = es;
    drop = __dadd_ru(drop, xes_bound(ea));
    if (drop == 0.0) {
        out = nearsum(kXK + 1, c, 1);
        return true;
    }
    double lo[kXK + 2], hi[kXK + 2];
#pragma unroll
    for (int j = 0; j <= kXK; j++) lo[j] = hi[j] = c[j];
    lo[kXK + 1] = -drop;
    hi[kXK + 1] = drop;
    const double rl = nearsum(kXK + 2, lo, 1), rh = nearsum(kXK + 2, hi, 1);
    out = rl;
    return dbits(rl) == dbits(rh);
}


// Warp sum of the lanes' bins (same B), then block sum into `out` (thread 0;
// `wsh` holds one XPart per warp).  Exact: every lane is normalised first, a
// warp's bins stay below 2^(W+4) g and a block of at most 8 warps below
// 2^(W+7) g.
__device__ __forceinline__ void xacc_block_reduce(XAcc &x, XPart *wsh, XPart &out) {
    xacc_normalize(x);
#pragma unroll
    for (int j = 0; j < kXK; j++)
        for (int o = 16; o > 0; o >>= 1) x.a[j] = __dadd_rn(x.a[j], __shfl_xor_sync(0xffffffffu, x.a[j], o));
    for (int o = 16; o > 0; o >>= 1) {
        x.drop = __dadd_ru(x.drop, __shfl_xor_sync(0xffffffffu, x.drop, o));
        x.es = __dadd_rn(x.es, __shfl_xor_sync(0xffffffffu, x.es, o));
        x.ea = __dadd_ru(x.ea, __shfl_xor_sync(0xffffffffu, x.ea, o));
    }
    const int fl = (int)__reduce_or_sync(0xffffffffu, (unsigned)x.flags);
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        wsh[w].B = (double)x.B;
#pragma unroll
        for (int j = 0; j < kXK; j++) wsh[w].a[j] = x.a[j];
        wsh[w].drop = x.drop;
        wsh[w].es = x.es;
        wsh[w].ea = x.ea;
        wsh[w].flags = (double)fl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int Bb = kXBmin;
        for (int i = 0; i < nw; i++) Bb = max(Bb, (int)wsh[i].B);
        XPart r;
        r.B = (double)Bb;
        for (int j = 0; j < kXK; j++) r.a[j] = 0.0;
        r.drop = r.es = r.ea = 0.0;
        int f = 0;
        for (int i = 0; i < nw; i++) {  // <= 8 warps of bins below 2^(W+4) g: exact
            const int d = Bb - (int)wsh[i].B;
            for (int j = 0; j < kXK; j++) {
                if (j + d < kXK)
                    r.a[j + d] = __dadd_rn(r.a[j + d], wsh[i].a[j]);
                else
                    r.drop = __dadd_ru(r.drop, fabs(wsh[i].a[j]));
            }
            r.drop = __dadd_ru(r.drop, wsh[i].drop);
            r.es = __dadd_rn(r.es, wsh[i].es);
            r.ea = __dadd_ru(r.ea, wsh[i].ea);
            f |= (int)wsh[i].flags;
        }
        r.flags = (double)f;
        out = r;
    }
}

// Exact sum of `np` block parts into a correctly rounded double (one block
// of 256 threads; the caller synchronises before and reads *result after).
// Parts are shifted onto the largest top bin with two spare bins above it;
// *certified = 0 when the drop bound leaves the rounding open or a flag is
// set.  `sh` is shared scratch of at least 256 * (kXK2 + 3) doubles.
constexpr int kXK2 = kXK + 2;
__device__ inline void xparts_round(const XPart *parts, int np, double *sh, double *result, int *certified) {
    __shared__ int s_B, s_flags;
    const int t = threadIdx.x;
    if (t == 0) {
        s_B = kXBmin;
        s_flags = 0;
    }
    __syncthreads();
    {  // the largest top bin and the flags, every thread over its parts
        int Bg = kXBmin, f = 0;
        for (int i = t; i < np; i += blockDim.x) {
            Bg = max(Bg, (int)__ldcg(&parts[i].B));
            f |= (int)__ldcg(&parts[i].flags);
        }
        Bg = __reduce_max_sync(0xffffffffu, Bg);
        f = (int)__reduce_or_sync(0xffffffffu, (unsigned)f);
        if ((t & 31) == 0) {
            atomicMax(&s_B, Bg);
            atomicOr(&s_flags, f);
        }
    }
    __syncthreads();
    const int Bt = s_B + 2;  // top of the 6-bin layout
    double c[kXK2], sig[kXK2], drop = 0.0, es = 0.0, ea = 0.0;
#pragma unroll
    for (int j = 0; j < kXK2; j++) {
        c[j] = 0.0;
        sig[j] = 1.5 * pow2((Bt - j) * kXW + 52);
    }
    for (int i = t; i < np; i += blockDim.x) {
        const int d = s_B - (int)__ldcg(&parts[i].B);
        for (int j = 0; j < kXK; j++) {
            const double v = __ldcg(&parts[i].a[j]);
            const int k = j + d + 2;
            if (k < kXK2)
                c[k] = __dadd_rn(c[k], v);
            else
                drop = __dadd_ru(drop, fabs(v));
        }
        drop = __dadd_ru(drop, __ldcg(&parts[i].drop));
        es = __dadd_rn(es, __ldcg(&parts[i].es));
        ea = __dadd_ru(ea, __ldcg(&parts[i].ea));
        // a part's bins are below 2^(W+7) g (8 warps of normalised lanes) and c's
        // below 2^(W-1) g after this carry: the next part adds exactly
#pragma unroll
        for (int j = kXK2 - 1; j >= 1; j--) {
            const double q = __dsub_rn(__dadd_rn(c[j], sig[j - 1]), sig[j - 1]);
            c[j] = __dsub_rn(c[j], q);
            c[j - 1] = __dadd_rn(c[j - 1], q);
        }
    }
    // every bin is now below 2^(W-1) g (the top two far below): 256 threads add
    // exactly in any order; warps first (shuffles), then the 8 warp sums
    // slots: the kXK2 bins, es, drop, ea
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int j = 0; j < kXK2; j++) c[j] = __dadd_rn(c[j], __shfl_xor_sync(0xffffffffu, c[j], o));
        es = __dadd_rn(es, __shfl_xor_sync(0xffffffffu, es, o));
        drop = __dadd_ru(drop, __shfl_xor_sync(0xffffffffu, drop, o));
        ea = __dadd_ru(ea, __shfl_xor_sync(0xffffffffu, ea, o));
    }
    const int nw = blockDim.x >> 5;
    if ((t & 31) == 0) {
        const int w = t >> 5;
#pragma unroll
        for (int j = 0; j < kXK2; j++) sh[j * nw + w] = c[j];
        sh[kXK2 * nw + w] = es;
        sh[(kXK2 + 1) * nw + w] = drop;
        sh[(kXK2 + 2) * nw + w] = ea;
    }
    __syncthreads();
    if (t == 0) {
        for (int j = 0; j < kXK2 + 3; j++) {
            double v = sh[j * nw];
            for (int w = 1; w < nw; w++)
                v = j == kXK2 + 1 || j == kXK2 + 2 ? __dadd_ru(v, sh[j * nw + w]) : __dadd_rn(v, sh[j * nw + w]);
            sh[j * nw] = v;
        }
    }
    if (t == 0) {
        double terms[kXK2 + 2];
        for (int j = 0; j <= kXK2; j++) terms[j] = sh[j * nw];
        const double D = __dadd_ru(sh[(kXK2 + 1) * nw], xes_bound(sh[(kXK2 + 2) * nw]));
        int ok = s_flags == 0;
        double r = 0.0;
        if (ok) {
            if (D == 0.0) {
                r = nearsum(kXK2 + 1, terms, 1);
            } else {
                double lo[kXK2 + 2], hi[kXK2 + 2];
                for (int j = 0; j <= kXK2; j++) lo[j] = hi[j] = terms[j];
                lo[kXK2 + 1] = -D;
                hi[kXK2 + 1] = D;
                const double rl = nearsum(kXK2 + 2, lo, 1), rh = nearsum(kXK2 + 2, hi, 1);
                ok = (dbits(rl) == dbits(rh));
                r = rl;
            }
        }
        *result = r;
        *certified = ok;
    }
}

constexpr int kXMaxBlocks = 1184;  // block parts a reduction holds (148 SMs x 8)

// Scratch of one one-pass exact reduction: the blocks' parts and the ticket
// that finds the last block (self-cleaning: the last block resets it).
struct XReduce {
    XPart part[kXMaxBlocks];
    unsigned ticket;
    int pad;
};

// End of a one-pass exact reduction over gridDim.x <= kXMaxBlocks blocks of
// 256 threads (every thread calls this): each block folds its lanes' bins
// into its part; returns true, in every thread of the last block only, with
// the certified rounding of the total in *result and *certified (shared
// memory, valid for all threads of that block).
// `sh`: shared scratch of 256 * (kXK2 + 3) doubles (the caller's, e.g. a
// streaming ring that is no longer in use).
__device__ inline bool xreduce_finish_sh(XAcc &acc, XReduce *xr, double *result, int *certified, double *sh) {
    __shared__ XPart wsh[8];
    __shared__ int last;
    xacc_block_reduce(acc, wsh, xr->part[blockIdx.x]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&xr->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    xparts_round(xr->part, gridDim.x, sh, result, certified);
    if (threadIdx.x == 0) xr->ticket = 0u;
    __syncthreads();
    return true;
}

__device__ inline bool xreduce_finish(XAcc &acc, XReduce *xr, double *result, int *certified) {
    __shared__ double sh[256 * (kXK2 + 3)];
    return xreduce_finish_sh(acc, xr, result, certified, sh);
}

}  // namespace ozb
