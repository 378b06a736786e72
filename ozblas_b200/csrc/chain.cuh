// chain.cuh — the predicted tau chain of a vector split, shared by the fused
// DOT and CSRMV.
//
// The reference splits a vector level by level with one global chain
// (src/cpu/ozblas_split.cpp:62-103): tau_s = (short)ceil(log2(max|r_s|)),
// sigma_s = 0.75 * 2^(rho + tau_s), slice = (r + sigma) - sigma, and the
// count rule of :272-289.  With the chain predicted as
// tau_{s+1} = tau_s + rho - 54, level s rounds to the grid
// g_s = 2^(rho + tau_s - 53); the partial sum of slices 0..s is RN_{g_s}(v),
// and the remainder after level s is zero exactly when v is a multiple of
// g_s.  One pass over the vector (max, lowest set bit) therefore fixes the
// whole plan: sigmas, the first all-zero level and the slice count.  The
// prediction itself is proven afterwards from the largest slice of the next
// level, which bounds the remainder from below.
#pragma once
#include "ozb_device.cuh"

namespace ozb {

constexpr int kChainLevels = 8;
constexpr int kLsbBias = 2100;  // lowest set bits are kept as kLsbBias - lsb (> 0) for atomicMax

// Per-vector statistics of the first pass (index 0: x, 1: y; zeroed first).
struct VecStats {
    double mx[2];  // max|v| (bit-pattern atomics)
    int lsb[2];    // kLsbBias - lowest set bit of a nonzero element; 0: all zero
    int bad[2];    // an element is Inf or NaN
};

__device__ __forceinline__ void scan_elem(double v, double &mx, int &lsb, int &bad) {
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    mx = ref_max(mx, fabs(v));
    const int be = (int)(b >> 52);
    if (be == 0x7ff) {
        bad = 1;
    } else if (b != 0) {
        const uint64_t m = be ? ((b & ((1ULL << 52) - 1)) | (1ULL << 52)) : b;
        const int l = (be ? be - 1075 : -1074) + (__ffsll((long long)m) - 1);
        lsb = max(lsb, kLsbBias - l);
    }
}

// scan_elem with fewer integer operations: the maximum by fmax (a NaN only
// matters together with `bad`, which every consumer checks first), the
// lowest set bit from the 32-bit halves.
__device__ __forceinline__ void scan_elem_fast(double v, double &mx, int &lsb, int &bad) {
    mx = fmax(mx, fabs(v));
    const unsigned hw = (unsigned)__double2hiint(v) & 0x7fffffffu, lw = (unsigned)__double2loint(v);
    const int be = (int)(hw >> 20);
    bad |= be == 0x7ff;
    // lowest set bit: the exponent of the last significand bit (the implicit
    // bit stands in for an all-zero fraction; subnormals use exponent -1074)
    const int c = lw ? __ffs(lw) - 1 : 31 + __ffs((hw & 0xfffffu) | 0x100000u);
    const int l = max(be, 1) - 1075 + c;
    if ((hw | lw) != 0u && be != 0x7ff) lsb = max(lsb, kLsbBias - l);
}

// The statistics of one vector in a streaming kernel, with the lowest set bit
// computed lazily: an element can lower the lowest set bit exponent `lb` only
// if its ulp exponent max(be, 1) - 1075 is below it, which a warp-uniform
// threshold (the warp's lowest lb, + 1075 in biased-exponent units) tests in
// a few integer operations; the exact exponent (and the candidate element)
// is computed only when some lane passes.  Inf / NaN show in the largest
// high word.
struct LazyStats {
    double mx = 0.0;    // max |v| (fmax: NaN shows in hmax instead)
    unsigned hmax = 0;  // largest high word of |v|
    int lb = 4000;      // lowest set-bit exponent (4000: no nonzero element yet)
    int thr = 5075;     // warp-uniform: a nonzero element with max(be, 1) >= thr cannot lower lb
    double cand = 0.0;  // an element whose lowest set bit is lb
};

__device__ __forceinline__ void lazy_elem(LazyStats &st, double v) {
    st.mx = fmax(st.mx, fabs(v));
    const unsigned hw = (unsigned)__double2hiint(v) & 0x7fffffffu, lw = (unsigned)__double2loint(v);
    st.hmax = max(st.hmax, hw);
    const int mb = max((int)(hw >> 20), 1);
    const bool pass = mb < st.thr && (hw | lw) != 0u && mb != 0x7ff;
    if (__any_sync(0xffffffffu, pass)) {  // uniform
        const int c = lw ? __ffs(lw) - 1 : 31 + __ffs((hw & 0xfffffu) | 0x100000u);
        const int l = mb - 1075 + c;
        if (pass && l < st.lb) {
            st.lb = l;
            st.cand = v;
        }
    }
}

// After each step: the warp's threshold from its lowest lb.
__device__ __forceinline__ void lazy_sync(LazyStats &st) { st.thr = __reduce_min_sync(0xffffffffu, st.lb) + 1075; }

__device__ __forceinline__ int lazy_key(const LazyStats &st) { return st.lb < 4000 ? kLsbBias - st.lb : 0; }
__device__ __forceinline__ int lazy_bad(const LazyStats &st) { return st.hmax >= 0x7ff00000u; }

// The per-lane form (lanes that scan different vectors, e.g. the rows of a
// matrix): the threshold is the lane's own, the exact exponent is computed
// when some lane of the warp passes.
__device__ __forceinline__ void lazy_elem1(LazyStats &st, double v) {
    st.mx = fmax(st.mx, fabs(v));
    const unsigned hw = (unsigned)__double2hiint(v) & 0x7fffffffu, lw = (unsigned)__double2loint(v);
    st.hmax = max(st.hmax, hw);
    const int mb = max((int)(hw >> 20), 1);
    const bool pass = mb < st.lb + 1075 && (hw | lw) != 0u && mb != 0x7ff;
    if (__any_sync(0xffffffffu, pass)) {  // uniform
        const int c = lw ? __ffs(lw) - 1 : 31 + __ffs((hw & 0xfffffu) | 0x100000u);
        const int l = mb - 1075 + c;
        if (pass && l < st.lb) st.lb = l;
    }
}

// Fold one thread's statistics of vector v into `vs` (every thread of the
// block calls this; `red` holds one double per warp).
__device__ __forceinline__ void scan_commit(VecStats *vs, int v, double mx, int lsb, int bad, double *red) {
    mx = block_max_nonneg(mx, red);
    lsb = __reduce_max_sync(0xffffffffu, lsb);
    bad = (int)__reduce_or_sync(0xffffffffu, (unsigned)bad);
    if ((threadIdx.x & 31) == 0) {
        if (lsb) atomicMax(&vs->lsb[v], lsb);
        if (bad) atomicOr(&vs->bad[v], 1);
    }
    if (threadIdx.x == 0) atomic_max_nonneg(&vs->mx[v], mx);
}

// Largest double whose tau_rule is t - 1 (so v > it  <=>  tau_rule(v) >= t),
// for normal binades; negative when t - 1 is not a normal exponent.
__device__ __forceinline__ double tau_floor_threshold(int t) {
    const int e = t - 1;
    if (e < -1022 || e > 1023) return -1.0;
    return from_bits(dbits(pow2(e)) + (uint64_t)tau_threshold(e));
}

struct TreePlan {
    double sig[2][kChainLevels];  // predicted sigma of each level
    unsigned hb[2][kChainLevels]; // level s is proven by a |slice s+1| whose high word exceeds hb
    int ith[2][kChainLevels];     // ... or by a slice s+1 of more than ith grid units (integer form)
    unsigned need[2];             // levels whose prediction must be proven (bit s)
    int tau0[2], G0[2];           // tau of level 0, exponent of its grid
    int z[2], ns[2];              // first all-zero level, slice count (count rule)
    int L, d, valid;
    unsigned magic;               // ceil(2^32 / d): floor(v / d) = umulhi(v, magic) for small v
};

// The plan of x (and y unless `same`) from the first pass's statistics.
__device__ inline void make_plan(const VecStats *vs, int rho, int maxS, bool same, TreePlan &pl) {
    const int d = 54 - rho;
    pl.d = d;
    pl.magic = (unsigned)((0x100000000ULL + (uint64_t)d - 1) / (uint64_t)d);
    pl.valid = 1;
    int L = 0;
    for (int v = 0; v < 2; v++) {
        const int u = same ? 0 : v;
        const double mx = vs->mx[u];
        if (vs->bad[u] || !(mx <= 1.7976931348623157e308)) pl.valid = 0;
        const int tau0 = tau_rule(mx);
        const int G0 = rho + tau0 - 53;
        int z = 0;
        if (vs->lsb[u] != 0) {
            const int num = G0 - (kLsbBias - vs->lsb[u]);
            z = num <= 0 ? 0 : (num + d - 1) / d;
        }
        int ns = (z < 1 ? 1 : z) + 1;  // src/cpu/ozblas_split.cpp:272-289
        if (ns > maxS) ns = maxS;
        if (ns > kChainLevels) pl.valid = 0;
        if (rho + tau0 > 1023 || G0 - (ns - 1) * d < -1022) pl.valid = 0;  // sigma overflow / grid not normal
        for (int s = 0; s < kChainLevels; s++) pl.sig[v][s] = 0.75 * pow2(rho + tau0 - s * d);
        pl.tau0[v] = tau0;
        pl.G0[v] = G0;
        pl.z[v] = z;
        pl.ns[v] = ns;
        L = ns > L ? ns : L;
        // Levels below the first all-zero one that feed a later slice leave a
        // nonzero remainder; each needs one whose tau is the predicted one.
        // |r_s| >= |slice s+1| - g_{s+1} / 2, so |slice s+1| above
        // thr_s + g_{s+1} proves it (high words compared, one unit of slack).
        const int lim = z < ns - 1 ? z : ns - 1;
        pl.need[v] = lim > 0 ? (1u << lim) - 1u : 0u;
        for (int s = 0; s < kChainLevels; s++) {
            pl.hb[v][s] = 0xffffffffu;
            pl.ith[v][s] = 0x7fffffff;
            if (s >= lim) continue;
            const double thr = tau_floor_threshold(tau0 + (s + 1) * (rho - 54));
            if (thr < 0.0) {
                pl.valid = 0;
                continue;
            }
            const double bnd = thr + pow2(G0 - (s + 1) * d);
            pl.hb[v][s] = (unsigned)(dbits(bnd) >> 32) + 1u;
            // |a| g > bnd  <=  |a| > floor(bnd / g), g = 2^(G0 - (s+1) d) (exact scaling, < 2^27)
            const double q = bnd * pow2((s + 1) * d - G0);
            pl.ith[v][s] = q < 2147483647.0 ? (int)floor(q) : 0x7fffffff;
        }
    }
    pl.L = L;
}

// Whether the reference's split of a vector with these statistics is complete
// (the remainder after its last level is zero), from the predicted chain
// tau_{s+1} = tau_s + rho - 54.  The actual chain descends no slower (the
// remainder after level s is at most g_s / 2), so its grids are no coarser
// and its first all-zero level is at most the predicted z: z <= maxS - 1
// makes the split complete whatever the actual chain.  False for Inf / NaN,
// a sigma beyond the double range, or a grid below the normal range (the
// caller then takes a path that follows the reference step by step).
__device__ __forceinline__ bool split_complete(const VecStats &vs, int v, int rho, int maxS) {
    if (vs.bad[v]) return false;
    const double mx = vs.mx[v];
    if (!(mx <= 1.7976931348623157e308)) return false;
    if (vs.lsb[v] == 0) return true;  // every element is zero
    const int tau0 = tau_rule(mx);
    if (rho + tau0 > 1023) return false;
    const int d = 54 - rho, G0 = rho + tau0 - 53;
    const int num = G0 - (kLsbBias - vs.lsb[v]);
    const int z = num <= 0 ? 0 : (num + d - 1) / d;
    return z <= maxS - 1 && G0 - z * d >= -1022;
}

// The plan straight from the first pass's statistics, computed by thread 0
// into shared memory (the caller synchronises the block).  Every CTA of the
// kernel that consumes the statistics does this; its last CTA zeroes them.
__device__ __forceinline__ void plan_in_block(const VecStats *g, int rho, int maxS, bool same, TreePlan &sh) {
    if (threadIdx.x != 0) return;
    VecStats vs;
    for (int v = 0; v < 2; v++) {
        vs.mx[v] = __ldcg(&g->mx[v]);
        vs.lsb[v] = __ldcg(&g->lsb[v]);
        vs.bad[v] = __ldcg(&g->bad[v]);
    }
    make_plan(&vs, rho, maxS, same, sh);
}

// Copy a plan from global memory into shared memory (whole block).
__device__ __forceinline__ void load_plan(const TreePlan *g, TreePlan &sh) {
    static_assert(sizeof(TreePlan) % 4 == 0, "plan layout");
    const unsigned *src = reinterpret_cast<const unsigned *>(g);
    unsigned *dst = reinterpret_cast<unsigned *>(&sh);
    for (int i = threadIdx.x; i < (int)(sizeof(TreePlan) / 4); i += blockDim.x) dst[i] = __ldcg(src + i);
}

// Deepest level that can hold a nonzero slice of an element whose exponent
// field is `key` (0x7ff: the element is zero): its lowest set bit is at least
// key - 1075.
__device__ __forceinline__ int plan_depth(const TreePlan &pl, int v, unsigned key) {
    if (key == 0x7ffu) return 0;
    const int num = pl.G0[v] - ((int)key - 1075);
    return num <= 0 ? 0 : (int)__umulhi((unsigned)(num + pl.d - 1), pl.magic);
}

__device__ __forceinline__ unsigned exp_key(double v) {
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    return b == 0 ? 0x7ffu : (unsigned)(b >> 52);
}

// Warp vote on the pending levels (bit s of `pending`, uniform) of elements
// cut to levels 0..T: returns the levels some lane proves.  Every lane calls
// this with the largest |slice s+1| high word it holds in hw[s].
template <int T>
__device__ __forceinline__ unsigned prove_levels(const unsigned (&hw)[kChainLevels], const unsigned *hb,
                                                 unsigned pending) {
    unsigned got = 0u;
#pragma unroll
    for (int s = 0; s < T; s++)
        if (pending & (1u << s))
            if (__any_sync(0xffffffffu, hw[s] > hb[s])) got |= 1u << s;
    return got;
}

__device__ __forceinline__ unsigned abs_hiword(double v) { return (unsigned)__double2hiint(v) & 0x7fffffffu; }

// Cut v into levels 0..T of the plan's chain (sigmas `sig`), G levels per
// base value: RN_g(b) = (b + sigma) - sigma is exact while |b| <= sigma / 3,
// and slice s = RN_s - RN_{s-1}; the next base is the remainder.
template <int G, int T>
__device__ __forceinline__ void cut_tree(double v, const double *sig, double (&q)[T + 1]) {
    double base = v, prev = 0.0;
#pragma unroll
    for (int s = 0; s <= T; s++) {
        if (s > 0 && (s % G) == 0) {
            base = base - prev;  // remainder after level s - 1
            prev = 0.0;
        }
        const double rn = (base + sig[s]) - sig[s];
        q[s] = rn - prev;
        prev = rn;
    }
}

// Levels per base value for rho: G - 1 <= (rho - 3) / (54 - rho), at most cap.
__host__ __device__ inline int chain_group(int rho, int cap) {
    const int d = 54 - rho;
    int G = d > 0 ? (rho - 3) / d + 1 : 1;
    if (G < 1) G = 1;
    return G > cap ? cap : G;
}

}  // namespace ozb
