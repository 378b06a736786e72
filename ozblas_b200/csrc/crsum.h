// crsum.h — certified fast path of the correctly rounded sum.
//
// NearSum (Rump, Ogita, Oishi; src/cpu/ozblas_sum.cpp:10-112) returns the
// double nearest to the exact sum of its terms.  That value is unique unless
// the exact sum is a midpoint between two doubles, so any method that finds
// it, and can prove that it found it, gives the same bits.  CrSum adds the
// terms with a cascade of TwoSums (Knuth): s + sum(q_i) equals the exact sum,
// e = fl(sum q_i) and a = fl(sum |q_i|).  With (r, err) = TwoSum(s, e) the
// exact sum is r + err + delta, |delta| <= gamma_{m-1} sum|q_i| <= c * a for
// c = 2^(ceil(log2 m) - 52).  If |err| + c * a is below half the gap between
// r and its neighbours (a quarter ulp on the side of a power of two), r is the
// nearest double.  When the test fails (a midpoint or a near-midpoint, a zero
// or tiny result, Inf / NaN, very large or very small error terms), the
// caller runs the reference's NearSum.  The same code runs on the host, where
// the tests compare it with the NearSum restatement.
#pragma once
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define OZB_HD __host__ __device__ __forceinline__
#else
#define OZB_HD inline
#endif

namespace ozb {

OZB_HD uint64_t crs_bits(double v) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(v);
#else
    uint64_t b;
    memcpy(&b, &v, 8);
    return b;
#endif
}

OZB_HD double crs_from_bits(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double v;
    memcpy(&v, &b, 8);
    return v;
#endif
}

struct CrSum {
    double s, e, a;
    int m;

    OZB_HD CrSum() : s(0.0), e(0.0), a(0.0), m(0) {}

    // TwoSum(s, p): s + p = t + q exactly (six additions, no branch).
    OZB_HD void add(double p) {
        const double t = s + p;
        const double bp = t - s;
        const double q = (s - (t - bp)) + (p - bp);
        s = t;
        e = e + q;
        a = a + (q < 0.0 ? -q : q);
        m++;
    }

    // True, with `out` the nearest double to the exact sum, when proven.
    OZB_HD bool finish(double &out) const {
        // a must be zero or comfortably normal, so that c * a is exact
        if (!(a == 0.0 || (a >= 0x1p-900 && a <= 0x1p+900))) return false;
        const double r = s + e;
        const double bp = r - s;
        const double err = (s - (r - bp)) + (e - bp);
        const uint64_t rb = crs_bits(r) & 0x7fffffffffffffffULL;
        const int ex = (int)(rb >> 52);
        if (ex < 64 || ex >= 0x7ff) return false;  // zero or tiny (|r| < 2^-959), Inf, NaN
        const bool pow2 = (rb & 0x000fffffffffffffULL) == 0;
        const double h = crs_from_bits((uint64_t)(ex - 53 - (pow2 ? 1 : 0)) << 52);
        const double ae = err < 0.0 ? -err : err;
        if (!(ae < h)) return false;
        int lg = 1;  // ceil(log2(max(m, 2)))
        while ((1 << lg) < m) lg++;
        const double c = crs_from_bits((uint64_t)(1023 + lg - 52) << 52);
        if (!(a * c < 0.5 * (h - ae))) return false;
        out = r;
        return true;
    }
};

}  // namespace ozb
