// ozb_rules.cuh — the integer rules that fix the bits of the Ozaki split.
//
// Shared by host and device code so that one definition is tested on the CPU
// (against glibc, through the exported ozb_rule_* functions) and used by the
// kernels.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define OZB_HD __host__ __device__ __forceinline__
#else
#define OZB_HD inline
#endif

namespace ozb {

OZB_HD uint64_t dbits(double v) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(v);
#else
    uint64_t b;
    __builtin_memcpy(&b, &v, 8);
    return b;
#endif
}

OZB_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}

OZB_HD int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __clz((int)x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}

// ceil(log2(d)) for an integer d >= 1, exactly.
OZB_HD int ceil_log2_int(uint32_t d) { return d <= 1 ? 0 : 32 - clz32(d - 1u); }

// The tau rule's threshold for exponent e: floor(ln2 * 2^(p-1)), p the bit
// length of |e| minus one (one less again just above -2^q, where the spacing
// of doubles halves).  It is a shift of floor(ln2 * 2^40) = 762123384785
// (the floor of a floor is the floor), so there is no table and no branch:
// the values are 1, 2, 5, 11, 22, 44, 88, 177, 354 for p = 2..10 and 0 below.
OZB_HD int64_t tau_threshold(int e) {
    const int ae = e < 0 ? -e : e;
    int p = (ae == 0) ? -1 : (31 - clz32((uint32_t)ae));
    if (e < 0 && (ae & (ae - 1)) == 0) p -= 1;  // just above -2^q the spacing halves
    return (int64_t)(762123384785ULL >> (41 - p));
}

// The split's tau: the reference evaluates (short)ceil(log2(max)) with libm
// (src/cpu/ozblas_split.cpp:145; src/cuda/cuozblas_split.cu:201).  For
// v = 2^e (1 + j 2^-52), log2(v) = e + log2(1 + j 2^-52) is rounded to the
// nearest double; it rounds down onto the integer e exactly when
// log2(1 + j 2^-52) is below half the spacing of doubles just above e, i.e.
// when j <= floor(ln2 * 2^(p-1)) with 2^(p-53) that half spacing.  So the
// result is e when j is at most that threshold (tau_threshold) and e + 1
// otherwise.  The rule is pinned against glibc's log2 over every exponent by
// the CPU tests.
// Zero, infinities and NaN (undefined behaviour in the reference, where it
// never changes a slice) return 0.
OZB_HD int tau_rule(double v) {
    const uint64_t b = dbits(v) & 0x7fffffffffffffffULL;
    const int be = (int)(b >> 52);
    uint64_t j = b & ((1ULL << 52) - 1);
    int e;
    if (be == 0x7ff) return 0;
    if (be == 0) {
        if (j == 0) return 0;
        const int msb = 63 - clz64(j);  // 0..51
        e = msb - 1074;
        j = (j << (52 - msb)) & ((1ULL << 52) - 1);
    } else {
        e = be - 1023;
    }
    if (j == 0) return e;
    return ((int64_t)j <= tau_threshold(e)) ? e : e + 1;
}

// The tau of float data, (short)ceil((float)log2((double)v)) in the reference
// (log21<float>, src/cpu/ozblas_aux.cpp:37-42, calls the double log2).  For
// v = 2^e (1 + j 2^-23) the float nearest to e + log2(1 + j 2^-23) is e when
// log2(1 + j 2^-23) is at most half the spacing of floats just above e, which
// gives the same thresholds in j as the double rule (floor(ln2 2^(p-1))): the
// spacing and j's unit both scale by 2^29.  The double rounding of log2 before
// the float rounding never crosses a threshold: j's nearest integers lie at
// least 0.09 units (2^-26 in log2) from it, against a double spacing of at most
// 2^-45 for |e| <= 149.  Pinned against the reference on every exponent by the
// CPU tests.
OZB_HD int tau_rule_f32(float v) {
#if defined(__CUDA_ARCH__)
    const uint32_t b = (uint32_t)__float_as_int(v) & 0x7fffffffu;
#else
    uint32_t b;
    __builtin_memcpy(&b, &v, 4);
    b &= 0x7fffffffu;
#endif
    const int be = (int)(b >> 23);
    uint32_t j = b & ((1u << 23) - 1);
    int e;
    if (be == 0xff) return 0;
    if (be == 0) {
        if (j == 0) return 0;
        const int msb = 31 - clz32(j);  // 0..22
        e = msb - 149;
        j = (j << (23 - msb)) & ((1u << 23) - 1);
    } else {
        e = be - 127;
    }
    if (j == 0) return e;
    return ((int64_t)j <= tau_threshold(e)) ? e : e + 1;
}

// rho = ceil(53 - (53 - log2(dim)) / 2) for splitEpsMode 0
// (src/cpu/ozblas_split.cpp:19-34) as an exact integer rule: the smallest r
// with 2^(2r - 53) >= dim.  Mode 9 ("overflow" variant) is
// ceil(27 + log2(dim) / 4); mode 2 (Dot2) is ceil(log2(dim) / 2).
OZB_HD int rho_rule(int dim, int splitEpsMode) {
    const int L = ceil_log2_int(dim < 1 ? 1u : (uint32_t)dim);
    if (splitEpsMode == 9) return 27 + (L + 3) / 4;
    if (splitEpsMode == 2) return (L + 1) / 2;
    const int t = (L & 1) ? L : L + 1;
    return (t + 53) / 2;
}

OZB_HD double from_bits(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double v;
    __builtin_memcpy(&v, &b, 8);
    return v;
#endif
}

// 2^e exactly as scalbn(1., e) gives it (subnormal below -1022, 0 below
// -1074, +inf above 1023).
OZB_HD double pow2(int e) {
    if (e > 1023) return from_bits(0x7ff0000000000000ULL);
    if (e >= -1022) return from_bits((uint64_t)(e + 1023) << 52);
    if (e >= -1074) return from_bits(1ULL << (e + 1074));
    return 0.0;
}

// v * 2^e rounded once to nearest, ties to even, as glibc's scalbn gives it
// (exact unless the result is subnormal; overflow to infinity), in integer
// arithmetic: no floating-point step that the compiler could fuse with the
// caller's following addition.  Zero, infinities and NaN pass through.
OZB_HD double scale2(double v, int e) {
    const uint64_t b = dbits(v);
    const uint64_t sign = b & 0x8000000000000000ULL;
    const int be = (int)((b >> 52) & 0x7ff);
    uint64_t M = b & ((1ULL << 52) - 1);
    if (be == 0x7ff || (b << 1) == 0) return v;
    int t;  // biased exponent of the result for significand M with the implicit bit at 2^52
    if (be == 0) {  // subnormal input: normalise
        const int msb = 63 - clz64(M);  // < 52
        M <<= (52 - msb);
        t = 1 - (52 - msb) + e;
    } else {
        M |= 1ULL << 52;
        t = be + e;
    }
    if (t > 2046) return from_bits(sign | 0x7ff0000000000000ULL);
    if (t >= 1) return from_bits(sign | ((uint64_t)t << 52) | (M & ((1ULL << 52) - 1)));
    const int sh = 1 - t;  // onto the subnormal grid 2^-1074
    if (sh > 54) return from_bits(sign);
    uint64_t q = M >> sh;
    const uint64_t rest = M & ((1ULL << sh) - 1), half = 1ULL << (sh - 1);
    if (rest > half || (rest == half && (q & 1))) q += 1;  // q = 2^52 is the smallest normal: same bits
    return from_bits(sign | q);
}

}  // namespace ozb
