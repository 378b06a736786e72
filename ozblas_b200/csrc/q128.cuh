// q128.cuh — IEEE binary128 in software, for the quad I/O form
// <__float128, double, double> (src/cpu/ozblas_gemm.cpp:316 and the
// binary128 helpers of src/cpu/ozblas_aux.cpp: scalbnq, fmaq, log2q).
//
// A value is kept as its 16 bytes (the layout of __float128 on x86-64: low
// 64 bits first).  Every operation here is exact or rounds once to nearest,
// ties to even, as IEEE 754 binary128 does: an exact result is formed as
// sign x N x 2^e with N a 256-bit integer (plus a sticky bit for the part
// of an addend that lies entirely below N's last bit), and round_pack()
// rounds it to 113 bits with gradual underflow and overflow to infinity.
// The same code runs on the host, where the tests compare it with gcc's
// __float128 arithmetic and libquadmath's fmaq.
#pragma once
#include <stdint.h>

#include "ozb_rules.cuh"

namespace ozb {

struct Q128 {
    uint64_t lo, hi;
};

typedef unsigned __int128 u128;

struct U256 {
    u128 lo, hi;
};

constexpr int kQBias = 16383;
constexpr int kQMinLsb = -16494;  // exponent of the last bit of the smallest subnormal

OZB_HD Q128 q_make(uint64_t hi, uint64_t lo) {
    Q128 r;
    r.lo = lo;
    r.hi = hi;
    return r;
}
OZB_HD Q128 q_zero(int sign) { return q_make((uint64_t)sign << 63, 0); }
OZB_HD Q128 q_inf(int sign) { return q_make(((uint64_t)sign << 63) | 0x7fff000000000000ULL, 0); }
OZB_HD Q128 q_nan() { return q_make(0x7fff800000000000ULL, 0); }
OZB_HD int q_sign(Q128 x) { return (int)(x.hi >> 63); }
OZB_HD int q_bexp(Q128 x) { return (int)((x.hi >> 48) & 0x7fff); }
OZB_HD bool q_is_zero(Q128 x) { return ((x.hi << 1) | x.lo) == 0; }
OZB_HD bool q_is_special(Q128 x) { return q_bexp(x) == 0x7fff; }
OZB_HD bool q_is_nan(Q128 x) { return q_is_special(x) && (((x.hi & 0xffffffffffffULL) | x.lo) != 0); }
OZB_HD Q128 q_abs(Q128 x) { return q_make(x.hi & 0x7fffffffffffffffULL, x.lo); }
OZB_HD Q128 q_neg(Q128 x) { return q_make(x.hi ^ 0x8000000000000000ULL, x.lo); }

// |a| < |b| for non-NaN values (the magnitudes order like their bit patterns).
OZB_HD bool q_mag_less(Q128 a, Q128 b) {
    const uint64_t ah = a.hi & 0x7fffffffffffffffULL, bh = b.hi & 0x7fffffffffffffffULL;
    return ah < bh || (ah == bh && a.lo < b.lo);
}

// x = (-1)^sign * m * 2^e with m < 2^113 (finite x).
OZB_HD void q_decode(Q128 x, int &sign, int &e, u128 &m) {
    sign = q_sign(x);
    const int be = q_bexp(x);
    const u128 frac = ((u128)(x.hi & 0xffffffffffffULL) << 64) | x.lo;
    if (be == 0) {
        m = frac;
        e = kQMinLsb;
    } else {
        m = frac | ((u128)1 << 112);
        e = be - kQBias - 112;
    }
}

OZB_HD int clz128(u128 v) {
    const uint64_t h = (uint64_t)(v >> 64);
    return h ? clz64(h) : 64 + clz64((uint64_t)v);
}
OZB_HD int bitlen128(u128 v) { return v ? 128 - clz128(v) : 0; }
OZB_HD int bitlen256(U256 v) { return v.hi ? 128 + bitlen128(v.hi) : bitlen128(v.lo); }
OZB_HD bool u256_zero(U256 v) { return v.hi == 0 && v.lo == 0; }
OZB_HD U256 u256(u128 v) {
    U256 r;
    r.hi = 0;
    r.lo = v;
    return r;
}

OZB_HD U256 u256_shl(U256 v, int s) {  // 0 <= s < 256, no bits lost by the caller's choice
    U256 r;
    if (s == 0) return v;
    if (s >= 128) {
        r.hi = v.lo << (s - 128);
        r.lo = 0;
    } else {
        r.hi = (v.hi << s) | (v.lo >> (128 - s));
        r.lo = v.lo << s;
    }
    return r;
}

// v >> s; *lost = whether any one bit was shifted out.
OZB_HD U256 u256_shr(U256 v, int s, bool *lost) {
    U256 r;
    if (s <= 0) {
        *lost = false;
        return v;
    }
    if (s >= 256) {
        *lost = !u256_zero(v);
        r.hi = r.lo = 0;
        return r;
    }
    if (s >= 128) {
        const int t = s - 128;
        *lost = (v.lo != 0) || (t > 0 && (v.hi << (128 - t)) != 0);
        r.lo = t ? (v.hi >> t) : v.hi;
        r.hi = 0;
    } else {
        *lost = (v.lo << (128 - s)) != 0;
        r.lo = (v.lo >> s) | (v.hi << (128 - s));
        r.hi = v.hi >> s;
    }
    return r;
}

OZB_HD U256 u256_add(U256 a, U256 b) {
    U256 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1 : 0);
    return r;
}
OZB_HD U256 u256_sub(U256 a, U256 b) {  // a >= b
    U256 r;
    r.lo = a.lo - b.lo;
    r.hi = a.hi - b.hi - (a.lo < b.lo ? 1 : 0);
    return r;
}
OZB_HD bool u256_less(U256 a, U256 b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

// 113 x 113-bit product, exact.
OZB_HD U256 mul113(u128 a, u128 b) {
    const uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64), b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
    const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
    U256 r = u256(p00);
    r = u256_add(r, u256_shl(u256(p01), 64));
    r = u256_add(r, u256_shl(u256(p10), 64));
    U256 h;
    h.hi = p11;
    h.lo = 0;
    return u256_add(r, h);
}

// Round sign * (N + f) * 2^e to binary128, nearest with ties to even, where
// 0 < f < 1 when `sticky` is set and f = 0 otherwise.  Callers set sticky only
// with N of at least 254 bits, so f always lies below the rounding bit.
OZB_HD Q128 q_round_pack(int sign, U256 N, int e, bool sticky) {
    if (u256_zero(N) && !sticky) return q_zero(sign);
    const int L = bitlen256(N);
    int s = L - 113;                 // right shift that leaves 113 bits
    if (e + s < kQMinLsb) s = kQMinLsb - e;  // gradual underflow: fewer bits
    u128 q;
    int lsb;
    if (s <= 0) {  // exact: shift left
        q = (u128)N.lo << (-s);
        lsb = e + s;
    } else {
        bool below = false;
        const U256 t = u256_shr(N, s - 1, &below);  // t = N >> (s - 1): last bit is the half bit
        const bool half = (t.lo & 1) != 0;
        q = (t.lo >> 1) | (t.hi << 127);
        const bool rest = below || sticky;
        if (half && (rest || (q & 1))) q += 1;
        lsb = e + s;
        if (q >> 113) {  // carried into a 114th bit
            q >>= 1;
            lsb += 1;
        }
    }
    if (q == 0) return q_zero(sign);
    if (q >> 112) {  // normal
        const int be = lsb + 112 + kQBias;
        if (be >= 0x7fff) return q_inf(sign);
        return q_make(((uint64_t)sign << 63) | ((uint64_t)be << 48) | ((uint64_t)(q >> 64) & 0xffffffffffffULL),
                      (uint64_t)q);
    }
    // subnormal (lsb == kQMinLsb)
    return q_make(((uint64_t)sign << 63) | ((uint64_t)(q >> 64) & 0xffffffffffffULL), (uint64_t)q);
}

// Exact sum of two signed 256-bit magnitudes at a common exponent, with a
// sticky part of the second: sa*A + sb*(B + f), 0 < f < 1 if sticky.
OZB_HD Q128 q_sum_pack(int sa, U256 A, int sb, U256 B, bool sticky, int e) {
    if (sa == sb) return q_round_pack(sa, u256_add(A, B), e, sticky);
    // A - (B + f): if A > B: (A - B - 1) + (1 - f); if A <= B the result has B's sign
    if (u256_less(B, A)) {
        if (!sticky) return q_round_pack(sa, u256_sub(A, B), e, false);
        U256 one = u256(1);
        return q_round_pack(sa, u256_sub(u256_sub(A, B), one), e, true);
    }
    if (!sticky) {
        const U256 d = u256_sub(B, A);
        if (u256_zero(d)) return q_zero(0);  // exact zero: +0 when rounding to nearest
        return q_round_pack(sb, d, e, false);
    }
    return q_round_pack(sb, u256_sub(B, A), e, true);  // (B + f) - A
}

// Align two exact values sx*X*2^ex and sy*Y*2^ey (bit lengths <= 226 and
// <= 113 or the reverse) and add them, rounding once.
OZB_HD Q128 q_add_exact(int sx, U256 X, int ex, int sy, U256 Y, int ey) {
    if (u256_zero(X)) {
        if (u256_zero(Y)) return q_zero(sx & sy);
        return q_round_pack(sy, Y, ey, false);
    }
    if (u256_zero(Y)) return q_round_pack(sx, X, ex, false);
    // make X the one with the higher top bit
    const int tx = ex + bitlen256(X), ty = ey + bitlen256(Y);
    if (ty > tx) {
        const int ts = sx;
        sx = sy;
        sy = ts;
        const U256 tv = X;
        X = Y;
        Y = tv;
        const int te = ex;
        ex = ey;
        ey = te;
    }
    // put X's top bit at bit 254 (one bit of headroom for the carry of X + Y)
    const int sh = 255 - bitlen256(X);
    X = u256_shl(X, sh);
    const int e = ex - sh;
    if (ey >= e) {  // Y fits exactly above e (its top is not above X's)
        Y = u256_shl(Y, ey - e);
        return q_sum_pack(sx, X, sy, Y, false, e);
    }
    bool lost = false;
    Y = u256_shr(Y, e - ey, &lost);
    return q_sum_pack(sx, X, sy, Y, lost, e);
}

OZB_HD Q128 q_add(Q128 a, Q128 b) {
    if (q_is_special(a) || q_is_special(b)) {
        if (q_is_nan(a) || q_is_nan(b)) return q_nan();
        if (q_is_special(a) && q_is_special(b)) return q_sign(a) == q_sign(b) ? a : q_nan();
        return q_is_special(a) ? a : b;
    }
    int sa, sb, ea, eb;
    u128 ma, mb;
    q_decode(a, sa, ea, ma);
    q_decode(b, sb, eb, mb);
    if (ma == 0 && mb == 0) return q_zero(sa & sb);
    return q_add_exact(sa, u256(ma), ea, sb, u256(mb), eb);
}

OZB_HD Q128 q_mul(Q128 a, Q128 b) {
    const int s = q_sign(a) ^ q_sign(b);
    if (q_is_special(a) || q_is_special(b)) {
        if (q_is_nan(a) || q_is_nan(b)) return q_nan();
        if (q_is_zero(a) || q_is_zero(b)) return q_nan();
        return q_inf(s);
    }
    int sa, sb, ea, eb;
    u128 ma, mb;
    q_decode(a, sa, ea, ma);
    q_decode(b, sb, eb, mb);
    if (ma == 0 || mb == 0) return q_zero(s);
    return q_round_pack(s, mul113(ma, mb), ea + eb, false);
}

// fma(a, b, c) = a * b + c rounded once.
OZB_HD Q128 q_fma(Q128 a, Q128 b, Q128 c) {
    const int sp = q_sign(a) ^ q_sign(b);
    if (q_is_special(a) || q_is_special(b) || q_is_special(c)) {
        if (q_is_nan(a) || q_is_nan(b) || q_is_nan(c)) return q_nan();
        if (q_is_special(a) || q_is_special(b)) {
            if (q_is_zero(a) || q_is_zero(b)) return q_nan();
            if (q_is_special(c) && q_sign(c) != sp) return q_nan();
            return q_inf(sp);
        }
        return c;
    }
    int sa, sb, sc, ea, eb, ec;
    u128 ma, mb, mc;
    q_decode(a, sa, ea, ma);
    q_decode(b, sb, eb, mb);
    q_decode(c, sc, ec, mc);
    if (ma == 0 || mb == 0) {
        if (mc == 0) return q_zero(sp & sc);
        return c;
    }
    if (mc == 0) return q_round_pack(sp, mul113(ma, mb), ea + eb, false);
    return q_add_exact(sp, mul113(ma, mb), ea + eb, sc, u256(mc), ec);
}

// (binary128) d * 2^k for a finite double d: exact for the exponent range
// the form produces (the double's 53 bits always fit; the scaling only
// rounds in binary128's subnormal range, as scalbnq does).
OZB_HD Q128 q_from_double_scaled(double d, int k) {
    const uint64_t b = dbits(d);
    const int s = (int)(b >> 63);
    const int be = (int)((b >> 52) & 0x7ff);
    uint64_t m = b & ((1ULL << 52) - 1);
    int e;
    if (be == 0) {
        if (m == 0) return q_zero(s);
        e = -1074;
    } else {
        m |= (1ULL << 52);
        e = be - 1075;
    }
    return q_round_pack(s, u256((u128)m), e + k, false);
}

// The double nearest to x (ties to even; gradual underflow; overflow to inf).
OZB_HD double q_to_double_rn(Q128 x) {
    const int s = q_sign(x);
    if (q_is_special(x)) {
        if (q_is_nan(x)) return from_bits(0x7ff8000000000000ULL);
        return from_bits(((uint64_t)s << 63) | 0x7ff0000000000000ULL);
    }
    int sg, e;
    u128 m;
    q_decode(x, sg, e, m);
    if (m == 0) return from_bits((uint64_t)s << 63);
    const int L = bitlen128(m);
    int sh = L - 53;
    if (e + sh < -1074) sh = -1074 - e;  // double subnormal range
    uint64_t q;
    int lsb;
    if (sh <= 0) {
        q = (uint64_t)(m << (-sh));
        lsb = e + sh;
    } else if (sh > 120) {
        return from_bits((uint64_t)s << 63);  // far below the smallest subnormal
    } else {
        const u128 t = m >> sh;
        const u128 rest = m - (t << sh);
        const u128 half = (u128)1 << (sh - 1);
        q = (uint64_t)t;
        if (rest > half || (rest == half && (q & 1))) q += 1;
        lsb = e + sh;
        if (q >> 53) {
            q >>= 1;
            lsb += 1;
        }
    }
    if (q == 0) return from_bits((uint64_t)s << 63);
    if (q >> 52) {
        const int be = lsb + 52 + 1023;
        if (be >= 0x7ff) return from_bits(((uint64_t)s << 63) | 0x7ff0000000000000ULL);
        return from_bits(((uint64_t)s << 63) | ((uint64_t)be << 52) | (q & ((1ULL << 52) - 1)));
    }
    return from_bits(((uint64_t)s << 63) | q);
}

// The split of the quad form (src/cpu/ozblas_split.cpp:181-221 with
// TYPE1 = __float128): sigma = 0.75 * 2^(rho + tau), slice = (x + sigma) -
// sigma, x -= slice.  For |x| <= 2^tau and rho >= 2, x + sigma stays in
// sigma's binade, so the slice is x rounded to the nearest multiple of
// g = 2^(rho + tau - 113), ties to even (sigma / g = 3 * 2^111 is even), and
// the remainder is exact.  Returns the slice as the double
// scalbnq(slice, -tau) = q * 2^(rho - 113) and replaces x by the remainder.
OZB_HD double q_split(Q128 &x, int rho, int tau) {
    int s, e;
    u128 m;
    q_decode(x, s, e, m);
    if (m == 0) return 0.0;  // (+-0 + sigma) - sigma = +0; the remainder keeps its sign
    const int gexp = rho + tau - 113;
    u128 q;
    if (e >= gexp) {  // x is a multiple of g: all of it goes to the slice
        q = m << (e - gexp);
        x = q_zero(0);
    } else {
        const int sh = gexp - e;
        if (sh > 114) {  // |x| < g / 2: nothing goes to the slice
            return 0.0;
        }
        q = m >> sh;
        const u128 rest = m - (q << sh);
        const u128 half = (u128)1 << (sh - 1);
        if (rest > half || (rest == half && (q & 1))) q += 1;
        // remainder m - q 2^sh (signed), at exponent e
        const u128 qs = q << sh;
        if (qs >= m) {
            const u128 r = qs - m;
            x = q_round_pack(s ^ 1, u256(r), e, false);
            if (r == 0) x = q_zero(0);
        } else {
            x = q_round_pack(s, u256(m - qs), e, false);
        }
    }
    if (q == 0) return 0.0;  // a slice that rounds to zero is +0, as (x + sigma) - sigma
    // q * 2^(rho - 113), q < 2^(114 - rho) fits a double exactly
    const double v = (double)(uint64_t)q * pow2(rho - 113);
    return s ? -v : v;
}

// tau = (short)ceil(log21(max)) for binary128 data.  The reference's
// ceil(log21(v)) resolves to the double ceil of log2q(v) converted to double
// (src/cpu/ozblas_split.cpp:201; ozblas_aux.cpp:43-46), so for
// v = 2^e (1 + j 2^-112) the result is e while log2q(v) rounds to the double
// e, i.e. while log2(1 + j 2^-112) is below half the spacing of doubles next
// to e, and e + 1 after.  The largest such j depends only on the binade of e
// (q = floor(log2 |e|), one class lower just above -2^q, as for the double
// rule); the table holds it for q = -1..13, found by bisection against the
// reference library and checked on every exponent by the CPU tests.
OZB_HD u128 tau_q_threshold(int e) {
    const int ae = e < 0 ? -e : e;
    if (ae == 0) return 0;
    int q = 31 - clz32((uint32_t)ae);
    if (e < 0 && (ae & (ae - 1)) == 0) q -= 1;
    switch (q) {
        case -1: return ((u128)0x0ULL << 64) | 0x02c5c85fdf473deaULL;
        case 0: return ((u128)0x0ULL << 64) | 0x058b90bfbe8e7bddULL;
        case 1: return ((u128)0x0ULL << 64) | 0x0b17217f7d1cf7d8ULL;
        case 2: return ((u128)0x0ULL << 64) | 0x162e42fefa39f02cULL;
        case 3: return ((u128)0x0ULL << 64) | 0x2c5c85fdf473e245ULL;
        case 4: return ((u128)0x0ULL << 64) | 0x58b90bfbe8e7cc3bULL;
        case 5: return ((u128)0x0ULL << 64) | 0xb17217f7d1cfb736ULL;
        case 6: return ((u128)0x1ULL << 64) | 0x62e42fefa39fe96bULL;
        case 7: return ((u128)0x2ULL << 64) | 0xc5c85fdf4741bed3ULL;
        case 8: return ((u128)0x5ULL << 64) | 0x8b90bfbe8e8b2d96ULL;
        case 9: return ((u128)0xbULL << 64) | 0x17217f7d1d351aeaULL;
        case 10: return ((u128)0x16ULL << 64) | 0x2e42fefa3ae534ccULL;
        case 11: return ((u128)0x2cULL << 64) | 0x5c85fdf477b66578ULL;
        case 12: return ((u128)0x58ULL << 64) | 0xb90bfbe8f71cba70ULL;
        case 13: return ((u128)0xb1ULL << 64) | 0x7217f7d20cf932e0ULL;
        default: return 0;
    }
}

// tau of a binary128 value (zero, infinities and NaN give 0).
OZB_HD int tau_rule_q(Q128 v) {
    const int be = q_bexp(v);
    if (be == 0x7fff) return 0;
    u128 j = ((u128)(v.hi & 0xffffffffffffULL) << 64) | v.lo;
    int e;
    if (be == 0) {
        if (j == 0) return 0;
        const int msb = 127 - clz128(j);  // 0..111
        e = msb - 16494;
        j = (j << (112 - msb)) & (((u128)1 << 112) - 1);
    } else {
        e = be - kQBias;
    }
    if (j == 0) return e;
    return (j <= tau_q_threshold(e)) ? e : e + 1;
}

}  // namespace ozb
