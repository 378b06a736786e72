// eft.cuh — error-free transformations for the Dot2 mode (splitEpsMode 2),
// as the reference defines them (src/cpu/eft.h:11-19 TwoSum, :51-57
// QuickTwoSum, :75-81 TwoProdFMA, :99-107 Dot2i, :129-137 QuadAdd, :166-174
// QuadMul).  Every product that feeds an addition is an explicitly rounded
// multiply, so the compiler cannot contract it into an fma.
#pragma once
#include <cuda_runtime.h>

namespace ozb {

struct DD {
    double x, y;
};

__device__ __forceinline__ void eft_two_sum(double a, double b, double &s, double &e) {
    const double ss = __dadd_rn(a, b);
    const double v = __dsub_rn(ss, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(ss, v)), __dsub_rn(b, v));
    s = ss;
}

__device__ __forceinline__ void eft_quick_two_sum(double a, double b, double &s, double &e) {
    const double ss = __dadd_rn(a, b);
    e = __dsub_rn(b, __dsub_rn(ss, a));
    s = ss;
}

// c += a * b in double-double (Dot2i)
__device__ __forceinline__ void eft_dot2i(double a, double b, DD &c) {
    const double h = __dmul_rn(a, b);
    const double r = fma(a, b, -h);
    double q;
    eft_two_sum(c.x, h, c.x, q);
    c.y = __dadd_rn(c.y, __dadd_rn(q, r));
}

__device__ __forceinline__ DD eft_quad_add(DD a, DD b) {
    DD t, c;
    eft_two_sum(a.x, b.x, t.x, t.y);
    t.y = __dadd_rn(t.y, __dadd_rn(a.y, b.y));
    eft_quick_two_sum(t.x, t.y, c.x, c.y);
    return c;
}

__device__ __forceinline__ DD eft_quad_mul(double a, DD b) {
    DD t, c;
    t.x = __dmul_rn(a, b.x);
    t.y = fma(a, b.x, -t.x);
    t.y = fma(a, b.y, t.y);
    eft_quick_two_sum(t.x, t.y, c.x, c.y);
    return c;
}

}  // namespace ozb
