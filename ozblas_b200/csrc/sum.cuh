// sum.cuh — the two summations of slice-pair products.
//
// FSum (sumMode 0): t = 0; t += P(ia, ib) for ik = 0..maxlevel ascending,
// ia ascending, ib = ik - ia (src/cpu/ozblas_sum.cpp:331-380; the storage
// index "sumOrder" of the reference does not change this order).
// NearSum (sumMode 1): Rump–Ogita–Oishi correctly rounded sum
// (src/cpu/ozblas_sum.cpp:10-112), restated below over terms at a stride.
// Both end with C = fma(alpha, t, beta * C) (src/cpu/ozblas_sum.cpp:366).
#pragma once
#include "crsum.h"
#include "ozb_device.cuh"

namespace ozb {

// Iterate the pair set in summation order.
template <typename F>
__host__ __device__ __forceinline__ void for_each_pair(int nA, int nB, int maxlevel, F f) {
    for (int ik = 0; ik <= maxlevel; ik++) {
        const int lo = ik - (nB - 1) > 0 ? ik - (nB - 1) : 0;
        const int hi = ik < nA - 1 ? ik : nA - 1;
        for (int ia = lo; ia <= hi; ia++) f(ia, ik - ia);
    }
}

__device__ __forceinline__ double sign1(double v) { return (v < 0) ? -1. : 1.; }

// ExtractVector-based transform, src/cpu/ozblas_sum.cpp:10-57.
__device__ inline void ns_transform(int n, double *v, int64_t ld, double rho, double &tau1, double &tau2) {
    const int emin = -1022, epse = 53;
    if (n == 0) {
        tau1 = rho;
        tau2 = 0.;
        return;
    }
    double mu = fabs(v[0]);
    for (int i = 1; i < n; i++) {
        const double a = fabs(v[i * ld]);
        mu = (mu > a) ? mu : a;
    }
    if (mu == 0.) {
        tau1 = rho;
        tau2 = 0.;
        return;
    }
    const int M = ceil_log2_int((uint32_t)(n + 2));
    double sigma = pow2(M + tau_rule(mu));
    double t = rho;
    for (;;) {
        double tau = 0.;
        for (int i = 0; i < n; i++) {
            const double tmp = (sigma + v[i * ld]) - sigma;
            v[i * ld] -= tmp;
            tau += tmp;
        }
        tau1 = t + tau;
        if ((sigma <= pow2(emin)) || (fabs(tau1) >= pow2(2 * M + 1 - epse) * sigma)) {
            tau2 = tau - (tau1 - t);
            return;
        }
        sigma = pow2(M - epse) * sigma;
        t = tau1;
    }
}

__device__ inline void ns_transformk(int n, double *v, int64_t ld, double rho, double &res, double &r) {
    double tmp = 0., tau1, tau2;
    ns_transform(n, v, ld, rho, tau1, tau2);
    for (int i = 0; i < n; i++) tmp += v[i * ld];
    res = tau1 + (tau2 + tmp);
    r = tau2 - (res - tau1);
}

// Correctly rounded sum of n terms at stride ld; the terms are overwritten
// when the certified fast path (crsum.h) cannot prove its result.
__device__ inline double nearsum(int n, double *v, int64_t ld) {
    {
        CrSum cs;
        for (int i = 0; i < n; i++) cs.add(v[i * ld]);
        double out;
        if (cs.finish(out)) return out;
    }
    const double eps = pow2(-53);
    double res, r, delta, r2, res2, mu, delta2, tmp;
    ns_transformk(n, v, ld, 0., res, r);
    ns_transformk(n, v, ld, r, delta, r2);
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
    ns_transformk(n, v, ld, r2, delta2, tmp);
    if (delta2 == 0) return res + mu;
    if (sign1(delta2) == sign1(mu)) return res2;
    return res;
}

}  // namespace ozb
