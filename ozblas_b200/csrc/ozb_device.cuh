// ozb_device.cuh — device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ozb_rules.cuh"

namespace ozb {

// std::max(a, b) as the reference's split uses it: a unless a < b.
__device__ __forceinline__ double ref_max(double a, double b) { return (a < b) ? b : a; }

// sigma for a dense split level: 0.75 * 2^(rho + tau) * shift
// (src/cpu/ozblas_split.cpp:146, evaluated left to right).
__device__ __forceinline__ double dense_sigma(int rho, double mx, int shift) {
    return 0.75 * pow2(rho + tau_rule(mx)) * (double)shift;
}

// sigma / splitShift for the sparse split (src/cpu/ozblas_split.cpp:809).
// The tuned shift is a power of two, and dividing by 2^k is the same
// correctly rounded scaling as multiplying by 2^-k, so no division is issued;
// any other shift divides.
__device__ __forceinline__ double shift_sigma(double s, int shift) {
    if ((shift & (shift - 1)) == 0 && shift > 0) return s * pow2(-(31 - __clz(shift)));
    return s / (double)shift;
}

// Block-wide max of non-negative doubles; every thread gets the result.
// `red` must hold one double per warp.
__device__ __forceinline__ double block_max_nonneg(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v = ref_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();  // protect red[] from the previous use
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = 0.0;
    for (int i = 0; i < nw; i++) r = ref_max(r, red[i]);
    return r;
}

// Non-negative doubles order like their bit patterns: atomicMax on the bits.
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

// 16-byte asynchronous global -> shared copy (zero fill when !pred).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
// 4- and 8-byte asynchronous copies (through L1), for gathers and small staging.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
// Zero-filling forms: `bytes` (0 or the copy size) are read, the rest of the
// destination is written with zeros.  `gmem` must be a valid address even
// when nothing is read.
__device__ __forceinline__ void cp_async8_zfill(void *smem, const void *gmem, unsigned bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async4_zfill(void *smem, const void *gmem, unsigned bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---- the INT8 form's digits, cut with integer operations ----
// With |x| < 2^E, the digits are the 7-bit groups of |x| 2^-E below the binary
// point, each carrying x's sign: d_s = trunc(x 2^(7(s+1) - E)) - 128 trunc(x 2^(7s - E)).
// |x| 2^-E = M / 2^f exactly, M the 53-bit significand (implicit bit included)
// and f = 1075 + E - (biased exponent, 1 for subnormals), so
// |d_s| = ((M << 7) >> (f - 7 s)) mod 128, which is 0 once f - 7 s leaves
// [0, 64).  These are the digits of the repeated t = 128 r, d = trunc(t),
// r = t - d on r = x 2^-E (exact steps) for every level below 146 (beyond,
// x 2^-E could underflow there).
struct DigitCut {
    uint64_t m7;  // M << 7
    int f;        // shift of digit 0; digit s uses f - 7 s
};

__device__ __forceinline__ DigitCut digit_cut(double x, int E) {
    const uint64_t a = (uint64_t)__double_as_longlong(x) & 0x7fffffffffffffffULL;
    int be = (int)(a >> 52);
    uint64_t M = a & ((1ULL << 52) - 1);
    if (be)
        M |= 1ULL << 52;
    else
        be = 1;
    return DigitCut{M << 7, 1075 + E - be};
}

// |d_s| of a cut, with sh = f - 7 s.
__device__ __forceinline__ uint32_t digit_mag(uint64_t m7, int sh) {
    return (unsigned)sh < 64u ? (uint32_t)(m7 >> sh) & 127u : 0u;
}

// Four packed digit magnitudes (bytes) with the signs applied: the bytes
// selected by `negmask` (0xff where x < 0) become 0 - |d| (two's complement).
__device__ __forceinline__ uint32_t digits_signed(uint32_t w, uint32_t negmask) {
    return (w & ~negmask) | (__vsub4(0u, w) & negmask);
}

}  // namespace ozb
