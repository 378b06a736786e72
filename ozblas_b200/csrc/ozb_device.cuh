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

}  // namespace ozb
