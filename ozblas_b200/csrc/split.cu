// split.cu — error-free extraction of FP64 slices (the "plain" Ozaki split).
//
// Arithmetic of every level (src/cpu/ozblas_split.cpp:137-178 dense,
// :62-103 vector, :779-815 sparse):
//   tau   = ceil(log2(max|r|))            (tau_rule: glibc's rounding)
//   sigma = 0.75 * 2^(rho+tau) * shift    (sparse: / shift)
//   slice = (r + sigma) - sigma;  r -= slice;  new max = max|r|
// Termination (src/cpu/ozblas_split.cpp:272-289): level 0 always runs;
// levels 1.. run until one leaves every remainder zero (that level counts)
// or maxS levels exist.  With z = the first level whose remainder is zero
// for a line, the count is min(maxS, max(1, max_lines z) + 1).
#include <cooperative_groups.h>

#include "ozb_device.cuh"
#include "ozb_internal.h"

namespace cg = cooperative_groups;

namespace ozb {

constexpr int kSplitThreads = 256;
constexpr int kSplitSmemMaxK = 26 * 1024;  // doubles kept on chip per line (208 KB)

// How a slice is stored.  Plain form: the FP64 slice itself.  Mixed form
// <double, float, float> (src/cpu/ozblas_split.cpp:181-221): scalbn(slice,
// -tau) in FP32, exact because a slice has at most 53 - rho <= 12 significant
// bits on the grid 2^(rho + tau - 53), with tau kept per line and level.
template <typename SL>
__device__ __forceinline__ SL slice_store(double sl, int tau);
template <>
__device__ __forceinline__ double slice_store<double>(double sl, int) {
    return sl;
}
template <>
__device__ __forceinline__ float slice_store<float>(double sl, int tau) {
    return (float)scalbn(sl, -tau);
}

// One CTA per line.  COUNT: atomicMax(*zmax, z_line).  WRITE: ns slices
// (and, for FP32 slices, tau of every level at exps[level * nl + line]).
// `rem` is either dynamic shared memory (k <= kSplitSmemMaxK) or a global
// scratch line of k doubles per CTA.
template <bool WRITE, typename SL = double>
__global__ void __launch_bounds__(kSplitThreads) k_split_lines(int k, int nl, const double *__restrict__ X, int ldx,
                                                               int rho, int levels, SL *__restrict__ out, int ldo,
                                                               short *__restrict__ exps,
                                                               double *__restrict__ gscratch,
                                                               int *__restrict__ zmax) {
    extern __shared__ double smem[];
    __shared__ double red[kSplitThreads / 32];
    const int line = blockIdx.x;
    if (line >= nl) return;
    double *rem = gscratch ? gscratch + (size_t)line * k : smem;
    const double *x = X + (size_t)line * ldx;
    double mx = 0.0;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double v = x[i];
        rem[i] = v;
        mx = ref_max(mx, fabs(v));
    }
    mx = block_max_nonneg(mx, red);
    int z = levels;  // COUNT: first level leaving a zero remainder (levels = maxS-1 cap)
    for (int s = 0; s < levels; s++) {
        const int tau = tau_rule(mx);
        const double sigma = 0.75 * pow2(rho + tau);  // dense_sigma(rho, mx, 1)
        double nm = 0.0;
        SL *o = WRITE ? out + ((size_t)s * nl + line) * ldo : nullptr;
        if (WRITE && exps && threadIdx.x == 0) exps[(size_t)s * nl + line] = (short)tau;
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            double r = rem[i];
            const double sl = (r + sigma) - sigma;
            r = r - sl;
            rem[i] = r;
            nm = ref_max(nm, fabs(r));
            if (WRITE) o[i] = slice_store<SL>(sl, tau);
        }
        if (WRITE)
            for (int i = k + threadIdx.x; i < ldo; i += blockDim.x) o[i] = (SL)0;
        mx = block_max_nonneg(nm, red);
        if (!WRITE && mx == 0.0) {
            z = s;
            break;
        }
    }
    if (!WRITE && threadIdx.x == 0) atomicMax(zmax, z);
}

template <typename SL>
static int launch_split_lines(cuozblasHandle_t *h, bool write, int k, int nl, const double *X, int ldx, int rho,
                              int levels, SL *out, int ldo, short *exps, int *zmax_dev) {
    State *st = state(h);
    double *gscratch = nullptr;
    size_t smem = 0;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    if (k > kSplitSmemMaxK) {
        gscratch = ar.take<double>((uint64_t)k * nl);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    } else {
        smem = sizeof(double) * (size_t)(k > 0 ? k : 1);
    }
    if (write) {
        OZB_CHECK(cudaFuncSetAttribute(k_split_lines<true, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kSplitSmemMaxK * sizeof(double))));
        counted(h);
        k_split_lines<true, SL><<<nl, kSplitThreads, smem, st->stream>>>(k, nl, X, ldx, rho, levels, out, ldo, exps,
                                                                         gscratch, nullptr);
    } else {
        OZB_CHECK(cudaFuncSetAttribute(k_split_lines<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kSplitSmemMaxK * sizeof(double))));
        counted(h);
        k_split_lines<false, double><<<nl, kSplitThreads, smem, st->stream>>>(k, nl, X, ldx, rho, levels, nullptr, 0,
                                                                      nullptr, gscratch, zmax_dev);
    }
    OZB_CHECK(cudaGetLastError());
    ar.release(mk);
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_lines_count(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int maxS, int *ns) {
    State *st = state(h);
    if (maxS <= 1 || nl == 0) {
        *ns = (nl == 0) ? (maxS < 2 ? maxS : 2) : 1;
        if (maxS <= 1) *ns = 1;
        return CUOZBLAS_STATUS_SUCCESS;
    }
    OZB_CHECK(cudaMemsetAsync(st->d_ints, 0, sizeof(int), st->stream));
    OZB_TRY(launch_split_lines<double>(h, false, k, nl, X, ldx, rho, maxS - 1, nullptr, 0, nullptr, st->d_ints));
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, st->d_ints, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    int zmax = st->h_ints[0];
    int c = (zmax < 1 ? 1 : zmax) + 1;
    *ns = c < maxS ? c : maxS;
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_lines_write(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, double *out,
                      int ldo) {
    if (nl == 0 || ns == 0) return CUOZBLAS_STATUS_SUCCESS;
    return launch_split_lines<double>(h, true, k, nl, X, ldx, rho, ns, out, ldo, nullptr, nullptr);
}

int split_lines_write_e(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, double *out,
                        int ldo, short *exps) {
    if (nl == 0 || ns == 0) return CUOZBLAS_STATUS_SUCCESS;
    return launch_split_lines<double>(h, true, k, nl, X, ldx, rho, ns, out, ldo, exps, nullptr);
}

int split_lines_write_f32(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, float *out,
                          int ldo, short *exps) {
    if (nl == 0 || ns == 0) return CUOZBLAS_STATUS_SUCCESS;
    return launch_split_lines<float>(h, true, k, nl, X, ldx, rho, ns, out, ldo, exps, nullptr);
}

// ---------------------------------------------------------------------------
// Transpose (column-major rows x cols -> cols x rows), 32x32 tiles.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void transpose_tile(int rows, int cols, const T *__restrict__ A, int lda,
                                               T *__restrict__ out, int ldo) {
    __shared__ T t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int r = r0 + threadIdx.x, c = c0 + j;
        t[j][threadIdx.x] = (r < rows && c < cols) ? A[(size_t)c * lda + r] : (T)0;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = c0 + threadIdx.x, r = r0 + j;
        if (r < rows && c < cols) out[(size_t)r * ldo + c] = t[threadIdx.x][j];
    }
}

__global__ void k_transpose(int rows, int cols, const double *__restrict__ A, int lda, double *__restrict__ out,
                            int ldo) {
    transpose_tile<double>(rows, cols, A, lda, out, ldo);
}

__global__ void k_transpose_f32(int rows, int cols, const float *__restrict__ A, int lda, float *__restrict__ out,
                                int ldo) {
    transpose_tile<float>(rows, cols, A, lda, out, ldo);
}

int transpose(cuozblasHandle_t *h, int rows, int cols, const double *A, int lda, double *out, int ldo) {
    if (rows == 0 || cols == 0) return CUOZBLAS_STATUS_SUCCESS;
    dim3 grid((rows + 31) / 32, (cols + 31) / 32), block(32, 8);
    counted(h);
    k_transpose<<<grid, block, 0, state(h)->stream>>>(rows, cols, A, lda, out, ldo);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

int transpose_f32(cuozblasHandle_t *h, int rows, int cols, const float *A, int lda, float *out, int ldo) {
    if (rows == 0 || cols == 0) return CUOZBLAS_STATUS_SUCCESS;
    dim3 grid((rows + 31) / 32, (cols + 31) / 32), block(32, 8);
    counted(h);
    k_transpose_f32<<<grid, block, 0, state(h)->stream>>>(rows, cols, A, lda, out, ldo);
    OZB_CHECK(cudaGetLastError());
    return CUOZBLAS_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Float data, FP64 slices: the mixed form <float, double, double>
// (src/cpu/ozblas_split.cpp:181-221 with TYPE1 = float).  The arithmetic is
// the reference's float arithmetic: tau = ceil((float)log2((double)max))
// (tau_rule_f32), sigma = (float)(0.75 * (float)2^(rho+tau) * shift),
// slice = (r + sigma) - sigma and r -= slice in float, and the slice stored
// as the double scalbn(slice, -tau) with tau at exps[level * nl + line].
// rho may be negative (k < 32).  One CTA per line, as k_split_lines; `rem`
// holds floats.  COUNT: atomicMax(*zmax, z_line).  WRITE: ns slices.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sd_sigma(int rho, int tau) {
    const float p = (float)pow2(rho + tau);  // (float)scalbn(1., rho + tau)
    return (float)(0.75 * (double)p);
}

template <bool WRITE>
__global__ void __launch_bounds__(kSplitThreads) k_split_lines_sd(int k, int nl, const float *__restrict__ X, int ldx,
                                                                  int rho, int levels, double *__restrict__ out,
                                                                  int ldo, short *__restrict__ exps,
                                                                  float *__restrict__ gscratch,
                                                                  int *__restrict__ zmax) {
    extern __shared__ float fsmem[];
    __shared__ double red[kSplitThreads / 32];
    const int line = blockIdx.x;
    if (line >= nl) return;
    float *rem = gscratch ? gscratch + (size_t)line * k : fsmem;
    const float *x = X + (size_t)line * ldx;
    float mx = 0.f;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const float v = x[i];
        rem[i] = v;
        const float av = fabsf(v);
        mx = (mx < av) ? av : mx;
    }
    mx = (float)block_max_nonneg((double)mx, red);  // exact: a max of floats
    int z = levels;
    for (int s = 0; s < levels; s++) {
        const int tau = tau_rule_f32(mx);
        const float sigma = sd_sigma(rho, tau);
        float nm = 0.f;
        double *o = WRITE ? out + ((size_t)s * nl + line) * ldo : nullptr;
        if (WRITE && threadIdx.x == 0) exps[(size_t)s * nl + line] = (short)tau;
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            float r = rem[i];
            const float sl = __fsub_rn(__fadd_rn(r, sigma), sigma);
            r = __fsub_rn(r, sl);
            rem[i] = r;
            const float ar = fabsf(r);
            nm = (nm < ar) ? ar : nm;
            if (WRITE) o[i] = scalbn((double)sl, -tau);  // exact, and exactly a float
        }
        if (WRITE)
            for (int i = k + threadIdx.x; i < ldo; i += blockDim.x) o[i] = 0.0;
        mx = (float)block_max_nonneg((double)nm, red);
        if (!WRITE && mx == 0.f) {
            z = s;
            break;
        }
    }
    if (!WRITE && threadIdx.x == 0) atomicMax(zmax, z);
}

static int launch_split_lines_sd(cuozblasHandle_t *h, bool write, int k, int nl, const float *X, int ldx, int rho,
                                 int levels, double *out, int ldo, short *exps, int *zmax_dev) {
    State *st = state(h);
    float *gscratch = nullptr;
    size_t smem = 0;
    Arena ar(h);
    const uint64_t mk = ar.mark();
    if (k > 2 * kSplitSmemMaxK) {
        gscratch = ar.take<float>((uint64_t)k * nl);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    } else {
        smem = sizeof(float) * (size_t)(k > 0 ? k : 1);
    }
    const int maxsmem = (int)(2 * kSplitSmemMaxK * sizeof(float));
    if (write) {
        OZB_CHECK(cudaFuncSetAttribute(k_split_lines_sd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem));
        counted(h);
        k_split_lines_sd<true><<<nl, kSplitThreads, smem, st->stream>>>(k, nl, X, ldx, rho, levels, out, ldo, exps,
                                                                         gscratch, nullptr);
    } else {
        OZB_CHECK(cudaFuncSetAttribute(k_split_lines_sd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem));
        counted(h);
        k_split_lines_sd<false><<<nl, kSplitThreads, smem, st->stream>>>(k, nl, X, ldx, rho, levels, nullptr, 0,
                                                                          nullptr, gscratch, zmax_dev);
    }
    OZB_CHECK(cudaGetLastError());
    ar.release(mk);
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_lines_count_sd(cuozblasHandle_t *h, int k, int nl, const float *X, int ldx, int rho, int maxS, int *ns) {
    State *st = state(h);
    if (maxS <= 1 || nl == 0) {
        *ns = (nl == 0) ? (maxS < 2 ? maxS : 2) : 1;
        if (maxS <= 1) *ns = 1;
        return CUOZBLAS_STATUS_SUCCESS;
    }
    OZB_CHECK(cudaMemsetAsync(st->d_ints, 0, sizeof(int), st->stream));
    OZB_TRY(launch_split_lines_sd(h, false, k, nl, X, ldx, rho, maxS - 1, nullptr, 0, nullptr, st->d_ints));
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, st->d_ints, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    const int zmax = st->h_ints[0];
    const int c = (zmax < 1 ? 1 : zmax) + 1;
    *ns = c < maxS ? c : maxS;
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_lines_write_sd(cuozblasHandle_t *h, int k, int nl, const float *X, int ldx, int rho, int ns, double *out,
                         int ldo, short *exps) {
    if (nl == 0 || ns == 0) return CUOZBLAS_STATUS_SUCCESS;
    return launch_split_lines_sd(h, true, k, nl, X, ldx, rho, ns, out, ldo, exps, nullptr);
}

// ---------------------------------------------------------------------------
// Vector split: one global tau chain (src/cpu/ozblas_split.cpp:62-103 and the
// driver :254-289 with n = 1).  One cooperative launch runs every level; the
// grid syncs after each level's max reduction.  rem: n doubles of scratch.
// slot[s] = max|remainder| entering level s (slot[0] = max|x|); *ns_out is
// written by block 0, and for FP32 slices exps[s] = tau of level s.
// ---------------------------------------------------------------------------
template <typename SL>
__global__ void __launch_bounds__(256) k_split_vector(int n, const double *__restrict__ x, int rho, int maxS,
                                                      SL *__restrict__ out, int ldo, short *__restrict__ exps,
                                                      double *__restrict__ rem, double *__restrict__ slot,
                                                      int *__restrict__ ns_out) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double red[8];
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double m = 0.0;
    for (size_t i = tid; i < (size_t)n; i += stride) m = ref_max(m, fabs(x[i]));
    m = block_max_nonneg(m, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&slot[0], m);
    grid.sync();
    int s = 0;
    for (; s < maxS; s++) {
        const double mx = slot[s];
        if (s >= 2 && slot[s] == 0.0) break;  // previous level left nothing: the count is s
        const int tau = tau_rule(mx);
        const double sigma = 0.75 * pow2(rho + tau);  // dense_sigma(rho, mx, 1)
        const double *src = (s == 0) ? x : rem;
        SL *o = out + (size_t)s * ldo;
        if (exps && tid == 0) exps[s] = (short)tau;
        double nm = 0.0;
        for (size_t i = tid; i < (size_t)n; i += stride) {
            double r = src[i];
            const double sl = (r + sigma) - sigma;
            r = r - sl;
            rem[i] = r;
            o[i] = slice_store<SL>(sl, tau);
            nm = ref_max(nm, fabs(r));
        }
        for (size_t i = (size_t)n + tid; i < (size_t)ldo; i += stride) o[i] = (SL)0;
        nm = block_max_nonneg(nm, red);
        if (threadIdx.x == 0) atomic_max_nonneg(&slot[s + 1], nm);
        grid.sync();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *ns_out = s;
}

template <typename SL>
static int split_vector_t(cuozblasHandle_t *h, int n, const double *x, int rho, int maxS, SL *out, int ldo,
                          short *exps, int *ns) {
    State *st = state(h);
    Arena ar(h);
    const uint64_t mk = ar.mark();
    double *rem = ar.take<double>(n > 0 ? n : 1);
    double *slot = ar.take<double>(kMaxSplitDefault + 2);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemsetAsync(slot, 0, sizeof(double) * (kMaxSplitDefault + 2), st->stream));
    int dev = 0, nsm = 0, per = 0;
    OZB_CHECK(cudaGetDevice(&dev));
    OZB_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    OZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_split_vector<SL>, 256, 0));
    int blocks = nsm * (per < 4 ? per : 4);
    const int need = (n + 255) / 256;
    if (blocks > need) blocks = need > 0 ? need : 1;
    int *ns_dev = st->d_ints;
    void *args[] = {&n, &x, &rho, &maxS, &out, &ldo, &exps, &rem, &slot, &ns_dev};
    counted(h);
    OZB_CHECK(cudaLaunchCooperativeKernel((void *)k_split_vector<SL>, dim3(blocks), dim3(256), args, 0, st->stream));
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, ns_dev, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    *ns = st->h_ints[0];
    ar.release(mk);
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_vector(cuozblasHandle_t *h, int n, const double *x, int rho, int maxS, double *out, int ldo, int *ns) {
    return split_vector_t<double>(h, n, x, rho, maxS, out, ldo, nullptr, ns);
}

int split_vector_f32(cuozblasHandle_t *h, int n, const double *x, int rho, int maxS, float *out, int ldo, short *exps,
                     int *ns) {
    return split_vector_t<float>(h, n, x, rho, maxS, out, ldo, exps, ns);
}

// ---------------------------------------------------------------------------
// CSR row split (src/cpu/ozblas_split.cpp:779-815, driver :875-928): one warp
// per row; rho from the row's nnz; sigma divided by shift.  Remainders live
// in `rem` (nnz doubles).  COUNT atomicMax(z); WRITE writes ns slices of nnz.
// ---------------------------------------------------------------------------
template <bool WRITE>
__global__ void __launch_bounds__(256) k_split_csr(int m, const double *__restrict__ val,
                                                   const int *__restrict__ rowptr, int epsmode, int shift,
                                                   int levels, double *__restrict__ rem, double *__restrict__ out,
                                                   int64_t ldo, int *__restrict__ zmax) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= m) return;
    const int lo = rowptr[warp], hi = rowptr[warp + 1];
    double mx = 0.0;
    for (int i = lo + lane; i < hi; i += 32) {
        const double v = val[i];
        rem[i] = v;
        mx = ref_max(mx, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) mx = ref_max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int z = levels;
    if (hi > lo) {
        const int rho = rho_rule(hi - lo, epsmode);
        for (int s = 0; s < levels; s++) {
            const double sigma = shift_sigma(0.75 * pow2(rho + tau_rule(mx)), shift);
            double nm = 0.0;
            for (int i = lo + lane; i < hi; i += 32) {
                double r = rem[i];
                const double sl = (r + sigma) - sigma;
                r = r - sl;
                rem[i] = r;
                nm = ref_max(nm, fabs(r));
                if (WRITE) out[(size_t)s * ldo + i] = sl;
            }
            for (int o = 16; o > 0; o >>= 1) nm = ref_max(nm, __shfl_xor_sync(0xffffffffu, nm, o));
            mx = nm;
            if (!WRITE && mx == 0.0) {
                z = s;
                break;
            }
        }
    } else {
        z = 0;
    }
    if (!WRITE && lane == 0) atomicMax(zmax, z);
}

int split_csr_count(cuozblasHandle_t *h, int m, const double *val, const int *rowptr, int epsmode, int shift,
                    int maxS, int *ns) {
    State *st = state(h);
    if (maxS <= 1) {
        *ns = 1;
        return CUOZBLAS_STATUS_SUCCESS;
    }
    int nnz = 0;
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, rowptr + m, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    nnz = st->h_ints[0];
    Arena ar(h);
    const uint64_t mk = ar.mark();
    double *rem = ar.take<double>(nnz > 0 ? nnz : 1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_CHECK(cudaMemsetAsync(st->d_ints, 0, sizeof(int), st->stream));
    const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
    if (m > 0) {
        counted(h);
        k_split_csr<false><<<blocks, 256, 0, st->stream>>>(m, val, rowptr, epsmode, shift, maxS - 1, rem, nullptr, 0,
                                                           st->d_ints);
    }
    OZB_CHECK(cudaGetLastError());
    OZB_CHECK(cudaMemcpyAsync(st->h_ints, st->d_ints, sizeof(int), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    const int zmax = st->h_ints[0];
    const int c = (zmax < 1 ? 1 : zmax) + 1;
    *ns = c < maxS ? c : maxS;
    ar.release(mk);
    return CUOZBLAS_STATUS_SUCCESS;
}

int split_csr_write(cuozblasHandle_t *h, int m, int nnz, const double *val, const int *rowptr, int epsmode,
                    int shift, int ns, double *out, int64_t ld) {
    State *st = state(h);
    Arena ar(h);
    const uint64_t mk = ar.mark();
    double *rem = ar.take<double>(nnz > 0 ? nnz : 1);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const int blocks = (int)(((int64_t)m * 32 + 255) / 256);
    if (m > 0) {
        counted(h);
        k_split_csr<true><<<blocks, 256, 0, st->stream>>>(m, val, rowptr, epsmode, shift, ns, rem, out, ld,
                                                          nullptr);
    }
    OZB_CHECK(cudaGetLastError());
    ar.release(mk);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb
