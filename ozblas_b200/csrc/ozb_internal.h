// ozb_internal.h — host-side state shared by the library's translation units.
#pragma once
#include <chrono>
#include <string.h>
#include <atomic>
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/cuozblas.h"
#include "ozb_rules.cuh"

namespace ozb {

constexpr int kMaxSplitDefault = 30;  // NumSplitDefaultMax, src/cuda/cuozblas_common.h:5
constexpr size_t kPersistBytes = 256 << 10;  // State::d_persist
constexpr int kArenaAlign = 256;

// Diagnostic switches from the environment, read when a handle is created
// (and again by cuozblasHandleReadEnv), never on a call path.  Each selects an
// equal-bits alternative path or a trace on stderr.
struct EnvSwitches {
    bool gemv_split = false;   // OZBLAS_GEMV_SPLIT: GEMV 'n' over materialised slices
    bool gemv_levels = false;  // OZBLAS_GEMV_LEVELS: fused GEMV with one read of A per level
    bool plain_dmma = false;   // OZBLAS_PLAIN_DMMA: plain GEMM pair products on DMMA
    bool sd_dmma = false;      // OZBLAS_SD_DMMA: <float,double,double> products on DMMA
    bool q_dmma = false;       // OZBLAS_Q_DMMA: quad-form products on DMMA
    bool ds_simt = false;      // OZBLAS_DS_SIMT: <double,float,float> on the FP32 SIMT kernel
    bool dot_tree = false;     // OZBLAS_DOT_TREE: DOT pass 2 on the FP64 tree
    bool dot_two_pass = false; // OZBLAS_DOT_TWO_PASS: NearSum DOT on the two-pass path
    bool csr_slices = false;   // OZBLAS_CSR_SLICES: NearSum CSRMV rows through their slices
    bool gemv_slices = false;  // OZBLAS_GEMV_SLICES: NearSum GEMV 'n' through its slices
    bool i8_levelwise = false; // OZBLAS_I8_LEVELWISE: the INT8 form's products level by level (k_i8_gemm)
    bool g_split3 = false;     // OZBLAS_GROUPED_SPLIT3: the grouped INT8 split as three launches
    int i8_block = 0;          // OZBLAS_I8_BLOCK: levels per block of the level-blocked INT8 kernel (1-4; -4..-1: cut across runs; 0: measured)
    bool cg_no_graph = false;  // OZBLAS_CG_NO_GRAPH: CG iterations on the host loop
    bool dot_trace = false;    // OZBLAS_DOT_TRACE
    bool cg_trace = false;     // OZBLAS_CG_TRACE
    void read();
};

// Per-handle private state; the reference handle's hstBatchAddr field points
// here (the batched-GEMM pointer arrays it held in the reference have no
// counterpart in this library).
struct State {
    cudaStream_t stream = 0;
    uint64_t off = 0;             // bump pointer into h->devWork
    uint64_t high_water = 0;
    int *d_ints = nullptr;        // small device int scratch (counters, error word)
    int *h_ints = nullptr;        // pinned host mirror
    char *h_stage = nullptr;      // pinned staging for schedule uploads (kStageBytes)
    int *h_mail = nullptr;        // pinned, device-mapped: counts a running kernel posts to the host (kMailInts)
    int *d_mail = nullptr;        // its device address
    int mail_seq = 0;             // the last post's tag
    double *h_dbl = nullptr;      // pinned host doubles (scalar results)
    int last_error = 0;
    int64_t splitA_ld = 0;        // slice stride of the pre-split A (cuozblasDcsrmvSplitA)
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // phase timers (split A/B, products, sum)
    bool plain_timers = false;    // ev[0..4] hold a plain-form call's phases, read at the call's end
    uint64_t launches = 0;        // kernels this handle has launched (cuozblasGetLaunchCount)
    // Device scratch that lives as long as the handle (zeroed at create; every
    // kernel that uses it leaves it zeroed): the one-pass DOT's statistics,
    // block parts and tickets, so a call needs no memset.
    void *d_persist = nullptr;
    EnvSwitches env;
    // The matrix of the last fused CSRMV and the level count its rows needed:
    // the next call on the same matrix holds that many levels per row on chip
    // (rows that need more go to the per-row kernel, so a stale count costs
    // only speed).
    struct {
        const void *val = nullptr, *colind = nullptr, *rowptr = nullptr;
        int m = -1, n = -1, nnz = -1, flags = 0, nA = 0;
    } csr_memo;
};


inline State *state(cuozblasHandle_t *h) { return reinterpret_cast<State *>(h->hstBatchAddr); }

// Count one kernel launch on the handle (every <<<>>> site calls this).
inline void counted(cuozblasHandle_t *h) { state(h)->launches++; }

// Phase timers of the reference handle (t_SplitA, t_SplitB, t_comp), taken
// with CUDA events on the handle's stream; read after the call's final sync.
inline void ev_record(cuozblasHandle_t *h, int i) { cudaEventRecord(state(h)->ev[i], state(h)->stream); }
inline float ev_ms(cuozblasHandle_t *h, int a, int b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, state(h)->ev[a], state(h)->ev[b]) != cudaSuccess) return 0.f;
    return ms;
}

// The device span of a call's kernels as the exec info's t_comp (events 0-2
// before the first launch, 3-4 after the last, read at the call's end).
inline void span_begin(cuozblasHandle_t *h) {
    for (int i = 0; i < 3; i++) ev_record(h, i);
}
inline void span_end(cuozblasHandle_t *h) {
    ev_record(h, 3);
    ev_record(h, 4);
    state(h)->plain_timers = true;
}

// Pinned staging of a handle, for host -> device uploads of schedules: a copy
// from pinned memory is a plain asynchronous DMA, one from pageable memory is
// staged by the driver on the calling thread.
constexpr size_t kStageBytes = size_t(8) << 20;
constexpr int kMailInts = 16384;

// Monotonic wall clock (s), for bounded host waits.
inline double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Upload `bytes` from host `src` to device `dst` on the handle's stream
// through the staging buffer when it has room (`used`: staging bytes this call
// has taken, 0 at its first upload, which first waits for the stream so that
// no earlier copy still reads the buffer), else straight from `src`.
inline cudaError_t stage_upload(State *st, void *dst, const void *src, size_t bytes, size_t &used) {
    if (bytes == 0) return cudaSuccess;
    const size_t at = (used + 15) & ~size_t(15);
    if (st->h_stage && at + bytes <= kStageBytes) {
        if (used == 0) {
            const cudaError_t e = cudaStreamSynchronize(st->stream);
            if (e != cudaSuccess) return e;
        }
        memcpy(st->h_stage + at, src, bytes);
        used = at + bytes;
        return cudaMemcpyAsync(dst, st->h_stage + at, bytes, cudaMemcpyHostToDevice, st->stream);
    }
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st->stream);
}

// Bump allocation from the handle's arena (no cudaMalloc on the call path).
struct Arena {
    cuozblasHandle_t *h;
    State *st;
    bool ok = true;
    explicit Arena(cuozblasHandle_t *hh) : h(hh), st(state(hh)) {}
    template <typename T>
    T *take(uint64_t count) {
        uint64_t bytes = count * sizeof(T);
        uint64_t start = (st->off + kArenaAlign - 1) / kArenaAlign * kArenaAlign;
        if (start + bytes > h->workSizeBytes) {
            ok = false;
            return nullptr;
        }
        st->off = start + bytes;
        if (st->off > st->high_water) st->high_water = st->off;
        h->memAddr = st->off;
        return reinterpret_cast<T *>(h->devWork + start);
    }
    uint64_t mark() const { return st->off; }
    void release(uint64_t m) { st->off = m; }
};

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR; }

#define OZB_CHECK(call)                                                     \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) {                                            \
            fprintf(stderr, "cuozblas: CUDA error %s at %s:%d\n",           \
                    cudaGetErrorString(_e), __FILE__, __LINE__);            \
            return CUOZBLAS_STATUS_CUDA_ERROR;                              \
        }                                                                   \
    } while (0)

#define OZB_TRY(expr)                               \
    do {                                            \
        int _s = (expr);                            \
        if (_s != CUOZBLAS_STATUS_SUCCESS) return _s; \
    } while (0)

inline bool is_trans(char t) { return !(t == 'n' || t == 'N'); }

// Streaming multiprocessors of the current device (cached per device).
inline int sm_count() {
    int dev = 0;
    cudaGetDevice(&dev);
    static int cache[64] = {0};
    if (dev >= 0 && dev < 64 && cache[dev] > 0) return cache[dev];
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n < 1) n = 1;
    if (dev >= 0 && dev < 64) cache[dev] = n;
    return n;
}

// Opt a kernel into `bytes` of dynamic shared memory on the current device.
// The attribute belongs to each device's context, so `done` keeps one bit per
// device (devices 64 and up set it on every call); concurrent first calls on
// one device both set it, which is harmless.
inline cudaError_t smem_optin(const void *func, int bytes, std::atomic<uint64_t> &done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t)1 << dev : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// Reference counterInit (src/cuda/cuozblas.cpp:3-21): resets the exec info,
// splitShift and the arena pointer (keeping a pre-split A below memMaskSplitA).
int counter_init(cuozblasHandle_t *h);

// ---- split (split.cu) ----
// Lines: `nl` lines of length k, line l at X + l*ldx (contiguous).  Returns
// the split count in *ns (reference termination rule) and, when `out` is
// non-null, writes ns slices of nl lines of ldo doubles (zero padded).
int split_lines_count(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int maxS, int *ns);
int split_lines_write(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, double *out,
                      int ldo);
// As split_lines_write, also recording tau of every level at exps[level * nl + line].
int split_lines_write_e(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, double *out,
                        int ldo, short *exps);
// Mixed form <double, float, float>: FP32 slices scalbn(slice, -tau) with tau
// per level at exps[level * nl + line] (lines) or exps[level] (vector).
int split_lines_write_f32(cuozblasHandle_t *h, int k, int nl, const double *X, int ldx, int rho, int ns, float *out,
                          int ldo, short *exps);
int split_vector_f32(cuozblasHandle_t *h, int n, const double *x, int rho, int maxS, float *out, int ldo, short *exps,
                     int *ns);
// Mixed form <float, double, double>: float data split in float arithmetic into
// FP64 slices scalbn(slice, -tau), tau at exps[level * nl + line].
int split_lines_count_sd(cuozblasHandle_t *h, int k, int nl, const float *X, int ldx, int rho, int maxS, int *ns);
int split_lines_write_sd(cuozblasHandle_t *h, int k, int nl, const float *X, int ldx, int rho, int ns, double *out,
                         int ldo, short *exps);
int transpose_f32(cuozblasHandle_t *h, int rows, int cols, const float *A, int lda, float *out, int ldo);
// Transpose rows x cols (column-major, ld) into cols x rows (ldo).
int transpose(cuozblasHandle_t *h, int rows, int cols, const double *A, int lda, double *out, int ldo);
// Vector split with one global tau chain (n-vector).  Writes ns slices of ldo.
int split_vector(cuozblasHandle_t *h, int n, const double *x, int rho, int maxS, double *out, int ldo, int *ns);
// CSR row split; slices laid out ns x nnz.  shift divides sigma.
int split_csr_count(cuozblasHandle_t *h, int m, const double *val, const int *rowptr, int epsmode, int shift,
                    int maxS, int *ns);
int split_csr_write(cuozblasHandle_t *h, int m, int nnz, const double *val, const int *rowptr, int epsmode,
                    int shift, int ns, double *out, int64_t ld);

// Copy n elements of esz (4, 8 or 16) bytes, `stride` elements apart, to a
// contiguous array (csrmv.cu).
int gather_strided(cuozblasHandle_t *h, int n, const void *src, int64_t stride, int esz, void *dst);

// ---- sums ----
int fsum_pairs_dot(cuozblasHandle_t *h, int nA, int nB, int maxlevel, const double *pairmat, double alpha,
                   double beta, double *out_dev);

// ---- mixed form <double, float, float> (gemm_f32.cu) ----
int rho_rule_f32(int dim, int splitEpsMode);
int gemm_f32_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                  const double *B, int ldb, double beta, double *C, int ldc, int fastMode);

// <double, float, float> with INT8 slices on tcgen05 (gemm_i8.cu), for rho >= 47
int gemm_ds_i8_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta, double *C, int ldc, int rho, int fastMode,
                    int *nA, int *nB, int *np);

// ---- mixed form <float, double, double> (gemm_plain.cu: the FP64-slice engine) ----
int rho_rule_sd(int dim, int splitEpsMode);
int gemm_sd_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int fastMode);

// ---- exact FP64 pair products for the quad form (gemm_plain.cu) ----
int gemm_pairs_store(cuozblasHandle_t *h, int m, int nc, int nlB, int ldk, const double *Sa, const double *Sb,
                     const int2 *dp, int np, double *pbuf);
int pair_products_skinny(cuozblasHandle_t *h, bool dot, int m, int k, int nA, int nB, const double *Sa,
                         const double *Sb, int ldk, double *P);

// exact FP64 pair products of int8-digit slices on tcgen05 (gemm_i8.cu)
int i8_exact_pairs(cuozblasHandle_t *h, int m, int n, int k_pad, const int8_t *digA, int lpadA, int planesA,
                   const int8_t *digB, int lpadB, int planesB, int D, const std::vector<int2> &pairs, int sbias,
                   const short *eas, const short *ebs, double *pbuf);

// ---- quad I/O form <__float128, double, double> (gemm_q.cu); binary128 as 16 bytes ----
int gemm_q_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, const void *alpha, const void *A, int lda,
                const void *B, int ldb, const void *beta, void *C, int ldc, int fastMode);

// ---- skinny forms (gemm_plain.cu, gemv_fused.cu) ----
int sum_rows_launch(cuozblasHandle_t *h, int m, int nA, int nB, int maxlevel, double *P, int64_t ldp, double alpha,
                    double beta, double *y, double *scratch);
int gemv_fused_n(cuozblasHandle_t *h, int m, int n, const double *A, int lda, const double *xs, int ldx, int nB,
                 int rho, int maxS, int fastMode, double alpha, double beta, double *y, int *nA_out);
int gemv_rn_n(cuozblasHandle_t *h, int m, int n, const double *A, int lda, const double *x, double alpha, double beta,
              double *y, bool *done, int *nA, int *nB);

// ---- plain GEMM core (gemm_plain.cu) ----
int gemm_plain_core(cuozblasHandle_t *h, char ta, char tb, int m, int n, int k, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta, double *C, int ldc, int fastMode);

}  // namespace ozb
