// api.cu — the C ABI of include/cuozblas.h: handle lifecycle and the
// BLAS-level entry points of the plain (FP64-slice) form.
#include <functional>
#include <vector>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <new>

#include "crsum.h"
#include "q128.cuh"
#include "ozb_internal.h"

namespace ozb {
int launch_axpy(cuozblasHandle_t *h, int n, double alpha, const double *x, double *y);
int launch_scal(cuozblasHandle_t *h, int n, double alpha, double *x);
constexpr int kNrm2PlainScratch = 257;  // 256 block partials + the result
int launch_nrm2_plain(cuozblasHandle_t *h, int n, const double *x, double *scratch);
int launch_csrmv_plain(cuozblasHandle_t *h, int m, const double *val, const int *colind, const int *rowptr,
                       const double *x, double alpha, double beta, double *y);
int csrmv_presplit(cuozblasHandle_t *h, int m, int n, double alpha, const double *As, int nA, int64_t ld_s,
                   const int *colind, const int *rowptr, const double *x, double beta, double *y);
int dot_fused(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret, bool *done, int *nA,
              int *nB);
int dot_exact(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret, bool *done, int *nA,
              int *nB);
int csrmv_fused(cuozblasHandle_t *h, int m, int n, double alpha, const double *val, const int *colind,
                const int *rowptr, const double *x, double beta, double *y, int shift, int na_hint, bool *done,
                int *nA_out, int *nB_out);
int cg_graph(cuozblasHandle_t *h, int n, const double *val, const int *colind, const int *rowptr, double *x,
             double *r, double *p, double *q, double nrmb, double tol, int maxiter, int shift, int na_hint,
             double &dold, int &iter, bool &stop, double t1, double *res, double *when,
             const std::function<int()> &host_head, const std::function<int(bool &)> &host_tail,
             const std::function<double()> &wall_now);

// CSRMV exec info as the reference records it (src/cpu/ozblas_csrmv.cpp:104-119)
static void csrmv_info(cuozblasHandle_t *h, int nA, int nB) {
    h->nSplitA = (float)nA;
    h->nSplitB = (float)nB;
    int maxlevel = (nA - 1) + (nB - 1);
    const int mn = nA - 1 < nB - 1 ? nA - 1 : nB - 1;
    maxlevel = (maxlevel - h->fastMode) > mn ? (maxlevel - h->fastMode) : mn;
    int ic = 0;
    for (int ia = 0; ia < (maxlevel + 1 < nA ? maxlevel + 1 : nA); ia++)
        ic += (nB < maxlevel + 1 - ia ? nB : maxlevel + 1 - ia);
    h->nSplitC = (float)ic;
}

static double wall() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

static bool env_on(const char *name) {
    const char *v = getenv(name);
    return v != nullptr && *v != '\0' && strcmp(v, "0") != 0;
}

void EnvSwitches::read() {
    gemv_split = env_on("OZBLAS_GEMV_SPLIT");
    gemv_levels = env_on("OZBLAS_GEMV_LEVELS");
    plain_dmma = env_on("OZBLAS_PLAIN_DMMA");
    sd_dmma = env_on("OZBLAS_SD_DMMA");
    q_dmma = env_on("OZBLAS_Q_DMMA");
    ds_simt = env_on("OZBLAS_DS_SIMT");
    dot_tree = env_on("OZBLAS_DOT_TREE");
    dot_two_pass = env_on("OZBLAS_DOT_TWO_PASS");
    csr_slices = env_on("OZBLAS_CSR_SLICES");
    gemv_slices = env_on("OZBLAS_GEMV_SLICES");
    i8_levelwise = env_on("OZBLAS_I8_LEVELWISE");
    g_split3 = env_on("OZBLAS_GROUPED_SPLIT3");
    {
        const char *v = getenv("OZBLAS_I8_BLOCK");
        i8_block = v ? atoi(v) : 0;
        if (i8_block < -4 || i8_block > 4) i8_block = 0;
    }
    cg_no_graph = env_on("OZBLAS_CG_NO_GRAPH");
    dot_trace = env_on("OZBLAS_DOT_TRACE");
    cg_trace = env_on("OZBLAS_CG_TRACE");
}

int counter_init(cuozblasHandle_t *h) {
    if (h == nullptr || h->initialized == 0 || state(h) == nullptr) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    h->splitShift = 1;
    h->t_SplitA = h->t_SplitB = h->t_comp = h->t_sum = h->t_total = 0.f;
    h->nSplitA = h->nSplitB = h->nSplitC = 0.f;
    h->mbk = h->nbk = 0;
    h->n_comp = 0.f;
    state(h)->off = h->memMaskSplitA;
    h->memAddr = h->memMaskSplitA;
    return CUOZBLAS_STATUS_SUCCESS;
}

// splitEpsMode 2 (Dot2) exists for DOT, NRM2, CSRMV and CG only, with
// fastMode 0 (the reference's DOT takes its Dot2 branch only then, and its
// CSRMV stores and sums Dot2 pairs inconsistently otherwise).
static int check_flags(cuozblasHandle_t *h, bool dot2 = false) {
    if (h->splitEpsMode == 2 && !(dot2 && h->fastMode == 0)) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (h->splitEpsMode != 0 && h->splitEpsMode != 9 && h->splitEpsMode != 2) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (h->sumMode != 0 && h->sumMode != 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (h->nSplitMax < 0 || h->nSplitMax > kMaxSplitDefault) return CUOZBLAS_STATUS_INVALID_VALUE;
    return CUOZBLAS_STATUS_SUCCESS;
}

static int finish(cuozblasHandle_t *h, double t0) {
    cudaError_t e = cudaStreamSynchronize(state(h)->stream);
    h->t_total = (float)(wall() - t0);
    State *st = state(h);
    if (st->plain_timers && e == cudaSuccess) {  // the plain form's phases (src/cpu/ozblas_gemm.cpp timers)
        h->t_SplitA = ev_ms(h, 0, 1) * 1e-3f;
        h->t_SplitB = ev_ms(h, 1, 2) * 1e-3f;
        h->t_comp = ev_ms(h, 2, 3) * 1e-3f;
        h->t_sum = ev_ms(h, 3, 4) * 1e-3f;
    }
    st->plain_timers = false;
    if (e != cudaSuccess) {
        fprintf(stderr, "cuozblas: CUDA error %s\n", cudaGetErrorString(e));
        return CUOZBLAS_STATUS_CUDA_ERROR;
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

// DOT into devWorkCommon[0], result to host.
static int dot_impl(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret) {
    State *st = state(h);
    bool done = false;
    int nA = 0, nB = 0;
    // NearSum: one pass over x and y (exact dot, certified rounding, proven split counts)
    if (h->splitEpsMode == 0 && h->sumMode == 1 && !st->env.dot_two_pass)
        OZB_TRY(dot_exact(h, n, x, y, ret, &done, &nA, &nB));
    if (h->splitEpsMode == 0 && !done) OZB_TRY(dot_fused(h, n, x, y, ret, &done, &nA, &nB));
    if (done) {
        h->nSplitA = (float)nA;
        h->nSplitB = (float)nB;
        h->nSplitC = 1.f;
        if (state(h)->env.dot_trace) fprintf(stderr, "cuozblas: dot fused nA=%d nB=%d\n", nA, nB);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    double *d = reinterpret_cast<double *>(h->devWorkCommon);
    OZB_CHECK(cudaMemsetAsync(d, 0, sizeof(double), st->stream));
    OZB_TRY(gemm_plain_core(h, 't', 'n', 1, 1, n, 1.0, x, n, y, n, 0.0, d, 1, 0));
    if (state(h)->env.dot_trace)
        fprintf(stderr, "cuozblas: dot general nA=%d nB=%d\n", (int)h->nSplitA, (int)h->nSplitB);
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, d, sizeof(double), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    *ret = st->h_dbl[0];
    return CUOZBLAS_STATUS_SUCCESS;
}

// The engines take a one-row op(A) of a 1 x 1 product and the one-column
// op(B) of an n = 1 product as contiguous vectors.  Stored with a leading
// dimension above 1 (A 'n' with lda > 1, B 't' with ldb > 1) their elements
// are strided: gather them into the arena and pass the contiguous form
// (A as 't' with lda = k, B as 'n' with ldb = k).  The gathered copies stay
// below the engine's own arena use for the whole call.
static int contiguous_vectors(cuozblasHandle_t *h, int esz, int m, int n, int k, char &ta, const void *&A, int &lda,
                              char &tb, const void *&B, int &ldb) {
    if (k <= 0) return CUOZBLAS_STATUS_SUCCESS;
    if (n == 1 && is_trans(tb) && ldb != 1) {
        if (ldb < 1) return CUOZBLAS_STATUS_INVALID_VALUE;
        Arena ar(h);
        char *g = ar.take<char>((uint64_t)k * esz);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(gather_strided(h, k, B, ldb, esz, g));
        B = g;
        tb = 'n';
        ldb = k;
    }
    if (m == 1 && n == 1 && !is_trans(ta) && lda != 1) {
        if (lda < 1) return CUOZBLAS_STATUS_INVALID_VALUE;
        Arena ar(h);
        char *g = ar.take<char>((uint64_t)k * esz);
        if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
        OZB_TRY(gather_strided(h, k, A, lda, esz, g));
        A = g;
        ta = 't';
        lda = k;
    }
    return CUOZBLAS_STATUS_SUCCESS;
}

template <typename T>
static int contiguous_vectors_t(cuozblasHandle_t *h, int m, int n, int k, char &ta, const T *&A, int &lda, char &tb,
                                const T *&B, int &ldb) {
    const void *a = A, *b = B;
    OZB_TRY(contiguous_vectors(h, (int)sizeof(T), m, n, k, ta, a, lda, tb, b, ldb));
    A = static_cast<const T *>(a);
    B = static_cast<const T *>(b);
    return CUOZBLAS_STATUS_SUCCESS;
}

}  // namespace ozb

using namespace ozb;

extern "C" {

const char *cuozblasVersion(void) { return "cuozblas-b200 0.1 (sm_100a; plain FP64-slice + INT8 tcgen05 forms)"; }

int cuozblasRuleTau(double v) { return tau_rule(v); }

int cuozblasRuleTauF32(float v) { return tau_rule_f32(v); }

double cuozblasRuleScale2(double v, int32_t e) { return scale2(v, e); }

int cuozblasRuleQ128(int op, const void *a, const void *b, const void *c, void *out) {
    Q128 x, y, z;
    if (!a || !out) return CUOZBLAS_STATUS_INVALID_VALUE;
    memcpy(&x, a, 16);
    switch (op) {
    case 0:
    case 1:
        memcpy(&y, b, 16);
        x = op == 0 ? q_add(x, y) : q_mul(x, y);
        memcpy(out, &x, 16);
        return CUOZBLAS_STATUS_SUCCESS;
    case 2:
        memcpy(&y, b, 16);
        memcpy(&z, c, 16);
        x = q_fma(x, y, z);
        memcpy(out, &x, 16);
        return CUOZBLAS_STATUS_SUCCESS;
    case 3: {
        const int t = tau_rule_q(x);
        memcpy(out, &t, sizeof(int));
        return CUOZBLAS_STATUS_SUCCESS;
    }
    case 4: {  // b: int rho, tau; out: remainder (16 bytes) then the slice (double)
        int rt[2];
        memcpy(rt, b, sizeof(rt));
        const double sl = q_split(x, rt[0], rt[1]);
        memcpy(out, &x, 16);
        memcpy((char *)out + 16, &sl, 8);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    case 5: {  // a: double, b: int k
        double d;
        int k;
        memcpy(&d, a, 8);
        memcpy(&k, b, sizeof(int));
        x = q_from_double_scaled(d, k);
        memcpy(out, &x, 16);
        return CUOZBLAS_STATUS_SUCCESS;
    }
    }
    return CUOZBLAS_STATUS_INVALID_VALUE;
}
int cuozblasRuleRho(int32_t dim, int32_t mode) { return rho_rule(dim, mode); }

int cuozblasRuleCrSum(int32_t n, const double *terms, double *out) {
    CrSum cs;
    for (int32_t i = 0; i < n; i++) cs.add(terms[i]);
    return cs.finish(*out) ? 1 : 0;
}

int cuozblasHandleCreate(cuozblasHandle_t *h, uint64_t workSizeBytes) {
    if (!h) return CUOZBLAS_STATUS_INVALID_VALUE;
    memset(h, 0, sizeof(*h));
    State *st = new (std::nothrow) State();
    if (!st) return CUOZBLAS_STATUS_CUDA_ERROR;
    h->workSizeBytes = workSizeBytes;
    // defaults of src/cuda/cuozblas.cpp:35-43
    h->nSplitMax = 0;
    h->memMaskSplitA = 0;
    h->splitShift = 1;
    h->splitMode = 0;
    h->fastMode = 0;
    h->reproMode = 1;
    h->sumMode = 0;
    h->useBatchedGemmFlag = 1;
    h->splitEpsMode = 0;
    h->precxFlag = 0;
    cudaError_t e = cudaMalloc((void **)&h->devWorkCommon, sizeof(double) * 512);
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->devWork, workSizeBytes > 0 ? workSizeBytes : 256);
    if (e == cudaSuccess) e = cudaMalloc((void **)&st->d_ints, sizeof(int) * 64);
    if (e == cudaSuccess) e = cudaMalloc(&st->d_persist, kPersistBytes);
    if (e == cudaSuccess) e = cudaMemset(st->d_persist, 0, kPersistBytes);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&st->h_ints, sizeof(int) * 64);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&st->h_dbl, sizeof(double) * 64);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&st->h_stage, kStageBytes);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&st->h_mail, sizeof(int) * kMailInts, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&st->d_mail, st->h_mail, 0);
    for (int i = 0; i < 5 && e == cudaSuccess; i++) e = cudaEventCreate(&st->ev[i]);
    if (e != cudaSuccess) {
        fprintf(stderr, "cuozblas: work memory allocation error (%1.3e bytes requested): %s\n",
                (double)workSizeBytes, cudaGetErrorString(e));
        if (h->devWork) cudaFree(h->devWork);
        if (h->devWorkCommon) cudaFree(h->devWorkCommon);
        if (st->d_ints) cudaFree(st->d_ints);
        if (st->d_persist) cudaFree(st->d_persist);
        if (st->h_ints) cudaFreeHost(st->h_ints);
        if (st->h_dbl) cudaFreeHost(st->h_dbl);
        if (st->h_stage) cudaFreeHost(st->h_stage);
        if (st->h_mail) cudaFreeHost(st->h_mail);
        delete st;
        memset(h, 0, sizeof(*h));
        return CUOZBLAS_STATUS_CUDA_ERROR;
    }
    st->env.read();
    h->hstBatchAddr = reinterpret_cast<char *>(st);
    h->devBatchAddr = nullptr;
    h->initialized = 1;
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasHandleReadEnv(cuozblasHandle_t *h) {
    if (!h || !h->initialized) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    state(h)->env.read();
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasHandleDestroy(cuozblasHandle_t *h) {
    if (!h || !h->initialized) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    State *st = state(h);
    cudaStreamSynchronize(st->stream);
    cudaFree(h->devWork);
    cudaFree(h->devWorkCommon);
    cudaFree(st->d_ints);
    cudaFree(st->d_persist);
    cudaFreeHost(st->h_ints);
    cudaFreeHost(st->h_dbl);
    if (st->h_stage) cudaFreeHost(st->h_stage);
    if (st->h_mail) cudaFreeHost(st->h_mail);
    for (int i = 0; i < 5; i++)
        if (st->ev[i]) cudaEventDestroy(st->ev[i]);
    delete st;
    h->devWork = h->devWorkCommon = nullptr;
    h->hstBatchAddr = nullptr;
    h->initialized = 0;
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasGetLaunchCount(cuozblasHandle_t *h, uint64_t *count) {
    if (!h || !h->initialized || !count) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    *count = state(h)->launches;
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasSetStream(cuozblasHandle_t *h, void *stream) {
    if (!h || !h->initialized) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    state(h)->stream = reinterpret_cast<cudaStream_t>(stream);
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasDgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                  const double *A, int32_t lda, const double *B, int32_t ldb, double beta, double *C, int32_t ldc) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h));
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    const double t0 = wall();
    OZB_TRY(contiguous_vectors_t(h, m, n, k, transa, A, lda, transb, B, ldb));
    OZB_TRY(gemm_plain_core(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, h->fastMode));
    return finish(h, t0);
}

int cuozblasDdot(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, const double *y, int32_t incy,
                 double *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h, true));
    if (incx != 1 || incy != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    const double t0 = wall();
    OZB_TRY(dot_impl(h, n, x, y, ret));
    h->t_SplitVec_total += h->t_SplitA + h->t_SplitB;
    return finish(h, t0);
}

int cuozblasDnrm2(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, double *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h, true));
    if (incx != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    const double t0 = wall();
    double d = 0.0;
    OZB_TRY(dot_impl(h, n, x, x, &d));
    *ret = sqrt(d);  // host sqrt, src/cuda/cuozblas_nrm2.cu:24-29
    return finish(h, t0);
}

int cuozblasDaxpy(cuozblasHandle_t *h, int32_t n, double alpha, const double *x, int32_t incx, double *y,
                  int32_t incy) {
    if (!h || !h->initialized) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    if (incx != 1 || incy != 1 || n < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    OZB_TRY(launch_axpy(h, n, alpha, x, y));
    return finish(h, wall());
}

int cuozblasDgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, double alpha, const double *A,
                  int32_t lda, const double *x, int32_t incx, double beta, double *y, int32_t incy) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h));
    if (incx != 1 || incy != 1 || m < 0 || n < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    const double t0 = wall();
    if (!is_trans(trans)) {
        if (m == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_plain_core(h, 'n', 'n', m, 1, n, alpha, A, lda, x, n, beta, y, m, h->fastMode));
    } else {
        if (n == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_plain_core(h, 't', 'n', n, 1, m, alpha, A, lda, x, m, beta, y, n, h->fastMode));
    }
    return finish(h, t0);
}

// Mixed form <double, float, float>: FSum only (the reference's mixed-type
// NearSum exits, src/cpu/ozblas_sum.cpp:273-296), no Dot2.
static int check_flags_f32(cuozblasHandle_t *h) {
    OZB_TRY(check_flags(h));
    if (h->sumMode != 0) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasDSgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                   const double *A, int32_t lda, const double *B, int32_t ldb, double beta, double *C, int32_t ldc) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    const double t0 = wall();
    OZB_TRY(contiguous_vectors_t(h, m, n, k, transa, A, lda, transb, B, ldb));
    OZB_TRY(gemm_f32_core(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, h->fastMode));
    return finish(h, t0);
}

int cuozblasDSgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, double alpha, const double *A,
                   int32_t lda, const double *x, int32_t incx, double beta, double *y, int32_t incy) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || m < 0 || n < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    if (!is_trans(trans)) {  // src/cpu/ozblas_gemv.cpp:22-26
        if (m == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_f32_core(h, 'n', 'n', m, 1, n, alpha, A, lda, x, n, beta, y, m, h->fastMode));
    } else {
        if (n == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_f32_core(h, 't', 'n', n, 1, m, alpha, A, lda, x, m, beta, y, n, h->fastMode));
    }
    return finish(h, t0);
}

// DOT of the mixed form: the GEMM with m = n = 1 (src/cpu/ozblas_dot.cpp:25),
// into devWorkCommon[0], result to the host.
static int dot_f32_impl(cuozblasHandle_t *h, int n, const double *x, const double *y, double *ret) {
    State *st = state(h);
    double *d = reinterpret_cast<double *>(h->devWorkCommon);
    OZB_CHECK(cudaMemsetAsync(d, 0, sizeof(double), st->stream));
    OZB_TRY(gemm_f32_core(h, 't', 'n', 1, 1, n, 1.0, x, n, y, n, 0.0, d, 1, 0));
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, d, sizeof(double), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    *ret = st->h_dbl[0];
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasDSdot(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, const double *y, int32_t incy,
                  double *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    OZB_TRY(dot_f32_impl(h, n, x, y, ret));
    h->t_SplitVec_total += h->t_SplitA + h->t_SplitB;
    return finish(h, t0);
}

int cuozblasDSnrm2(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, double *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    double d = 0.0;
    OZB_TRY(dot_f32_impl(h, n, x, x, &d));
    *ret = sqrt(d);  // host sqrt, src/cpu/ozblas_nrm2.cpp:24-29
    return finish(h, t0);
}

// Mixed form <float, double, double>: float data and results, FP64 slices;
// FSum only, no Dot2, as the other mixed form.
int cuozblasSDgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, float alpha,
                   const float *A, int32_t lda, const float *B, int32_t ldb, float beta, float *C, int32_t ldc) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1)) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    const double t0 = wall();
    OZB_TRY(contiguous_vectors_t(h, m, n, k, transa, A, lda, transb, B, ldb));
    OZB_TRY(gemm_sd_core(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, h->fastMode));
    return finish(h, t0);
}

int cuozblasSDgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, float alpha, const float *A, int32_t lda,
                   const float *x, int32_t incx, float beta, float *y, int32_t incy) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || m < 0 || n < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    if (!is_trans(trans)) {  // src/cpu/ozblas_gemv.cpp:22-26
        if (m == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_sd_core(h, 'n', 'n', m, 1, n, alpha, A, lda, x, n, beta, y, m, h->fastMode));
    } else {
        if (n == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_sd_core(h, 't', 'n', n, 1, m, alpha, A, lda, x, m, beta, y, n, h->fastMode));
    }
    return finish(h, t0);
}

static int dot_sd_impl(cuozblasHandle_t *h, int n, const float *x, const float *y, float *ret) {
    State *st = state(h);
    float *d = reinterpret_cast<float *>(h->devWorkCommon);
    OZB_CHECK(cudaMemsetAsync(d, 0, sizeof(float), st->stream));
    OZB_TRY(gemm_sd_core(h, 't', 'n', 1, 1, n, 1.f, x, n, y, n, 0.f, d, 1, 0));
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, d, sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    memcpy(ret, st->h_dbl, sizeof(float));
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasSDdot(cuozblasHandle_t *h, int32_t n, const float *x, int32_t incx, const float *y, int32_t incy,
                  float *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    OZB_TRY(dot_sd_impl(h, n, x, y, ret));
    h->t_SplitVec_total += h->t_SplitA + h->t_SplitB;
    return finish(h, t0);
}

int cuozblasSDnrm2(cuozblasHandle_t *h, int32_t n, const float *x, int32_t incx, float *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    float d = 0.f;
    OZB_TRY(dot_sd_impl(h, n, x, x, &d));
    *ret = (float)sqrt((double)d);  // the reference's sqrt on a float (src/cpu/ozblas_nrm2.cpp:24-29)
    return finish(h, t0);
}

// Quad I/O form <__float128, double, double>: binary128 data and results as
// 16-byte values (alpha, beta and DOT/NRM2 results in host memory); FSum only.
int cuozblasQgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, const void *alpha,
                  const void *A, int32_t lda, const void *B, int32_t ldb, const void *beta, void *C, int32_t ldc) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (m < 0 || n < 0 || k < 0 || ldc < (m > 1 ? m : 1) || !alpha || !beta) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    if (m == 0 || n == 0) return CUOZBLAS_STATUS_SUCCESS;
    const double t0 = wall();
    OZB_TRY(contiguous_vectors(h, 16, m, n, k, transa, A, lda, transb, B, ldb));
    OZB_TRY(gemm_q_core(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, h->fastMode));
    return finish(h, t0);
}

int cuozblasQgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, const void *alpha, const void *A,
                  int32_t lda, const void *x, int32_t incx, const void *beta, void *y, int32_t incy) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || m < 0 || n < 0 || !alpha || !beta) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    if (!is_trans(trans)) {  // src/cpu/ozblas_gemv.cpp:22-26
        if (m == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_q_core(h, 'n', 'n', m, 1, n, alpha, A, lda, x, n, beta, y, m, h->fastMode));
    } else {
        if (n == 0) return CUOZBLAS_STATUS_SUCCESS;
        OZB_TRY(gemm_q_core(h, 't', 'n', n, 1, m, alpha, A, lda, x, m, beta, y, n, h->fastMode));
    }
    return finish(h, t0);
}

static int dot_q_impl(cuozblasHandle_t *h, int n, const void *x, const void *y, void *ret) {
    State *st = state(h);
    void *d = h->devWorkCommon;
    static const uint64_t one[2] = {0, 0x3fff000000000000ULL}, zero[2] = {0, 0};
    OZB_CHECK(cudaMemsetAsync(d, 0, 16, st->stream));
    OZB_TRY(gemm_q_core(h, 't', 'n', 1, 1, n, one, x, n, y, n, zero, d, 1, 0));
    OZB_CHECK(cudaMemcpyAsync(st->h_dbl, d, 16, cudaMemcpyDeviceToHost, st->stream));
    OZB_CHECK(cudaStreamSynchronize(st->stream));
    memcpy(ret, st->h_dbl, 16);
    return CUOZBLAS_STATUS_SUCCESS;
}

int cuozblasQdot(cuozblasHandle_t *h, int32_t n, const void *x, int32_t incx, const void *y, int32_t incy,
                 void *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || incy != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    OZB_TRY(dot_q_impl(h, n, x, y, ret));
    h->t_SplitVec_total += h->t_SplitA + h->t_SplitB;
    return finish(h, t0);
}

int cuozblasQnrm2(cuozblasHandle_t *h, int32_t n, const void *x, int32_t incx, void *ret) {
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags_f32(h));
    if (incx != 1 || n < 0 || ret == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    if (h->reproMode == 0 && h->nSplitMax == 1) return CUOZBLAS_STATUS_NOT_SUPPORTED;
    const double t0 = wall();
    Q128 d;
    OZB_TRY(dot_q_impl(h, n, x, x, &d));
    // the reference's sqrt(ret) on a __float128 resolves to the double sqrt
    // (src/cpu/ozblas_nrm2.cpp:27): the binary128 of sqrt((double)ret)
    const double dd = q_to_double_rn(d);
    const Q128 r = q_from_double_scaled(sqrt(dd), 0);
    memcpy(ret, &r, 16);
    return finish(h, t0);
}

static int64_t splitA_ld(int nnz) { return ((int64_t)(nnz > 0 ? nnz : 1) + 31) / 32 * 32; }

int cuozblasDcsrmv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, int32_t nnz, double alpha,
                   const void *descrA, const double *val, const int32_t *colind, const int32_t *rowptr,
                   const double *x, double beta, double *y) {
    (void)descrA;
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h, true));
    if (is_trans(trans) || m < 0 || n < 0 || nnz < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    const double t0 = wall();
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    if (h->memMaskSplitA != 0) {  // `val` is the pre-split A of cuozblasDcsrmvSplitA
        OZB_TRY(csrmv_presplit(h, m, n, alpha, val, h->nSplitA_, state(h)->splitA_ld, colind, rowptr, x, beta, y));
        return finish(h, t0);
    }
    if (h->fastMode == 0 && h->splitEpsMode != 2) {
        bool done = false;
        int fa = 0, fb = 0;
        auto &memo = state(h)->csr_memo;
        const int flags = h->splitEpsMode * 64 + maxS;
        const bool same = memo.val == val && memo.colind == colind && memo.rowptr == rowptr && memo.m == m &&
                          memo.n == n && memo.nnz == nnz && memo.flags == flags;
        const int hint = same && memo.nA > 0 ? memo.nA : 4;
        OZB_TRY(csrmv_fused(h, m, n, alpha, val, colind, rowptr, x, beta, y, 1, hint, &done, &fa, &fb));
        if (done) {
            memo.val = val;
            memo.colind = colind;
            memo.rowptr = rowptr;
            memo.m = m;
            memo.n = n;
            memo.nnz = nnz;
            memo.flags = flags;
            memo.nA = fa;
            csrmv_info(h, fa, fb);
            return finish(h, t0);
        }
    }
    Arena ar(h);
    const int64_t ld = splitA_ld(nnz);
    int nA = 0;
    OZB_TRY(split_csr_count(h, m, val, rowptr, h->splitEpsMode, 1, maxS, &nA));
    double *As = ar.take<double>((uint64_t)nA * ld);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_TRY(split_csr_write(h, m, nnz, val, rowptr, h->splitEpsMode, 1, nA, As, ld));
    OZB_TRY(csrmv_presplit(h, m, n, alpha, As, nA, ld, colind, rowptr, x, beta, y));
    return finish(h, t0);
}

int cuozblasDcsrmvSplitA(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, int32_t nnz, const void *descrA,
                         const double *val, const int32_t *rowptr, double **splitA) {
    (void)descrA;
    (void)n;
    OZB_TRY(counter_init(h));
    OZB_TRY(check_flags(h, true));
    if (is_trans(trans) || m < 0 || nnz < 0 || splitA == nullptr) return CUOZBLAS_STATUS_INVALID_VALUE;
    const int maxS = h->nSplitMax > 0 ? h->nSplitMax : kMaxSplitDefault;
    const double t0 = wall();
    // tuning of splitShift (src/cuda/cuozblas_csrmv.cu:186-201), counts only
    int s = 0;
    OZB_TRY(split_csr_count(h, m, val, rowptr, h->splitEpsMode, 1, maxS, &s));
    int shift = 1;
    if (h->nSplitMax == 0) {
        int sold;
        do {
            sold = s;
            shift *= 2;
            OZB_TRY(split_csr_count(h, m, val, rowptr, h->splitEpsMode, shift, maxS, &s));
        } while (sold == s && shift < 512);
        if (sold == s) shift = 1;
        OZB_TRY(split_csr_count(h, m, val, rowptr, h->splitEpsMode, shift, maxS, &s));
    }
    // the preserved region starts at the arena base
    State *st = state(h);
    st->off = 0;
    Arena ar(h);
    const int64_t ld = splitA_ld(nnz);
    double *As = ar.take<double>((uint64_t)s * ld);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    OZB_TRY(split_csr_write(h, m, nnz, val, rowptr, h->splitEpsMode, shift, s, As, ld));
    h->memMaskSplitA = st->off;
    h->splitShift = shift;
    h->nSplitA_ = s;
    h->nSplitA = (float)s;
    state(h)->splitA_ld = ld;
    *splitA = As;
    return finish(h, t0);
}

int cuozblasDcg(cuozblasHandle_t *h, char trans, int32_t n, int32_t nnz, const void *descrA, const double *val,
                const int32_t *colind, const int32_t *rowptr, const double *b, double *x, int32_t maxiter,
                double tol) {
    if (!h || !h->initialized) return CUOZBLAS_STATUS_NOT_INITIALIZED;
    if (is_trans(trans) || n < 0 || nnz < 0 || maxiter < 0) return CUOZBLAS_STATUS_INVALID_VALUE;
    h->t_SplitMat_total = h->t_SplitVec_total = h->t_Sum_total = 0.;
    h->t_AXPY_SCAL_total = h->t_DOT_NRM2_total = h->t_SpMV_SpMM_total = 0.;
    double *hist1 = reinterpret_cast<double *>(h->cg_verbose1);
    double *hist2 = reinterpret_cast<double *>(h->cg_verbose2);
    const double t1 = wall();
    h->cg_numiter = 0;
    double *As = nullptr;
    OZB_TRY(cuozblasDcsrmvSplitA(h, trans, n, n, nnz, descrA, val, rowptr, &As));
    // The pre-split rows are re-cut on the fly with the same tuned shift:
    // identical slices (each row's chain is independent of the others).
    const int cg_shift = h->splitShift;
    // CG vectors live above the preserved split of A for the whole solve
    State *st = state(h);
    st->off = h->memMaskSplitA;
    Arena ar(h);
    const uint64_t nn = (uint64_t)(n > 0 ? n : 1);
    double *r = ar.take<double>(nn), *p = ar.take<double>(nn), *q = ar.take<double>(nn), *tv = ar.take<double>(nn);
    double *nrm_scr = ar.take<double>(kNrm2PlainScratch);
    if (!ar.ok) return CUOZBLAS_STATUS_WORKSPACE;
    const uint64_t keep = h->memMaskSplitA;
    h->memMaskSplitA = st->off;
    int status = CUOZBLAS_STATUS_SUCCESS;
    auto fail = [&](int s) {
        h->memMaskSplitA = 0;
        h->splitShift = 1;
        return s;
    };
    (void)keep;
    double nrmb = 0.0, dold = 0.0, tmp = 0.0;
    if ((status = cuozblasDnrm2(h, n, b, 1, &nrmb))) return fail(status);
    if (cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st->stream) != cudaSuccess ||
        cudaMemsetAsync(q, 0, sizeof(double) * nn, st->stream) != cudaSuccess)
        return fail(CUOZBLAS_STATUS_CUDA_ERROR);
    auto spmv = [&](double al, const double *xv, double be, double *yv) -> int {
        if (h->fastMode == 0 && h->splitEpsMode != 2) {
            OZB_TRY(counter_init(h));
            bool done = false;
            int fa = 0, fb = 0;
            OZB_TRY(csrmv_fused(h, n, n, al, val, colind, rowptr, xv, be, yv, cg_shift, h->nSplitA_, &done, &fa,
                                      &fb));
            if (state(h)->env.dot_trace && done) fprintf(stderr, "cuozblas: spmv fused nB=%d\n", fb);
            if (done) return CUOZBLAS_STATUS_SUCCESS;
        }
        const int rs = cuozblasDcsrmv(h, trans, n, n, nnz, al, descrA, As, colind, rowptr, xv, be, yv);
        if (state(h)->env.dot_trace) fprintf(stderr, "cuozblas: spmv general nB=%d\n", (int)h->nSplitB);
        return rs;
    };
    if ((status = spmv(-1., x, 1., r))) return fail(status);
    if ((status = cuozblasDdot(h, n, r, 1, r, 1, &dold))) return fail(status);
    double resi = sqrt(dold);
    auto true_res = [&]() -> double {
        // t = b - A x in plain FP64, then a plain FP64 norm on the device (diagnostic only,
        // src/cuda/cuozblas_cg.cu:3-24: a cuSPARSE csrmv and a cuBLAS nrm2 there)
        cudaMemcpyAsync(tv, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st->stream);
        launch_csrmv_plain(h, n, val, colind, rowptr, x, -1., 1., tv);
        launch_nrm2_plain(h, n, tv, nrm_scr);
        cudaMemcpyAsync(st->h_dbl, nrm_scr, sizeof(double), cudaMemcpyDeviceToHost, st->stream);
        cudaStreamSynchronize(st->stream);
        return st->h_dbl[0];
    };
    if (h->verbose > 0) {
        const double t2 = wall();
        if (hist1) hist1[0] = resi / nrmb;
        if (hist2) hist2[0] = h->trueresFlag ? true_res() / nrmb : t2 - t1;
    }
    if (cudaMemcpyAsync(p, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st->stream) != cudaSuccess)
        return fail(CUOZBLAS_STATUS_CUDA_ERROR);
    // per iteration: resi / nrmb and the second history value (elapsed time or
    // the true residual); recorded by the reference's rule at the end
    std::vector<double> res_all((size_t)maxiter + 1), when_all((size_t)maxiter + 1);
    int it = 0;
    bool stop = false;
    // one iteration in two halves: up to the x and r updates, and the rest
    auto host_head = [&]() -> int {
        h->cg_numiter = it + 1;
        OZB_TRY(spmv(1., p, 0., q));
        OZB_TRY(cuozblasDdot(h, n, p, 1, q, 1, &tmp));
        const double alpha = dold / tmp;
        OZB_TRY(launch_axpy(h, n, alpha, p, x));
        OZB_TRY(launch_axpy(h, n, -alpha, q, r));
        return CUOZBLAS_STATUS_SUCCESS;
    };
    auto host_tail = [&](bool &stp) -> int {
        it++;
        h->cg_numiter = it;
        double dnew = 0.0;
        OZB_TRY(cuozblasDdot(h, n, r, 1, r, 1, &dnew));
        resi = sqrt(dnew);
        const double beta = dnew / dold;
        dold = dnew;
        OZB_TRY(launch_scal(h, n, beta, p));
        OZB_TRY(launch_axpy(h, n, 1.0, r, p));
        res_all[(size_t)it] = resi / nrmb;
        if (h->verbose > 0) when_all[(size_t)it] = h->trueresFlag ? true_res() / nrmb : wall() - t1;
        if (resi / nrmb < tol) stp = true;
        return CUOZBLAS_STATUS_SUCCESS;
    };
    auto host_iter = [&](bool &stp) -> int {
        OZB_TRY(host_head());
        return host_tail(stp);
    };
    // The fused steps run as captured graphs when both fused paths apply
    // (plain split, full pair set) and the history needs no host work.
    const bool graphs = h->fastMode == 0 && h->splitEpsMode == 0 && n > 0 &&
                        !(h->verbose > 0 && h->trueresFlag) && !state(h)->env.cg_no_graph;
    if (graphs) {
        if ((status = cg_graph(h, n, val, colind, rowptr, x, r, p, q, nrmb, tol, maxiter, cg_shift, h->nSplitA_, dold,
                               it, stop, t1, res_all.data(), when_all.data(), host_head, host_tail, wall)))
            return fail(status);
    }
    while (!stop && it < maxiter)
        if ((status = host_iter(stop))) return fail(status);
    h->cg_numiter = it;
    if (h->verbose > 0) {  // src/cpu/ozblas_cg.cpp:104-115
        int verbose_cnt = 1;
        for (int i = 1; i <= it; i++)
            if (res_all[(size_t)i] < tol || i % h->verbose == 0) {
                if (hist1) hist1[verbose_cnt] = res_all[(size_t)i];
                if (hist2) hist2[verbose_cnt] = when_all[(size_t)i];
                verbose_cnt++;
            }
    }
    cudaError_t e = cudaStreamSynchronize(st->stream);
    h->memMaskSplitA = 0;  // src/cuda/cuozblas_cg.cu:124-127
    h->splitShift = 1;
    return e == cudaSuccess ? CUOZBLAS_STATUS_SUCCESS : CUOZBLAS_STATUS_CUDA_ERROR;
}

}  // extern "C"
