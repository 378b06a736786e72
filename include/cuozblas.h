/*
 * cuozblas.h — drop-in interface of the B200 (sm_100a) Ozaki-scheme library.
 *
 * Two views of one library (libcuozblas_b200.so):
 *
 *  1. The reference's C++ API, unchanged: cuozblasHandle_t with the field
 *     order and types of mukunoki/ozblas include/cuozblas.h:7-63, and the
 *     templates of include/cuozblas.h:66-80.  The library exports the same
 *     explicit instantiations for FP64 input/output, so code compiled against
 *     the reference header links against this library unchanged.
 *
 *  2. A C ABI (extern "C", plain pointers and sizes) for FFI callers
 *     (ctypes, cgo, JNI, N-API).  Each entry returns a cuozblasStatus_t
 *     instead of calling exit(1) as the reference does.
 *
 * Conventions (as in the reference): column-major matrices, 0-based CSR with
 * 32-bit indices, alpha/beta and scalar results on the host, vectors and
 * matrices in device memory.  Calls are stream-ordered on the handle's
 * stream (cuozblasSetStream; default: the legacy default stream) and return
 * after the result is complete on that stream.  One call at a time per handle.
 */
#ifndef CUOZBLAS_B200_H
#define CUOZBLAS_B200_H

#include <stdint.h>

/* cuBLAS / cuSPARSE handle types as the CUDA headers define them; the
 * library never creates or uses either (no cuBLAS on the hot path). */
typedef struct cublasContext *cublasHandle_t;
typedef struct cusparseContext *cusparseHandle_t;
typedef struct cusparseMatDescr *cusparseMatDescr_t;

/* Layout identical to mukunoki/ozblas include/cuozblas.h:7-63. */
typedef struct {
    cublasHandle_t ch;     /* always NULL here */
    cusparseHandle_t csh;  /* always NULL here */

    /* core */
    char *devWork;          /* device arena, cudaMalloc'd once at create */
    char *devWorkCommon;    /* 512 doubles of device scratch */
    uint64_t workSizeBytes;
    uint64_t memAddr;       /* bytes of the arena in use by the last call */
    int32_t nSplitMax;      /* 0: split until exact (at most 30 slices) */
    char *hstBatchAddr;     /* holds the library's private per-handle state */
    char *devBatchAddr;     /* unused (NULL) */

    int32_t initialized;

    /* option flags */
    int32_t splitMode;
    int32_t fastMode;       /* levels dropped from the slice-pair set */
    int32_t reproMode;      /* must be 1 (reproducible); 0 with nSplitMax 1 = plain FP64 */
    int32_t sumMode;        /* 0: ordered FP64 sum; 1: NearSum (correctly rounded) */
    int32_t useBatchedGemmFlag;
    int32_t splitEpsMode;   /* 0, 9, or 2 (Dot2: DOT, NRM2, CSRMV and CG with fastMode 0) */
    int32_t precxFlag;

    /* exec info */
    float nSplitA;
    float nSplitB;
    float nSplitC;

    float t_SplitA;
    float t_SplitB;
    float t_comp;
    float t_sum;
    float t_total;
    float n_comp;
    int32_t mbk;
    int32_t nbk;

    /* for SpMV in iterative solvers */
    int32_t nSplitA_;
    int32_t splitShift;
    uint64_t memMaskSplitA;

    /* for CG */
    int32_t trueresFlag;
    int32_t verbose;
    int32_t cg_numiter;
    void *cg_verbose1;      /* host array of relative residuals (verbose > 0) */
    void *cg_verbose2;      /* host array of elapsed seconds (trueresFlag == 0) */
    double t_SplitMat_total;
    double t_SplitVec_total;
    double t_Sum_total;
    double t_AXPY_SCAL_total;
    double t_DOT_NRM2_total;
    double t_SpMV_SpMM_total;

} cuozblasHandle_t;

typedef enum {
    CUOZBLAS_STATUS_SUCCESS = 0,
    CUOZBLAS_STATUS_NOT_INITIALIZED = 1,
    CUOZBLAS_STATUS_INVALID_VALUE = 2,  /* inc != 1, transposed CSRMV, bad sizes or flags */
    CUOZBLAS_STATUS_WORKSPACE = 3,      /* the arena given at create is too small */
    CUOZBLAS_STATUS_NOT_SUPPORTED = 4,  /* e.g. Dot2 for GEMM/GEMV, NearSum in the mixed and quad forms */
    CUOZBLAS_STATUS_INT32_BOUND = 5,    /* INT8 form: k beyond the exact INT32 bound */
    CUOZBLAS_STATUS_DEVICE_TIMEOUT = 6, /* a bounded device-side wait gave up */
    CUOZBLAS_STATUS_CUDA_ERROR = 7
} cuozblasStatus_t;

#ifdef __cplusplus
/* ---- reference C++ API (include/cuozblas.h:66-80) ---- */
extern void cuozblasCreate(cuozblasHandle_t *, uint64_t);
extern void cuozblasDestroy(cuozblasHandle_t *);

template <typename TYPE1, typename TYPE2, typename TYPE3>
int32_t cuozblasRnrm2(cuozblasHandle_t *oh, const int32_t n, const TYPE1 *devX, const int32_t incx, TYPE1 *ret);
template <typename TYPE>
int32_t cuozblasRaxpy(cuozblasHandle_t *oh, const int32_t n, const TYPE alpha, const TYPE *devX, const int32_t incx,
                      TYPE *devY, const int32_t incy);
template <typename TYPE1, typename TYPE2, typename TYPE3>
int32_t cuozblasRdot(cuozblasHandle_t *oh, const int32_t n, const TYPE1 *devA, const int32_t incx, const TYPE1 *devB,
                     const int32_t incy, TYPE1 *ret);
template <typename TYPE1, typename TYPE2, typename TYPE3>
int32_t cuozblasRgemv(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n, const TYPE1 alpha,
                      const TYPE1 *devA, const int32_t lda, const TYPE1 *devB, const int32_t incx, const TYPE1 beta,
                      TYPE1 *devC, const int32_t incy);
template <typename TYPE1, typename TYPE2, typename TYPE3>
int32_t cuozblasRgemm(cuozblasHandle_t *oh, const char tranA, const char tranB, const int32_t m, const int32_t n,
                      const int32_t k, const TYPE1 alpha, const TYPE1 *devA, const int32_t lda, const TYPE1 *devB,
                      const int32_t ldb, const TYPE1 beta, TYPE1 *devC, const int32_t ldc);
template <typename TYPE1, typename TYPE2>
int32_t cuozblasRcsrmv(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n, const int32_t nnz,
                       const TYPE1 alpha, const cusparseMatDescr_t descrA, const TYPE1 *devA,
                       const int32_t *devAcolind, const int32_t *devArowptr, const TYPE1 *devB, const TYPE1 beta,
                       TYPE1 *devC);
template <typename TYPE1, typename TYPE2>
TYPE2 *cuozblasRcsrmvSplitA(cuozblasHandle_t *oh, const char tranA, const int32_t m, const int32_t n,
                            const int32_t nnz, const cusparseMatDescr_t descrA, const TYPE1 *devA,
                            const int32_t *devArowptr);
template <typename TYPE1, typename TYPE2>
int32_t cuozblasRcg(cuozblasHandle_t *oh, const char tranA, const int32_t dimN, const int32_t dimNNZ,
                    const cusparseMatDescr_t descrA, const TYPE1 *matA, const int32_t *matAcolind,
                    const int32_t *matArowptr, const TYPE1 *vecB, TYPE1 *vecX, int32_t maxiter, TYPE1 tol);
/* Exported instantiations: <double,double,double>, <double,float,float> and
 * <float,double,double> for nrm2/dot/gemv/gemm,
 * <double> for axpy, <double,double> for csrmv/csrmvSplitA/cg, and the INT8
 * precision form cuozblasRgemm<double,int8_t,int32_t> (the instantiation
 * the reference leaves commented out at src/cuda/cuozblas_gemm.cu:292). */
extern "C" {
#endif

/* ---- C ABI ---- */

/* cuozblasCreate (include/cuozblas.h:66; src/cuda/cuozblas.cpp:23-64):
 * sets the reference defaults and cudaMallocs the arena once. */
int cuozblasHandleCreate(cuozblasHandle_t *h, uint64_t workSizeBytes);
/* cuozblasDestroy (include/cuozblas.h:67; src/cuda/cuozblas.cpp:66-75) */
int cuozblasHandleDestroy(cuozblasHandle_t *h);
/* Extension: run the handle's work on `stream` (a cudaStream_t). */
int cuozblasSetStream(cuozblasHandle_t *h, void *stream);
/* Extension: number of kernels the handle has launched since create. */
int cuozblasGetLaunchCount(cuozblasHandle_t *h, uint64_t *count);
/* Re-read the OZBLAS_* diagnostic switches from the environment into the
 * handle (they are read once when the handle is created; each selects an
 * equal-bits alternative path or a stderr trace).  No reference counterpart. */
int cuozblasHandleReadEnv(cuozblasHandle_t *h);


/* cuozblasRdot<double,double,double> (include/cuozblas.h:75; src/cuda/cuozblas_dot.cu:3-40).
 * *ret is a host pointer, written before return. */
int cuozblasDdot(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, const double *y, int32_t incy,
                 double *ret);
/* cuozblasRnrm2<double,double,double> (include/cuozblas.h:73; src/cuda/cuozblas_nrm2.cu:3-33) */
int cuozblasDnrm2(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, double *ret);
/* cuozblasRaxpy<double> (include/cuozblas.h:74; src/cuda/cuozblas_axpy.cu:18-40): y = fma(alpha, x, y) */
int cuozblasDaxpy(cuozblasHandle_t *h, int32_t n, double alpha, const double *x, int32_t incx, double *y,
                  int32_t incy);
/* cuozblasRgemv<double,double,double> (include/cuozblas.h:76; src/cuda/cuozblas_gemv.cu:3-30) */
int cuozblasDgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, double alpha, const double *A,
                  int32_t lda, const double *x, int32_t incx, double beta, double *y, int32_t incy);
/* cuozblasRgemm<double,double,double> (include/cuozblas.h:77; src/cuda/cuozblas_gemm.cu:7-284):
 * plain form, FP64 slices, bit-exact to the reference CPU path. */
int cuozblasDgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                  const double *A, int32_t lda, const double *B, int32_t ldb, double beta, double *C, int32_t ldc);
/* cuozblasRcsrmv<double,double> (include/cuozblas.h:78; src/cuda/cuozblas_csrmv.cu:3-133).
 * descrA is accepted and ignored (general matrix, 0-based). */
int cuozblasDcsrmv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, int32_t nnz, double alpha,
                   const void *descrA, const double *val, const int32_t *colind, const int32_t *rowptr,
                   const double *x, double beta, double *y);
/* cuozblasRcsrmvSplitA<double,double> (include/cuozblas.h:79; src/cuda/cuozblas_csrmv.cu:141-217):
 * splits A once (with splitShift tuning) into the arena; *splitA receives
 * the pointer to pass as `val` to later cuozblasDcsrmv calls. */
int cuozblasDcsrmvSplitA(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, int32_t nnz, const void *descrA,
                         const double *val, const int32_t *rowptr, double **splitA);
/* cuozblasRcg<double,double> (include/cuozblas.h:80; src/cuda/cuozblas_cg.cu:25-131) */
int cuozblasDcg(cuozblasHandle_t *h, char trans, int32_t n, int32_t nnz, const void *descrA, const double *val,
                const int32_t *colind, const int32_t *rowptr, const double *b, double *x, int32_t maxiter,
                double tol);

/* Mixed form <double,float,float> (include/cuozblas.h:75-77 instantiated at
 * src/cuda/cuozblas_gemm.cu:286, src/cuda/cuozblas_dot.cu, cuozblas_nrm2.cu,
 * cuozblas_gemv.cu): FP64 data with FP32 slices and FP32 slice products,
 * bit-exact to the reference CPU path (src/cpu/ozblas_gemm.cpp with TYPE2 =
 * TYPE3 = float).  sumMode 0 (FSum) only: the reference has no NearSum for
 * mixed types (CUOZBLAS_STATUS_NOT_SUPPORTED here, exit(1) there); no Dot2. */
int cuozblasDSgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                   const double *A, int32_t lda, const double *B, int32_t ldb, double beta, double *C, int32_t ldc);
int cuozblasDSgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, double alpha, const double *A,
                   int32_t lda, const double *x, int32_t incx, double beta, double *y, int32_t incy);
int cuozblasDSdot(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, const double *y, int32_t incy,
                  double *ret);
int cuozblasDSnrm2(cuozblasHandle_t *h, int32_t n, const double *x, int32_t incx, double *ret);

/* Mixed form <float,double,double> (include/cuozblas.h:75-77 instantiated at
 * src/cuda/cuozblas_gemm.cu:290 and the DOT/NRM2/GEMV files): float data and
 * results with FP64 slices and exact FP64 slice products, bit-exact to the
 * reference CPU path (src/cpu/ozblas_gemm.cpp with TYPE1 = float).  The split
 * runs in float arithmetic; each pair product is rounded to float, scaled in
 * float and summed in float.  sumMode 0 only, no Dot2.  *ret of SDdot/SDnrm2
 * is a host pointer. */
int cuozblasSDgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, float alpha,
                   const float *A, int32_t lda, const float *B, int32_t ldb, float beta, float *C, int32_t ldc);
int cuozblasSDgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, float alpha, const float *A, int32_t lda,
                   const float *x, int32_t incx, float beta, float *y, int32_t incy);
int cuozblasSDdot(cuozblasHandle_t *h, int32_t n, const float *x, int32_t incx, const float *y, int32_t incy,
                  float *ret);
int cuozblasSDnrm2(cuozblasHandle_t *h, int32_t n, const float *x, int32_t incx, float *ret);

/* Quad I/O form <__float128,double,double> (the reference's CPU instantiation,
 * src/cpu/ozblas_gemm.cpp:316, with src/cpu/ozblas_dot.cpp, ozblas_nrm2.cpp,
 * ozblas_gemv.cpp): binary128 data and results, FP64 slices and exact FP64
 * slice products, the ordered sum and fmaq(alpha, t, beta C) in binary128.
 * Arrays hold 16-byte IEEE binary128 values (the x86-64 __float128 layout);
 * alpha, beta and *ret are host pointers to one such value.  Bit-identical to
 * the reference CPU library; sumMode 0 only.  (The reference needs MPLAPACK
 * to split a one-column panel, i.e. for DOT, NRM2, GEMV and m or n = 1.) */
int cuozblasQgemm(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, const void *alpha,
                  const void *A, int32_t lda, const void *B, int32_t ldb, const void *beta, void *C, int32_t ldc);
int cuozblasQgemv(cuozblasHandle_t *h, char trans, int32_t m, int32_t n, const void *alpha, const void *A,
                  int32_t lda, const void *x, int32_t incx, const void *beta, void *y, int32_t incy);
int cuozblasQdot(cuozblasHandle_t *h, int32_t n, const void *x, int32_t incx, const void *y, int32_t incy,
                 void *ret);
int cuozblasQnrm2(cuozblasHandle_t *h, int32_t n, const void *x, int32_t incx, void *ret);

/* INT8 precision form (no reference implementation; the reference stubs it
 * at src/cuda/cuozblas_gemm.cu:292 and src/cuda/cuozblas_blas_wrapper.cu:147-208):
 * INT8 slices on tcgen05 tensor cores with INT32 accumulation.
 * nSplitMax = slices per operand (0: chosen per operand from its exponent
 * range), fastMode != 0: triangular pair set. */
int cuozblasDgemmI8(cuozblasHandle_t *h, char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha,
                    const double *A, int32_t lda, const double *B, int32_t ldb, double beta, double *C,
                    int32_t ldc);

/* Many INT8 precision-form DGEMMs of different shapes in one persistent
 * grouped launch.  No counterpart in the reference (its batched path,
 * src/cuda/cuozblas_gemm.cu:165-178, batches the slice pairs of one
 * product).  Arrays of `count` entries in host memory; A[b], B[b], C[b] are
 * device pointers (column-major, as cuozblasDgemmI8).  Every problem's
 * result is bit-identical to cuozblasDgemmI8 on it with the same handle
 * flags (nSplitMax, fastMode).  nSplitA/B report the largest digit counts,
 * nSplitC the largest pair count. */
int cuozblasDgemmI8Batched(cuozblasHandle_t *h, char transa, char transb, int32_t count, const int32_t *m,
                           const int32_t *n, const int32_t *k, const double *alpha, const double *const *A,
                           const int32_t *lda, const double *const *B, const int32_t *ldb, const double *beta,
                           double *const *C, const int32_t *ldc);

/* Allocation-free INT8 precision-form DGEMM.  No counterpart in the
 * reference.  For callers that cannot allocate device memory (real-time or
 * embedded hosts whose device memory is budgeted once at start-up, hosts
 * whose own allocator already owns the whole device): same arithmetic and
 * results as cuozblasDgemmI8, with the flags passed directly and no handle;
 * the scratch is a 64 MiB file-scope device array inside the library
 * (resident on every GPU that loads it), so the call makes no cudaMalloc,
 * cudaFree or other allocation.  Problems whose digits and work do not fit
 * in those 64 MiB (about m = n = k = 1300 at 13 digits) return
 * CUOZBLAS_STATUS_WORKSPACE with a message.  The first call on a device
 * looks up the array's device address and should precede any stream
 * capture.  All calls share the array: calls that overlap on the GPU race.
 * `stream` is a cudaStream_t (NULL: legacy default stream). */
int cuozblasDgemmI8Static(char transa, char transb, int32_t m, int32_t n, int32_t k, double alpha, const double *A,
                          int32_t lda, const double *B, int32_t ldb, double beta, double *C, int32_t ldc,
                          int32_t nSplitMax, int32_t fastMode, void *stream);

/* Testing hook, no reference counterpart: on the current device, the limit
 * (ns) of every bounded mbarrier wait of the INT8 product kernel (0: the
 * default 2 s) and, with hold_copies != 0, a producer that issues no copies,
 * so that the tensor-core issuer's wait runs out and cuozblasDgemmI8 returns
 * CUOZBLAS_STATUS_DEVICE_TIMEOUT; the kernel releases its tensor memory
 * first and the context stays usable.  Call (0, 0) to restore. */
int cuozblasSetI8WaitTest(uint64_t ns, int32_t hold_copies);

/* Rule checks exported for the host-side tests (same code the kernels use). */
int cuozblasRuleTau(double v);
/* tau of float data for the <float,double,double> form: (short)ceil((float)log2((double)v)) */
int cuozblasRuleTauF32(float v);
/* v * 2^e rounded once to nearest (the scaling of the mixed forms' ordered sums) */
double cuozblasRuleScale2(double v, int32_t e);
/* The software binary128 of the quad form, on the host: op 0 *out = *a + *b,
 * 1 *a * *b, 2 fma(*a, *b, *c), 3 (int) tau of *a, 4 the split of *a with
 * (int) rho, tau at b (out: remainder, then the slice as a double),
 * 5 (double)*a * 2^(int)*b.  Values are 16-byte IEEE binary128. */
int cuozblasRuleQ128(int op, const void *a, const void *b, const void *c, void *out);
/* The INT8 form's level-blocked schedule, on the host (the steps the product
 * kernels run): digit counts nA, nB, nkb 128-wide K steps, the triangular or
 * full pair set, `width` levels per block within the runs of levels (1-4) or,
 * negative, equal cuts of at most -width levels across them.  Writes 12 int32
 * per step (L0, L1, kb0, kb1, run_hi, flags, fexp, cexp, mid, fexp_mid,
 * cexp_mid, first_mid) into out and returns the number of steps; -1 when the
 * schedule does not apply (for a cut across runs: a crossing block would need
 * several K chunks), -2 when max_steps is too small. */
int cuozblasRuleI8Schedule(int32_t nA, int32_t nB, int32_t nkb, int32_t triangular, int32_t width, int32_t *out,
                           int32_t max_steps);
int cuozblasRuleRho(int32_t dim, int32_t splitEpsMode);
/* Certified fast path of the correctly rounded sum (the NearSum result when it
 * returns 1; 0: not proven, the library then runs NearSum itself). */
int cuozblasRuleCrSum(int32_t n, const double *terms, double *out);
/* Library build identification ("sm_100a ..."). */
const char *cuozblasVersion(void);

#ifdef __cplusplus
}
#endif

#endif /* CUOZBLAS_B200_H */
