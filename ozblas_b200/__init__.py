"""ozblas_b200 — B200 (sm_100a) Ozaki-scheme BLAS behind the cuozblas.h interface.

Python view of the C ABI declared in ``include/cuozblas.h`` (ctypes over the
in-tree ``libcuozblas_b200.so``).  Names and argument meanings follow the
reference C++ API of mukunoki/ozblas (include/cuozblas.h:66-80):

    h = Handle(work_bytes)                # cuozblasCreate
    h.nSplitMax, h.sumMode, h.fastMode    # handle flags, same fields
    dgemm(h, 'n', 'n', m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    ddot(h, n, x, y) -> float             # result on the host, like the reference
    dnrm2, dgemv, daxpy, dcsrmv, dcsrmv_split_a, dcg, dgemm_i8

Device arguments are CUDA tensors (torch) or raw device addresses (int).
There is no CPU fallback: importing fails loudly when the library is missing.
Errors are raised as ``OzblasError`` carrying the cuozblasStatus_t code
(where the reference would have called exit(1)).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcuozblas_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python ozblas_b200/build.py` (nvcc, sm_100a). "
        "ozblas_b200 has no CPU fallback.")

_lib = C.CDLL(LIB_PATH)

STATUS = {
    0: "SUCCESS", 1: "NOT_INITIALIZED", 2: "INVALID_VALUE", 3: "WORKSPACE", 4: "NOT_SUPPORTED",
    5: "INT32_BOUND", 6: "DEVICE_TIMEOUT", 7: "CUDA_ERROR",
}


class OzblasError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: CUOZBLAS_STATUS_{STATUS.get(code, code)} ({code})")
        self.code = code


class HandleStruct(C.Structure):
    """cuozblasHandle_t, field for field (mukunoki/ozblas include/cuozblas.h:7-63)."""
    _fields_ = [
        ("ch", C.c_void_p), ("csh", C.c_void_p),
        ("devWork", C.c_void_p), ("devWorkCommon", C.c_void_p),
        ("workSizeBytes", C.c_uint64), ("memAddr", C.c_uint64), ("nSplitMax", C.c_int32),
        ("hstBatchAddr", C.c_void_p), ("devBatchAddr", C.c_void_p),
        ("initialized", C.c_int32),
        ("splitMode", C.c_int32), ("fastMode", C.c_int32), ("reproMode", C.c_int32), ("sumMode", C.c_int32),
        ("useBatchedGemmFlag", C.c_int32), ("splitEpsMode", C.c_int32), ("precxFlag", C.c_int32),
        ("nSplitA", C.c_float), ("nSplitB", C.c_float), ("nSplitC", C.c_float),
        ("t_SplitA", C.c_float), ("t_SplitB", C.c_float), ("t_comp", C.c_float), ("t_sum", C.c_float),
        ("t_total", C.c_float), ("n_comp", C.c_float), ("mbk", C.c_int32), ("nbk", C.c_int32),
        ("nSplitA_", C.c_int32), ("splitShift", C.c_int32), ("memMaskSplitA", C.c_uint64),
        ("trueresFlag", C.c_int32), ("verbose", C.c_int32), ("cg_numiter", C.c_int32),
        ("cg_verbose1", C.c_void_p), ("cg_verbose2", C.c_void_p),
        ("t_SplitMat_total", C.c_double), ("t_SplitVec_total", C.c_double), ("t_Sum_total", C.c_double),
        ("t_AXPY_SCAL_total", C.c_double), ("t_DOT_NRM2_total", C.c_double), ("t_SpMV_SpMM_total", C.c_double),
    ]


_HP = C.POINTER(HandleStruct)
_vp = C.c_void_p
_i32 = C.c_int32
_d = C.c_double
_ch = C.c_char


def _sig(name, args, res=C.c_int):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res
    return f


_create = _sig("cuozblasHandleCreate", [_HP, C.c_uint64])
_destroy = _sig("cuozblasHandleDestroy", [_HP])
_setstream = _sig("cuozblasSetStream", [_HP, _vp])
_launches = _sig("cuozblasGetLaunchCount", [_HP, C.POINTER(C.c_uint64)])
_readenv = _sig("cuozblasHandleReadEnv", [_HP])
_i8_wait = _sig("cuozblasSetI8WaitTest", [C.c_uint64, _i32])
_ddot = _sig("cuozblasDdot", [_HP, _i32, _vp, _i32, _vp, _i32, C.POINTER(_d)])
_dnrm2 = _sig("cuozblasDnrm2", [_HP, _i32, _vp, _i32, C.POINTER(_d)])
_daxpy = _sig("cuozblasDaxpy", [_HP, _i32, _d, _vp, _i32, _vp, _i32])
_dgemv = _sig("cuozblasDgemv", [_HP, _ch, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp, _i32])
_dgemm = _sig("cuozblasDgemm", [_HP, _ch, _ch, _i32, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp, _i32])
_dsgemm = _sig("cuozblasDSgemm", [_HP, _ch, _ch, _i32, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp, _i32])
_dsgemv = _sig("cuozblasDSgemv", [_HP, _ch, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp, _i32])
_dsdot = _sig("cuozblasDSdot", [_HP, _i32, _vp, _i32, _vp, _i32, C.POINTER(_d)])
_dsnrm2 = _sig("cuozblasDSnrm2", [_HP, _i32, _vp, _i32, C.POINTER(_d)])
_f = C.c_float
_sdgemm = _sig("cuozblasSDgemm", [_HP, _ch, _ch, _i32, _i32, _i32, _f, _vp, _i32, _vp, _i32, _f, _vp, _i32])
_sdgemv = _sig("cuozblasSDgemv", [_HP, _ch, _i32, _i32, _f, _vp, _i32, _vp, _i32, _f, _vp, _i32])
_sddot = _sig("cuozblasSDdot", [_HP, _i32, _vp, _i32, _vp, _i32, C.POINTER(_f)])
_sdnrm2 = _sig("cuozblasSDnrm2", [_HP, _i32, _vp, _i32, C.POINTER(_f)])
_qgemm = _sig("cuozblasQgemm", [_HP, _ch, _ch, _i32, _i32, _i32, _vp, _vp, _i32, _vp, _i32, _vp, _vp, _i32])
_qgemv = _sig("cuozblasQgemv", [_HP, _ch, _i32, _i32, _vp, _vp, _i32, _vp, _i32, _vp, _vp, _i32])
_qdot = _sig("cuozblasQdot", [_HP, _i32, _vp, _i32, _vp, _i32, _vp])
_qnrm2 = _sig("cuozblasQnrm2", [_HP, _i32, _vp, _i32, _vp])
_dgemm_i8 = _sig("cuozblasDgemmI8", [_HP, _ch, _ch, _i32, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp, _i32])
_dgemm_i8_static = _sig("cuozblasDgemmI8Static", [_ch, _ch, _i32, _i32, _i32, _d, _vp, _i32, _vp, _i32, _d, _vp,
                                                  _i32, _i32, _i32, _vp])
_PI32, _PD, _PVP = C.POINTER(_i32), C.POINTER(_d), C.POINTER(_vp)
_dgemm_i8_batched = _sig("cuozblasDgemmI8Batched", [_HP, _ch, _ch, _i32, _PI32, _PI32, _PI32, _PD, _PVP, _PI32, _PVP,
                                                    _PI32, _PD, _PVP, _PI32])
_dcsrmv = _sig("cuozblasDcsrmv", [_HP, _ch, _i32, _i32, _i32, _d, _vp, _vp, _vp, _vp, _vp, _d, _vp])
_dsplita = _sig("cuozblasDcsrmvSplitA", [_HP, _ch, _i32, _i32, _i32, _vp, _vp, _vp, C.POINTER(_vp)])
_dcg = _sig("cuozblasDcg", [_HP, _ch, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _d])
rule_tau = _sig("cuozblasRuleTau", [_d])
rule_rho = _sig("cuozblasRuleRho", [_i32, _i32])
rule_tau_f32 = _sig("cuozblasRuleTauF32", [C.c_float])
rule_crsum = _sig("cuozblasRuleCrSum", [_i32, _vp, _PD])
_version = _sig("cuozblasVersion", [], C.c_char_p)

#: every C-ABI symbol include/cuozblas.h declares (checked by the CPU tests)
C_ABI_SYMBOLS = [
    "cuozblasHandleCreate", "cuozblasHandleDestroy", "cuozblasSetStream", "cuozblasGetLaunchCount",
    "cuozblasHandleReadEnv", "cuozblasSetI8WaitTest", "cuozblasDdot", "cuozblasDnrm2",
    "cuozblasDaxpy", "cuozblasDgemv", "cuozblasDgemm", "cuozblasDcsrmv", "cuozblasDcsrmvSplitA", "cuozblasDcg",
    "cuozblasDgemmI8", "cuozblasDgemmI8Static", "cuozblasDgemmI8Batched", "cuozblasRuleTau", "cuozblasRuleRho",
    "cuozblasRuleCrSum", "cuozblasDSgemm", "cuozblasDSgemv", "cuozblasDSdot", "cuozblasDSnrm2",
    "cuozblasRuleTauF32", "cuozblasRuleQ128", "cuozblasRuleScale2", "cuozblasRuleI8Schedule", "cuozblasQgemm", "cuozblasQgemv", "cuozblasQdot", "cuozblasQnrm2",
    "cuozblasSDgemm", "cuozblasSDgemv", "cuozblasSDdot", "cuozblasSDnrm2",
    "cuozblasVersion",
]


def version() -> str:
    return _version().decode()


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("device tensor expected (x.is_cuda is False)")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x)}")


def _chk(fn, code):
    if code != 0:
        raise OzblasError(fn, code)


class Handle:
    """cuozblasHandle_t owned from Python; attribute access reaches the C struct."""

    def __init__(self, work_bytes: int = 4 << 30, stream=None):
        object.__setattr__(self, "_h", HandleStruct())
        _chk("cuozblasHandleCreate", _create(C.byref(self._h), int(work_bytes)))
        if stream is not None:
            self.set_stream(stream)

    def set_stream(self, stream):
        s = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
        _chk("cuozblasSetStream", _setstream(C.byref(self._h), s))

    def launch_count(self) -> int:
        """Kernels this handle has launched since it was created."""
        c = C.c_uint64()
        _chk("cuozblasGetLaunchCount", _launches(C.byref(self._h), C.byref(c)))
        return c.value

    def read_env(self):
        """Re-read the OZBLAS_* diagnostic switches (read once at creation) into the handle."""
        _chk("cuozblasHandleReadEnv", _readenv(C.byref(self._h)))

    @property
    def ref(self):
        return C.byref(self._h)

    def close(self):
        if self._h.initialized:
            _chk("cuozblasHandleDestroy", _destroy(C.byref(self._h)))

    def __getattr__(self, name):
        return getattr(object.__getattribute__(self, "_h"), name)

    def __setattr__(self, name, value):
        setattr(self._h, name, value)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    _chk("cuozblasDgemm", _dgemm(h.ref, ta.encode(), tb.encode(), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb,
                                 beta, _ptr(Cm), ldc))


def dsgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    """Mixed form <double, float, float>: FP64 data, FP32 slices and slice products (FSum)."""
    _chk("cuozblasDSgemm", _dsgemm(h.ref, ta.encode(), tb.encode(), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb,
                                   beta, _ptr(Cm), ldc))


def dsgemv(h, trans, m, n, alpha, A, lda, x, beta, y, incx=1, incy=1):
    _chk("cuozblasDSgemv", _dsgemv(h.ref, trans.encode(), m, n, alpha, _ptr(A), lda, _ptr(x), incx, beta, _ptr(y),
                                   incy))


def dsdot(h, n, x, y, incx=1, incy=1) -> float:
    r = _d()
    _chk("cuozblasDSdot", _dsdot(h.ref, n, _ptr(x), incx, _ptr(y), incy, C.byref(r)))
    return r.value


def dsnrm2(h, n, x, incx=1) -> float:
    r = _d()
    _chk("cuozblasDSnrm2", _dsnrm2(h.ref, n, _ptr(x), incx, C.byref(r)))
    return r.value


def sdgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    """Mixed form <float, double, double>: float data and C, FP64 slices and slice products (FSum)."""
    _chk("cuozblasSDgemm", _sdgemm(h.ref, ta.encode(), tb.encode(), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb,
                                   beta, _ptr(Cm), ldc))


def sdgemv(h, trans, m, n, alpha, A, lda, x, beta, y, incx=1, incy=1):
    _chk("cuozblasSDgemv", _sdgemv(h.ref, trans.encode(), m, n, alpha, _ptr(A), lda, _ptr(x), incx, beta, _ptr(y),
                                   incy))


def sddot(h, n, x, y, incx=1, incy=1) -> float:
    r = _f()
    _chk("cuozblasSDdot", _sddot(h.ref, n, _ptr(x), incx, _ptr(y), incy, C.byref(r)))
    return r.value


def sdnrm2(h, n, x, incx=1) -> float:
    r = _f()
    _chk("cuozblasSDnrm2", _sdnrm2(h.ref, n, _ptr(x), incx, C.byref(r)))
    return r.value


def _q16(v):
    """A host binary128 scalar (16 bytes: uint64 (lo, hi)) as a ctypes buffer."""
    import numpy as _np
    a = _np.ascontiguousarray(v, dtype=_np.uint64).reshape(2)
    return (C.c_uint64 * 2)(int(a[0]), int(a[1]))


def qgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    """Quad I/O form <__float128, double, double>: A, B, C device buffers of 16-byte binary128 values;
    alpha, beta host binary128 scalars given as two uint64 (lo, hi)."""
    _chk("cuozblasQgemm", _qgemm(h.ref, ta.encode(), tb.encode(), m, n, k, C.cast(_q16(alpha), _vp), _ptr(A), lda,
                                 _ptr(B), ldb, C.cast(_q16(beta), _vp), _ptr(Cm), ldc))


def qgemv(h, trans, m, n, alpha, A, lda, x, beta, y, incx=1, incy=1):
    _chk("cuozblasQgemv", _qgemv(h.ref, trans.encode(), m, n, C.cast(_q16(alpha), _vp), _ptr(A), lda, _ptr(x), incx,
                                 C.cast(_q16(beta), _vp), _ptr(y), incy))


def qdot(h, n, x, y, incx=1, incy=1):
    """Binary128 DOT; returns the result's two uint64 (lo, hi)."""
    r = (C.c_uint64 * 2)()
    _chk("cuozblasQdot", _qdot(h.ref, n, _ptr(x), incx, _ptr(y), incy, C.cast(r, _vp)))
    return (r[0], r[1])


def qnrm2(h, n, x, incx=1):
    r = (C.c_uint64 * 2)()
    _chk("cuozblasQnrm2", _qnrm2(h.ref, n, _ptr(x), incx, C.cast(r, _vp)))
    return (r[0], r[1])


def set_i8_wait_test(ns: int, hold_copies: bool = False):
    """Testing hook: the bounded-wait limit of the INT8 product kernel on the current device (0: default 2 s) and
    whether its producer holds back every copy (so a wait runs out); (0, False) restores."""
    _chk("cuozblasSetI8WaitTest", _i8_wait(int(ns), 1 if hold_copies else 0))


def dgemm_i8(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc):
    _chk("cuozblasDgemmI8", _dgemm_i8(h.ref, ta.encode(), tb.encode(), m, n, k, alpha, _ptr(A), lda, _ptr(B),
                                      ldb, beta, _ptr(Cm), ldc))


def dgemm_i8_batched(h, ta, tb, ms, ns, ks, alphas, As, ldas, Bs, ldbs, betas, Cs, ldcs):
    """Many INT8 DGEMMs of different shapes in one grouped launch; per-problem lists (device buffers for A, B, C)."""
    cnt = len(ms)
    arr = lambda t, v: (t * cnt)(*v)
    _chk("cuozblasDgemmI8Batched", _dgemm_i8_batched(
        h.ref, ta.encode(), tb.encode(), cnt, arr(_i32, ms), arr(_i32, ns), arr(_i32, ks), arr(_d, alphas),
        arr(_vp, [_ptr(a) for a in As]), arr(_i32, ldas), arr(_vp, [_ptr(b) for b in Bs]), arr(_i32, ldbs),
        arr(_d, betas), arr(_vp, [_ptr(c) for c in Cs]), arr(_i32, ldcs)))


def dgemm_i8_static(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, nSplitMax=0, fastMode=0, stream=None):
    """INT8 DGEMM without a handle and without any allocation (library-internal 64 MiB scratch)."""
    s = None if stream is None else (stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream))
    _chk("cuozblasDgemmI8Static", _dgemm_i8_static(ta.encode(), tb.encode(), m, n, k, alpha, _ptr(A), lda, _ptr(B),
                                                   ldb, beta, _ptr(Cm), ldc, nSplitMax, fastMode, s))


def ddot(h, n, x, y, incx=1, incy=1) -> float:
    r = _d()
    _chk("cuozblasDdot", _ddot(h.ref, n, _ptr(x), incx, _ptr(y), incy, C.byref(r)))
    return r.value


def dnrm2(h, n, x, incx=1) -> float:
    r = _d()
    _chk("cuozblasDnrm2", _dnrm2(h.ref, n, _ptr(x), incx, C.byref(r)))
    return r.value


def daxpy(h, n, alpha, x, y, incx=1, incy=1):
    _chk("cuozblasDaxpy", _daxpy(h.ref, n, alpha, _ptr(x), incx, _ptr(y), incy))


def dgemv(h, trans, m, n, alpha, A, lda, x, beta, y, incx=1, incy=1):
    _chk("cuozblasDgemv", _dgemv(h.ref, trans.encode(), m, n, alpha, _ptr(A), lda, _ptr(x), incx, beta, _ptr(y),
                                 incy))


def dcsrmv(h, trans, m, n, nnz, alpha, val, colind, rowptr, x, beta, y, descr=None):
    _chk("cuozblasDcsrmv", _dcsrmv(h.ref, trans.encode(), m, n, nnz, alpha, descr, _ptr(val), _ptr(colind),
                                   _ptr(rowptr), _ptr(x), beta, _ptr(y)))


def dcsrmv_split_a(h, trans, m, n, nnz, val, rowptr, descr=None) -> int:
    out = _vp()
    _chk("cuozblasDcsrmvSplitA", _dsplita(h.ref, trans.encode(), m, n, nnz, descr, _ptr(val), _ptr(rowptr),
                                          C.byref(out)))
    return out.value


def dcg(h, trans, n, nnz, val, colind, rowptr, b, x, maxiter, tol, hist1=None, hist2=None, descr=None):
    """CG; hist1/hist2 are host numpy float64 arrays of maxiter+1 entries (history per `h.verbose`)."""
    h.cg_verbose1 = hist1.ctypes.data if hist1 is not None else None
    h.cg_verbose2 = hist2.ctypes.data if hist2 is not None else None
    _chk("cuozblasDcg", _dcg(h.ref, trans.encode(), n, nnz, descr, _ptr(val), _ptr(colind), _ptr(rowptr), _ptr(b),
                             _ptr(x), maxiter, tol))
    return h.cg_numiter
