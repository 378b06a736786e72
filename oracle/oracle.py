"""ctypes bindings for the CPU oracles (test infrastructure only).

* ``Restatement`` wraps ``_build/liboracle.so`` (ozoracle.c): the C
  restatement of the reference CPU path, the exact dot-product accumulator
  and the seeded input generators.
* ``Reference`` wraps ``_ref/libozblas_ref.so``: the reference OzBLAS CPU
  library (mukunoki/ozblas src/cpu) built unmodified from its sources, with
  the thin extern "C" layer in refshim/ref_capi.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The library ``ozblas_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libozblas_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(_ip)


def build_oracle(force=False):
    """Compile ozoracle.c with gcc (works on any box with this image)."""
    if force or not os.path.exists(LIB_ORACLE):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
    return LIB_ORACLE


class Flags(C.Structure):
    _fields_ = [
        ("nSplitMax", C.c_int),
        ("splitMode", C.c_int),
        ("fastMode", C.c_int),
        ("reproMode", C.c_int),
        ("sumMode", C.c_int),
        ("splitEpsMode", C.c_int),
    ]


class Info(C.Structure):
    _fields_ = [
        ("nSplitA", C.c_float),
        ("nSplitB", C.c_float),
        ("nSplitC", C.c_float),
        ("splitShift", C.c_int),
        ("nSplitA_", C.c_int),
        ("cg_numiter", C.c_int),
    ]


def make_flags(nSplitMax=0, fastMode=0, sumMode=0, splitEpsMode=0, splitMode=0, reproMode=1):
    return Flags(nSplitMax, splitMode, fastMode, reproMode, sumMode, splitEpsMode)


class Restatement:
    """The C restatement of the reference CPU path plus generators and exact sums."""

    def __init__(self):
        build_oracle()
        L = C.CDLL(LIB_ORACLE)
        self.L = L
        F = C.POINTER(Flags)
        I = C.POINTER(Info)
        L.oz_rho.restype = C.c_int
        L.oz_rho.argtypes = [C.c_int, C.c_int]
        L.oz_tau_libm.restype = C.c_int
        L.oz_tau_libm.argtypes = [C.c_double]
        L.oz_split_cols.restype = C.c_int
        L.oz_split_cols.argtypes = [F, C.c_int, C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int]
        L.oz_rho_f32.restype = C.c_int
        L.oz_rho_f32.argtypes = [C.c_int, C.c_int]
        L.oz_split_cols_f32.restype = C.c_int
        L.oz_split_cols_f32.argtypes = [F, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int,
                                        C.POINTER(C.c_short)]
        L.oz_dgemm_f32.restype = C.c_int
        L.oz_dgemm_f32.argtypes = [F, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int,
                                   _dp, C.c_int, C.c_double, _dp, C.c_int, I]
        _fp = C.POINTER(C.c_float)
        L.oz_rho_sd.restype = C.c_int
        L.oz_rho_sd.argtypes = [C.c_int, C.c_int]
        L.oz_tau_sd_libm.restype = C.c_short
        L.oz_tau_sd_libm.argtypes = [C.c_float]
        L.oz_tau_sd_sweep.restype = C.c_long
        L.oz_tau_sd_sweep.argtypes = [C.c_void_p, C.c_uint, C.POINTER(C.c_uint)]
        L.oz_split_cols_sd.restype = C.c_int
        L.oz_split_cols_sd.argtypes = [F, C.c_int, C.c_int, _fp, C.c_int, C.c_int, _dp, C.c_int,
                                       C.POINTER(C.c_short)]
        L.oz_sgemm_d.restype = C.c_int
        L.oz_sgemm_d.argtypes = [F, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_float, _fp, C.c_int, _fp,
                                 C.c_int, C.c_float, _fp, C.c_int, I]
        _vp = C.c_void_p
        L.oz_rho_q.restype = C.c_int
        L.oz_rho_q.argtypes = [C.c_int, C.c_int]
        L.oz_tau_q_libm.restype = C.c_int
        L.oz_tau_q_libm.argtypes = [_vp]
        L.oz_split_cols_q.restype = C.c_int
        L.oz_split_cols_q.argtypes = [F, C.c_int, C.c_int, _vp, C.c_int, _dp, C.c_int, C.POINTER(C.c_short)]
        L.oz_qgemm_d.restype = C.c_int
        L.oz_qgemm_d.argtypes = [F, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int,
                                 _vp, _vp, C.c_int, I]
        L.oz_gen_phi_q.argtypes = [C.c_int, C.c_int, C.c_int, _vp, C.c_double, C.c_int]
        for nm in ("oz_q_add", "oz_q_mul"):
            getattr(L, nm).argtypes = [_vp, _vp, _vp]
        L.oz_q_fma.argtypes = [_vp, _vp, _vp, _vp]
        L.oz_q_scale.argtypes = [_vp, C.c_long, C.c_int]
        L.oz_q_from_double.argtypes = [C.c_double, _vp]
        L.oz_q128_check.restype = C.c_long
        L.oz_q128_check.argtypes = [_vp, C.c_int, C.c_long, C.c_uint, _vp]
        L.oz_q_to_double.restype = C.c_double
        L.oz_q_to_double.argtypes = [_vp]
        L.oz_split_rows_csr.restype = C.c_int
        L.oz_split_rows_csr.argtypes = [F, C.c_int, _dp, _ip, C.c_int, _dp, C.c_int]
        L.oz_nearsum.restype = C.c_double
        L.oz_nearsum.argtypes = [C.c_int, _dp]
        L.oz_dgemm.restype = C.c_int
        L.oz_dgemm.argtypes = [F, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp,
                               C.c_int, C.c_double, _dp, C.c_int, I]
        L.oz_ddot.restype = C.c_double
        L.oz_ddot.argtypes = [F, C.c_int, _dp, _dp, I]
        L.oz_dnrm2.restype = C.c_double
        L.oz_dnrm2.argtypes = [F, C.c_int, _dp, I]
        L.oz_dgemv.restype = C.c_int
        L.oz_dgemv.argtypes = [F, C.c_char, C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp, C.c_double, _dp, I]
        L.oz_dcsrmv.restype = C.c_int
        L.oz_dcsrmv.argtypes = [F, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _ip, _ip, _dp, C.c_double, _dp, I]
        L.oz_dcsrmv_split_a.restype = C.c_int
        L.oz_dcsrmv_split_a.argtypes = [F, C.c_int, C.c_int, _dp, _ip, _dp, C.c_int, _ip, _ip]
        L.oz_dcg.restype = C.c_int
        L.oz_dcg.argtypes = [F, C.c_int, C.c_int, _dp, _ip, _ip, _dp, _dp, C.c_int, C.c_double, _dp, I]
        L.oz_exact_dot_rn.restype = C.c_double
        L.oz_exact_dot_rn.argtypes = [C.c_int, _dp, C.c_int, _dp, C.c_int]
        L.oz_exact_dot_err.restype = None
        L.oz_exact_dot_err.argtypes = [C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_double, _dp, _dp]
        L.oz_exact_sum_rn.restype = C.c_double
        L.oz_exact_sum_rn.argtypes = [C.c_int, _dp]
        L.oz_exact_gemm_block.restype = None
        L.oz_exact_gemm_block.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, _dp, _dp]
        L.oz_gen_phi.restype = None
        L.oz_gen_phi.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_double, C.c_int]
        L.oz_gen_normal.restype = None
        L.oz_gen_normal.argtypes = [C.c_int, _dp, C.c_int]
        L.oz_stencil7_nnz.restype = C.c_int64
        L.oz_stencil7_nnz.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oz_gen_stencil7.restype = None
        L.oz_gen_stencil7.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _ip]
        L.oz_gen_poisson_shift.restype = None
        L.oz_gen_poisson_shift.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _dp]
        L.oz_csrmv_fma.restype = None
        L.oz_csrmv_fma.argtypes = [C.c_int, _dp, _ip, _ip, _dp, _dp]

    # ---- generators ----
    def phi_matrix(self, m, n, phi, seed, ld=None):
        ld = ld or m
        a = np.zeros((n, ld), dtype=np.float64)  # column-major storage: row j of `a` is column j
        self.L.oz_gen_phi(m, n, ld, _d(a), phi, seed)
        return a

    def phi_vector(self, n, phi, seed):
        v = np.zeros(max(n, 1), dtype=np.float64)
        self.L.oz_gen_phi(n, 1, n, _d(v), phi, seed)
        return v[:n]

    def normal(self, n, seed):
        v = np.zeros(n, dtype=np.float64)
        self.L.oz_gen_normal(n, _d(v), seed)
        return v

    def stencil7(self, nx, ny, nz):
        n = nx * ny * nz
        nnz = self.L.oz_stencil7_nnz(nx, ny, nz)
        rowptr = np.zeros(n + 1, dtype=np.int32)
        colind = np.zeros(nnz, dtype=np.int32)
        self.L.oz_gen_stencil7(nx, ny, nz, _i(rowptr), _i(colind))
        return rowptr, colind

    def poisson_shift(self, nx, ny, nz, seed, rowptr, colind):
        val = np.zeros(len(colind), dtype=np.float64)
        self.L.oz_gen_poisson_shift(nx, ny, nz, seed, _i(rowptr), _i(colind), _d(val))
        return val

    def csrmv_fma(self, val, colind, rowptr, x):
        m = len(rowptr) - 1
        y = np.zeros(m, dtype=np.float64)
        self.L.oz_csrmv_fma(m, _d(val), _i(colind), _i(rowptr), _d(x), _d(y))
        return y

    # ---- restated routines ----
    def rho(self, dim, mode=0):
        return self.L.oz_rho(dim, mode)

    def tau_libm(self, v):
        return self.L.oz_tau_libm(v)

    def split_cols(self, flags, X, shift=1):
        """X: (ncol, k) array = column-major k x ncol panel.  Returns (nsplit, slices[nsplit, ncol, k])."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        ncol, k = X.shape
        maxS = flags.nSplitMax if flags.nSplitMax > 0 else 30
        out = np.zeros((maxS + 1, ncol, max(k, 1)), dtype=np.float64)
        s = self.L.oz_split_cols(C.byref(flags), k, ncol, _d(X), max(k, 1), shift, _d(out), max(k, 1))
        return s, out[:s, :, :k]

    def rho_f32(self, dim, mode=0):
        return self.L.oz_rho_f32(dim, mode)

    def split_cols_f32(self, flags, X, shift=1):
        """Mixed form: (nsplit, float slices[nsplit, ncol, k], short exps[nsplit, ncol])."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        ncol, k = X.shape
        maxS = flags.nSplitMax if flags.nSplitMax > 0 else 30
        out = np.zeros((maxS + 1, ncol, max(k, 1)), dtype=np.float32)
        ex = np.zeros((maxS + 1, max(ncol, 1)), dtype=np.int16)
        s = self.L.oz_split_cols_f32(C.byref(flags), k, ncol, _d(X), max(k, 1), shift,
                                     out.ctypes.data_as(C.POINTER(C.c_float)), max(k, 1),
                                     ex.ctypes.data_as(C.POINTER(C.c_short)))
        return s, out[:s, :, :k], ex[:s, :ncol]

    def dgemm_f32(self, flags, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """GEMM <double, float, float> (FSum only); (C, info), or (None, None) for unsupported flags."""
        info = Info()
        Cc = np.array(C_, dtype=np.float64, copy=True)
        r = self.L.oz_dgemm_f32(C.byref(flags), ta.encode(), tb.encode(), m, n, k, alpha, _d(A), lda, _d(B), ldb,
                                beta, _d(Cc), ldc, C.byref(info))
        return (Cc, info) if r == 0 else (None, None)

    def rho_sd(self, dim, mode=0):
        return self.L.oz_rho_sd(dim, mode)

    def tau_sd_libm(self, v):
        return self.L.oz_tau_sd_libm(v)

    def tau_sd_sweep(self, rule_fn_addr, stride):
        """Disagreements of a C rule int(float) with the reference's float tau over strided float bits."""
        first = C.c_uint(0)
        bad = self.L.oz_tau_sd_sweep(rule_fn_addr, stride, C.byref(first))
        return bad, first.value

    def split_cols_sd(self, flags, X, shift=1):
        """<float, double, double>: (nsplit, double slices[nsplit, ncol, k], short exps[nsplit, ncol])."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        ncol, k = X.shape
        maxS = flags.nSplitMax if flags.nSplitMax > 0 else 30
        out = np.zeros((maxS + 1, ncol, max(k, 1)), dtype=np.float64)
        ex = np.zeros((maxS + 1, max(ncol, 1)), dtype=np.int16)
        s = self.L.oz_split_cols_sd(C.byref(flags), k, ncol, _f(X), max(k, 1), shift, _d(out), max(k, 1),
                                    ex.ctypes.data_as(C.POINTER(C.c_short)))
        return s, out[:s, :, :k], ex[:s, :ncol]

    def sgemm_d(self, flags, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """GEMM <float, double, double> (FSum only); (C, info), or (None, None) for unsupported flags."""
        info = Info()
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(B, dtype=np.float32)
        Cc = np.array(C_, dtype=np.float32, copy=True)
        r = self.L.oz_sgemm_d(C.byref(flags), ta.encode(), tb.encode(), m, n, k, alpha, _f(A), lda, _f(B), ldb,
                              beta, _f(Cc), ldc, C.byref(info))
        return (Cc, info) if r == 0 else (None, None)

    # ---- quad I/O form: binary128 arrays are uint64 arrays with a last axis (lo, hi) ----
    def rho_q(self, dim, mode=0):
        return self.L.oz_rho_q(dim, mode)

    def tau_q_libm(self, v):
        v = np.ascontiguousarray(v, dtype=np.uint64)
        return self.L.oz_tau_q_libm(v.ctypes.data)

    def phi_matrix_q(self, m, n, phi, seed, ld=None):
        ld = ld or m
        a = np.zeros((n, ld, 2), dtype=np.uint64)
        self.L.oz_gen_phi_q(m, n, ld, a.ctypes.data, phi, seed)
        return a

    def phi_vector_q(self, n, phi, seed):
        v = np.zeros((max(n, 1), 2), dtype=np.uint64)
        self.L.oz_gen_phi_q(n, 1, n, v.ctypes.data, phi, seed)
        return v[:n]

    def q(self, d):
        """binary128 of a double (exact)."""
        r = np.zeros(2, dtype=np.uint64)
        self.L.oz_q_from_double(float(d), r.ctypes.data)
        return r

    def q_scale(self, x, e):
        """Copy of a binary128 array scaled by 2^e (scalbnq)."""
        y = np.array(x, dtype=np.uint64, copy=True)
        self.L.oz_q_scale(y.ctypes.data, y.size // 2, e)
        return y

    def q_to_double(self, v):
        v = np.ascontiguousarray(v, dtype=np.uint64)
        return self.L.oz_q_to_double(v.ctypes.data)

    def q_op(self, op, a, b, c=None):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        r = np.zeros(2, dtype=np.uint64)
        if op == "fma":
            c = np.ascontiguousarray(c, dtype=np.uint64)
            self.L.oz_q_fma(a.ctypes.data, b.ctypes.data, c.ctypes.data, r.ctypes.data)
        else:
            getattr(self.L, "oz_q_" + op)(a.ctypes.data, b.ctypes.data, r.ctypes.data)
        return r

    def q128_check(self, rule_addr, op, n, seed=1):
        """Mismatches of a software binary128 rule against __float128 / libquadmath (see ozoracle.c)."""
        first = np.zeros(10, dtype=np.uint64)
        bad = self.L.oz_q128_check(rule_addr, op, n, seed, first.ctypes.data)
        return bad, first

    def qgemm_d(self, flags, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """GEMM <__float128, double, double> (FSum only); (C, info), or (None, None) for unsupported flags."""
        info = Info()
        A = np.ascontiguousarray(A, dtype=np.uint64)
        B = np.ascontiguousarray(B, dtype=np.uint64)
        al = np.ascontiguousarray(alpha, dtype=np.uint64)
        be = np.ascontiguousarray(beta, dtype=np.uint64)
        Cc = np.array(C_, dtype=np.uint64, copy=True)
        r = self.L.oz_qgemm_d(C.byref(flags), ta.encode(), tb.encode(), m, n, k, al.ctypes.data, A.ctypes.data, lda,
                              B.ctypes.data, ldb, be.ctypes.data, Cc.ctypes.data, ldc, C.byref(info))
        return (Cc, info) if r == 0 else (None, None)

    def split_csr(self, flags, val, rowptr, shift=1):
        m = len(rowptr) - 1
        nnz = len(val)
        maxS = flags.nSplitMax if flags.nSplitMax > 0 else 30
        out = np.zeros((maxS + 1, max(nnz, 1)), dtype=np.float64)
        s = self.L.oz_split_rows_csr(C.byref(flags), m, _d(val), _i(rowptr), shift, _d(out), max(nnz, 1))
        return s, out[:s, :nnz]

    def nearsum(self, v):
        v = np.array(v, dtype=np.float64)
        return self.L.oz_nearsum(len(v), _d(v))

    def dgemm(self, flags, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        info = Info()
        Cc = np.array(C_, dtype=np.float64, copy=True)
        self.L.oz_dgemm(C.byref(flags), ta.encode(), tb.encode(), m, n, k, alpha, _d(A), lda, _d(B), ldb, beta,
                        _d(Cc), ldc, C.byref(info))
        return Cc, info

    def ddot(self, flags, x, y):
        info = Info()
        r = self.L.oz_ddot(C.byref(flags), len(x), _d(x), _d(y), C.byref(info))
        return r, info

    def dnrm2(self, flags, x):
        info = Info()
        return self.L.oz_dnrm2(C.byref(flags), len(x), _d(x), C.byref(info)), info

    def dgemv(self, flags, ta, m, n, alpha, A, lda, x, beta, y):
        info = Info()
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.oz_dgemv(C.byref(flags), ta.encode(), m, n, alpha, _d(A), lda, _d(x), beta, _d(yy), C.byref(info))
        return yy, info

    def dcsrmv(self, flags, m, n, alpha, val, colind, rowptr, x, beta, y):
        info = Info()
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.oz_dcsrmv(C.byref(flags), m, n, len(val), alpha, _d(val), _i(colind), _i(rowptr), _d(x), beta,
                         _d(yy), C.byref(info))
        return yy, info

    def dcsrmv_split_a(self, flags, val, rowptr):
        m = len(rowptr) - 1
        nnz = len(val)
        maxS = flags.nSplitMax if flags.nSplitMax > 0 else 30
        out = np.zeros((maxS + 1, max(nnz, 1)), dtype=np.float64)
        ns = C.c_int()
        sh = C.c_int()
        self.L.oz_dcsrmv_split_a(C.byref(flags), m, nnz, _d(val), _i(rowptr), _d(out), max(nnz, 1),
                                 C.byref(ns), C.byref(sh))
        return ns.value, sh.value, out[:ns.value, :nnz]

    def dcg(self, flags, val, colind, rowptr, b, x0, maxiter, tol):
        n = len(b)
        info = Info()
        x = np.array(x0, dtype=np.float64, copy=True)
        hist = np.zeros(maxiter + 1, dtype=np.float64)
        self.L.oz_dcg(C.byref(flags), n, len(val), _d(val), _i(colind), _i(rowptr), _d(b), _d(x), maxiter, tol,
                      _d(hist), C.byref(info))
        return x, hist[: info.cg_numiter + 1], info

    # ---- exact arithmetic ----
    def exact_dot(self, x, y):
        return self.L.oz_exact_dot_rn(len(x), _d(x), 1, _d(y), 1)

    def exact_dot_err(self, x, y, c, incx=1, incy=1, n=None):
        n = len(x) if n is None else n
        rn = C.c_double()
        rel = C.c_double()
        self.L.oz_exact_dot_err(n, _d(x), incx, _d(y), incy, c, C.byref(rn), C.byref(rel))
        return rn.value, rel.value

    def exact_gemm_block(self, Arows, Bcols, Cblk):
        """RN(exact) and the relative error of every computed entry of a GEMM block: Arows (nr x k, row i of op(A)),
        Bcols (nc x k, column j of op(B)), Cblk (nc x nr: column-major nr x nc block of computed values)."""
        Arows = np.ascontiguousarray(Arows, dtype=np.float64)
        Bcols = np.ascontiguousarray(Bcols, dtype=np.float64)
        Cblk = np.ascontiguousarray(Cblk, dtype=np.float64)
        nr, k = Arows.shape
        nc = Bcols.shape[0]
        assert Bcols.shape[1] == k and Cblk.size == nr * nc
        rn = np.zeros(nr * nc)
        rel = np.zeros(nr * nc)
        self.L.oz_exact_gemm_block(k, nr, _d(Arows), nc, _d(Bcols), _d(Cblk), _d(rn), _d(rel))
        return rn.reshape(nc, nr), rel.reshape(nc, nr)

    def exact_sum(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        return self.L.oz_exact_sum_rn(len(v), _d(v))


class Reference:
    """The reference OzBLAS CPU library (built from its own sources into _ref/)."""

    def __init__(self, work_bytes=int(16e9), threads=None):
        if not os.path.exists(LIB_REF):
            raise FileNotFoundError(LIB_REF)
        L = C.CDLL(LIB_REF)
        self.L = L
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_uint64]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_flags.argtypes = [C.c_void_p] + [C.c_int] * 9
        L.ref_get_info.argtypes = [C.c_void_p, C.POINTER(C.c_float), _ip]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_get_threads.restype = C.c_int
        L.ref_dgemm.argtypes = [C.c_void_p, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, _dp,
                                C.c_int, _dp, C.c_int, C.c_double, _dp, C.c_int]
        L.ref_dgemm_f32.argtypes = L.ref_dgemm.argtypes
        L.ref_ddot_f32.restype = C.c_double
        L.ref_ddot_f32.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.ref_dnrm2_f32.restype = C.c_double
        L.ref_dnrm2_f32.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_dgemv_f32.argtypes = [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp,
                                    C.c_double, _dp]
        _fp = C.POINTER(C.c_float)
        L.ref_sgemm_d.argtypes = [C.c_void_p, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_float, _fp,
                                  C.c_int, _fp, C.c_int, C.c_float, _fp, C.c_int]
        L.ref_sdot_d.restype = C.c_float
        L.ref_sdot_d.argtypes = [C.c_void_p, C.c_int, _fp, _fp]
        L.ref_snrm2_d.restype = C.c_float
        L.ref_snrm2_d.argtypes = [C.c_void_p, C.c_int, _fp]
        L.ref_sgemv_d.argtypes = [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_float, _fp, C.c_int, _fp,
                                  C.c_float, _fp]
        L.ref_log21f.restype = C.c_float
        L.ref_log21f.argtypes = [C.c_float]
        L.ref_qgemm_d.argtypes = [C.c_void_p, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.ref_qdot_d.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_qnrm2_d.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_tau_q.restype = C.c_int
        L.ref_tau_q.argtypes = [C.c_void_p]
        L.ref_ddot.restype = C.c_double
        L.ref_ddot.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.ref_dnrm2.restype = C.c_double
        L.ref_dnrm2.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_dgemv.argtypes = [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp,
                                C.c_double, _dp]
        L.ref_daxpy.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.ref_dcsrmv.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _ip, _ip, _dp,
                                 C.c_double, _dp]
        L.ref_dcg.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _ip, _ip, _dp, _dp, C.c_int, C.c_double, _dp,
                              _dp]
        L.ref_split_panel.restype = C.c_int
        L.ref_split_panel.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, _ip]
        L.ref_split_sparse.restype = C.c_int
        L.ref_split_sparse.argtypes = [C.c_void_p, C.c_int, _dp, _ip, C.c_int, _dp, _ip]
        L.ref_tau.restype = C.c_int
        L.ref_tau.argtypes = [C.c_double]
        if threads:
            L.ref_set_threads(threads)
        self.h = L.ref_create(work_bytes)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_flags(self, nSplitMax=0, fastMode=0, sumMode=0, splitEpsMode=0, splitMode=0, reproMode=1,
                  useBatchedGemmFlag=0, verbose=1, trueresFlag=0):
        self.L.ref_set_flags(self.h, nSplitMax, splitMode, fastMode, reproMode, sumMode, splitEpsMode,
                             useBatchedGemmFlag, verbose, trueresFlag)

    def info(self):
        f = (C.c_float * 3)()
        i = (C.c_int * 5)()
        self.L.ref_get_info(self.h, f, i)
        return dict(nSplitA=f[0], nSplitB=f[1], nSplitC=f[2], mbk=i[0], nbk=i[1], splitShift=i[2],
                    nSplitA_=i[3], cg_numiter=i[4])

    def threads(self, n=None):
        if n:
            self.L.ref_set_threads(n)
        return self.L.ref_get_threads()

    def dgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        Cc = np.array(C_, dtype=np.float64, copy=True)
        self.L.ref_dgemm(self.h, ta.encode(), tb.encode(), m, n, k, alpha, _d(A), lda, _d(B), ldb, beta, _d(Cc),
                         ldc)
        return Cc

    def dgemm_f32(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """ozblasRgemm<double, float, float>: double data, FP32 slices and slice products."""
        Cc = np.array(C_, dtype=np.float64, copy=True)
        self.L.ref_dgemm_f32(self.h, ta.encode(), tb.encode(), m, n, k, alpha, _d(A), lda, _d(B), ldb, beta,
                             _d(Cc), ldc)
        return Cc

    def sgemm_d(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """ozblasRgemm<float, double, double>: float data, FP64 slices and slice products."""
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(B, dtype=np.float32)
        Cc = np.array(C_, dtype=np.float32, copy=True)
        self.L.ref_sgemm_d(self.h, ta.encode(), tb.encode(), m, n, k, alpha, _f(A), lda, _f(B), ldb, beta, _f(Cc),
                           ldc)
        return Cc

    def sdot_d(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        return self.L.ref_sdot_d(self.h, len(x), _f(x), _f(y))

    def snrm2_d(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        return self.L.ref_snrm2_d(self.h, len(x), _f(x))

    def sgemv_d(self, ta, m, n, alpha, A, lda, x, beta, y):
        A = np.ascontiguousarray(A, dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        yy = np.array(y, dtype=np.float32, copy=True)
        self.L.ref_sgemv_d(self.h, ta.encode(), m, n, alpha, _f(A), lda, _f(x), beta, _f(yy))
        return yy

    def log21f(self, v):
        return self.L.ref_log21f(v)

    def qgemm_d(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc):
        """ozblasRgemm<__float128, double, double> on 16-byte binary128 arrays (uint64 pairs)."""
        A = np.ascontiguousarray(A, dtype=np.uint64)
        B = np.ascontiguousarray(B, dtype=np.uint64)
        al = np.ascontiguousarray(alpha, dtype=np.uint64)
        be = np.ascontiguousarray(beta, dtype=np.uint64)
        Cc = np.array(C_, dtype=np.uint64, copy=True)
        self.L.ref_qgemm_d(self.h, ta.encode(), tb.encode(), m, n, k, al.ctypes.data, A.ctypes.data, lda,
                           B.ctypes.data, ldb, be.ctypes.data, Cc.ctypes.data, ldc)
        return Cc

    def qdot_d(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        y = np.ascontiguousarray(y, dtype=np.uint64)
        r = np.zeros(2, dtype=np.uint64)
        self.L.ref_qdot_d(self.h, len(x), x.ctypes.data, y.ctypes.data, r.ctypes.data)
        return r

    def qnrm2_d(self, x):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        r = np.zeros(2, dtype=np.uint64)
        self.L.ref_qnrm2_d(self.h, len(x), x.ctypes.data, r.ctypes.data)
        return r

    def tau_q(self, v):
        v = np.ascontiguousarray(v, dtype=np.uint64)
        return self.L.ref_tau_q(v.ctypes.data)

    def ddot_f32(self, x, y):
        return self.L.ref_ddot_f32(self.h, len(x), _d(x), _d(y))

    def dnrm2_f32(self, x):
        return self.L.ref_dnrm2_f32(self.h, len(x), _d(x))

    def dgemv_f32(self, ta, m, n, alpha, A, lda, x, beta, y):
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.ref_dgemv_f32(self.h, ta.encode(), m, n, alpha, _d(A), lda, _d(x), beta, _d(yy))
        return yy

    def ddot(self, x, y):
        return self.L.ref_ddot(self.h, len(x), _d(x), _d(y))

    def dnrm2(self, x):
        return self.L.ref_dnrm2(self.h, len(x), _d(x))

    def dgemv(self, ta, m, n, alpha, A, lda, x, beta, y):
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.ref_dgemv(self.h, ta.encode(), m, n, alpha, _d(A), lda, _d(x), beta, _d(yy))
        return yy

    def daxpy(self, alpha, x, y):
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.ref_daxpy(self.h, len(x), alpha, _d(x), _d(yy))
        return yy

    def dcsrmv(self, m, n, alpha, val, colind, rowptr, x, beta, y):
        yy = np.array(y, dtype=np.float64, copy=True)
        self.L.ref_dcsrmv(self.h, m, n, len(val), alpha, _d(val), _i(colind), _i(rowptr), _d(x), beta, _d(yy))
        return yy

    def dcg(self, val, colind, rowptr, b, x0, maxiter, tol):
        x = np.array(x0, dtype=np.float64, copy=True)
        h1 = np.zeros(maxiter + 2, dtype=np.float64)
        h2 = np.zeros(maxiter + 2, dtype=np.float64)
        self.L.ref_dcg(self.h, len(b), len(val), _d(val), _i(colind), _i(rowptr), _d(b), _d(x), maxiter, tol,
                       _d(h1), _d(h2))
        it = self.info()["cg_numiter"]
        return x, h1[: it + 1]

    def split_panel(self, X, nSplitMax=0):
        X = np.ascontiguousarray(X, dtype=np.float64)
        ncol, k = X.shape
        maxS = nSplitMax if nSplitMax > 0 else 30
        ld = ((k + 7) // 8) * 8
        out = np.zeros((maxS + 2) * ld * max(ncol, 1) + 2 * k, dtype=np.float64)
        ldo = C.c_int()
        s = self.L.ref_split_panel(self.h, k, ncol, _d(X), k, _d(out), C.byref(ldo))
        ld = ldo.value
        sl = out[: s * ld * ncol].reshape(s, ncol, ld)[:, :, :k]
        return s, sl

    def split_sparse(self, val, rowptr, nSplitMax=0):
        m = len(rowptr) - 1
        nnz = len(val)
        maxS = nSplitMax if nSplitMax > 0 else 30
        ld = ((nnz + 7) // 8) * 8
        out = np.zeros((maxS + 2) * max(ld, 8), dtype=np.float64)
        ldo = C.c_int()
        s = self.L.ref_split_sparse(self.h, m, _d(val), _i(rowptr), nnz, _d(out), C.byref(ldo))
        ld = ldo.value
        return s, out[: s * ld].reshape(s, ld)[:, :nnz]

    def tau(self, v):
        return self.L.ref_tau(v)


def have_reference():
    return os.path.exists(LIB_REF)
