"""Generate the golden fixtures from the reference library itself.

    python tests/golden/make_golden.py [--cg]

Inputs are regenerated from seeds by the reference harness's phi generator
(testing/testing_common.cpp:703-717, restated in oracle/ozoracle.c) and the
stencil/Poisson builders; outputs come from the reference OzBLAS CPU library
(oracle/_ref, built unmodified from mukunoki/ozblas src/cpu).  Small cases
are stored whole (small.npz); full-size configurations are stored as the
SHA-256 of their FP64 output bytes plus sampled values (full.json).
``--cg`` also runs the 2000-iteration CG on the 100^3 Poisson problem
(about 15 minutes) into cg100.json.

Needs oracle/_ref (built where the reference sources exist).  The fixtures it
writes are committed; the tests only read them.
"""
import hashlib
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference, Restatement  # noqa: E402

# m, n, k, ta, tb, sumMode, fastMode, alpha, beta, phi
GEMM_CASES = [
    (1, 1, 1, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (2, 3, 7, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "t", "n", 1, 0, 1.0, 0.0, 1.0),
    (7, 9, 130, "n", "t", 0, 0, -0.5, 2.0, 1.0),
    (20, 20, 64, "t", "t", 0, 2, 1.0, 1.0, 1.0),
    (16, 12, 77, "n", "n", 1, 1, 1.0, 0.0, 1.0),
    (65, 129, 33, "n", "n", 0, 0, 1.5, -1.0, 2.0),
    (130, 70, 300, "n", "n", 1, 0, 1.0, 0.0, 4.0),
    (64, 64, 1, "n", "n", 0, 0, 1.0, 0.0, 0.5),
    (100, 3, 512, "t", "n", 0, 0, 1.0, 0.0, 1.0),
]
DOT_CASES = [(1, 1.0), (7, 1.0), (1000, 2.0), (100003, 2.0)]
GEMV_CASES = [(50, 70, "n", 0, 0), (50, 70, "t", 1, 0), (300, 257, "n", 1, 0), (64, 1000, "n", 0, 1)]
CSR_GRIDS = [(4, 3, 2), (12, 10, 9)]


def gemm_inputs(R, case):
    m, n, k, ta, tb, sm, fm, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    return R.phi_matrix(ar, ac, phi, 1), R.phi_matrix(br, bc, phi, 2), R.phi_matrix(m, n, 1.0, 3), ar, br


def case_key(prefix, case):
    return prefix + "_" + "_".join(str(c) for c in case)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def hexd(v):
    return float(v).hex()


def small(R, ref):
    out = {}
    for case in GEMM_CASES:
        m, n, k, ta, tb, sm, fm, alpha, beta, phi = case
        A, B, C0, lda, ldb = gemm_inputs(R, case)
        ref.set_flags(sumMode=sm, fastMode=fm)
        out[case_key("gemm", case)] = ref.dgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C0, m)
        inf = ref.info()
        out[case_key("gemm", case) + "_split"] = np.array([inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]])
    for n, phi in DOT_CASES:
        x, y = R.phi_vector(n, phi, 1), R.phi_vector(n, phi, 2)
        for sm in (0, 1):
            ref.set_flags(sumMode=sm)
            out[f"dot_{n}_{phi}_{sm}"] = np.array([ref.ddot(x, y), ref.dnrm2(x)])
    for m, n, tr, sm, fm in GEMV_CASES:
        A = R.phi_matrix(m, n, 1.0, 1)
        xl, yl = (n, m) if tr == "n" else (m, n)
        x, y0 = R.phi_vector(xl, 1.0, 2), R.phi_vector(yl, 1.0, 3)
        ref.set_flags(sumMode=sm, fastMode=fm)
        out[f"gemv_{m}_{n}_{tr}_{sm}_{fm}"] = ref.dgemv(tr, m, n, 0.75, A, m, x, 0.5, y0)
    for g in CSR_GRIDS:
        rowptr, colind = R.stencil7(*g)
        nn = len(rowptr) - 1
        val = R.phi_vector(len(colind), 1.0, 1)
        x, y0 = R.phi_vector(nn, 1.0, 2), R.phi_vector(nn, 1.0, 3)
        for sm in (0, 1):
            for al, be in [(1.0, 0.0), (-1.0, 1.0), (0.5, 2.0)]:
                ref.set_flags(sumMode=sm)
                out[f"csrmv_{g[0]}x{g[1]}x{g[2]}_{sm}_{al}_{be}"] = ref.dcsrmv(nn, nn, al, val, colind, rowptr, x,
                                                                              be, y0)
    for sm in (0, 1):
        # one solve per fresh process: the reference computes q = A p with
        # beta = 0 into a freshly new-ed (uninitialised) q
        # (src/cpu/ozblas_cg.cpp:48,84), so heap memory reused from an earlier
        # solve can turn 0 * garbage into NaN
        ctx = mp.get_context("spawn")
        with ctx.Pool(1) as pool:
            x, h = pool.apply(_cg12_fresh, (sm,))
        out[f"cg12_{sm}_x"] = x
        out[f"cg12_{sm}_hist"] = h
    np.savez_compressed(os.path.join(HERE, "small.npz"), **out)
    print("small.npz:", len(out), "arrays")


def _cg12_fresh(sm):
    R = Restatement()
    ref = Reference(work_bytes=int(1e9))
    nx = 12
    rowptr, colind = R.stencil7(nx, nx, nx)
    nn = len(rowptr) - 1
    val = R.poisson_shift(nx, nx, nx, 3, rowptr, colind)
    b = R.csrmv_fma(val, colind, rowptr, R.normal(nn, 4))
    ref.set_flags(sumMode=sm, verbose=1)
    return ref.dcg(val, colind, rowptr, b, np.zeros(nn), 60, 0.0)


def full(R, ref):
    res = {}
    m = n = k = 1024
    A, B = R.phi_matrix(m, k, 1.0, 1), R.phi_matrix(k, n, 1.0, 2)
    for sm in (0, 1):
        ref.set_flags(sumMode=sm)
        C = ref.dgemm("n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
        inf = ref.info()
        res[f"gemm1024_{sm}"] = dict(sha256=sha(C), sample=[hexd(C[j, i]) for i, j in [(0, 0), (1023, 0), (5, 700),
                                                                                       (1023, 1023)]],
                                     nSplit=[inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]])
    nv = 1 << 24
    x, y = R.phi_vector(nv, 2.0, 1), R.phi_vector(nv, 2.0, 2)
    for sm in (0, 1):
        ref.set_flags(sumMode=sm)
        d = ref.ddot(x, y)
        inf = ref.info()
        res[f"dot2p24_{sm}"] = dict(dot=hexd(d), nrm2=hexd(ref.dnrm2(x)), nSplit=[inf["nSplitA"], inf["nSplitB"]])
    A = R.phi_matrix(8192, 8192, 1.0, 1)
    xg = R.phi_vector(8192, 1.0, 2)
    for sm in (0, 1):
        ref.set_flags(sumMode=sm)
        yg = ref.dgemv("n", 8192, 8192, 1.0, A, 8192, xg, 0.0, np.zeros(8192))
        res[f"gemv8192_{sm}"] = dict(sha256=sha(yg), sample=[hexd(yg[i]) for i in (0, 4095, 8191)])
    del A
    rowptr, colind = R.stencil7(128, 128, 128)
    nn = len(rowptr) - 1
    val = R.phi_vector(len(colind), 1.0, 1)
    xs = R.phi_vector(nn, 1.0, 2)
    for sm in (0, 1):
        ref.set_flags(sumMode=sm)
        yv = ref.dcsrmv(nn, nn, 1.0, val, colind, rowptr, xs, 0.0, np.zeros(nn))
        inf = ref.info()
        res[f"csrmv128_{sm}"] = dict(sha256=sha(yv), sample=[hexd(yv[i]) for i in (0, nn // 2, nn - 1)],
                                     nSplit=[inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]])
    with open(os.path.join(HERE, "full.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("full.json:", list(res))


def cg100(R, ref, iters=2000):
    nx = 100
    rowptr, colind = R.stencil7(nx, nx, nx)
    nn = len(rowptr) - 1
    val = R.poisson_shift(nx, nx, nx, 3, rowptr, colind)
    b = R.csrmv_fma(val, colind, rowptr, R.normal(nn, 4))
    ref.set_flags(sumMode=1, verbose=1)
    x, h = ref.dcg(val, colind, rowptr, b, np.zeros(nn), iters, 0.0)
    inf = ref.info()
    res = dict(iters=iters, sumMode=1, hist_sha256=sha(h), x_sha256=sha(x), hist_head=[hexd(v) for v in h[:5]],
               hist_tail=[hexd(v) for v in h[-5:]], splitShift=inf["splitShift"], nSplitA_=inf["nSplitA_"],
               cg_numiter=inf["cg_numiter"])
    np.save(os.path.join(HERE, "cg100_hist.npy"), h)
    with open(os.path.join(HERE, "cg100.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("cg100.json", res["cg_numiter"], h[-1])


if __name__ == "__main__":
    R = Restatement()
    ref = Reference(work_bytes=int(40e9))
    if "--cg" in sys.argv:
        cg100(R, ref)
    else:
        small(R, ref)
        full(R, ref)
