"""The oracle itself, pinned (CPU only).

* The C restatement (oracle/ozoracle.c) against the golden fixtures made by
  the reference library (tests/golden/make_golden.py): bit-exact.
* The restatement against the live reference library (oracle/_ref) on more
  shapes and flags, when that library is present: bit-exact, split counts
  included.
* The exact accumulator against mpmath.
* The library's C ABI: loads and exports every symbol include/cuozblas.h declares.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.oracle import make_flags
from tests.conftest import bits_equal, first_diff
from tests.golden.make_golden import (CSR_GRIDS, DOT_CASES, GEMM_CASES, GEMV_CASES, case_key, gemm_inputs,
                                      sha)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def small():
    return np.load(os.path.join(GOLD, "small.npz"))


@pytest.mark.parametrize("case", GEMM_CASES, ids=lambda c: case_key("g", c))
def test_gemm_golden(case, oracle, small):
    m, n, k, ta, tb, sm, fm, alpha, beta, phi = case
    A, B, C0, lda, ldb = gemm_inputs(oracle, case)
    out, info = oracle.dgemm(make_flags(sumMode=sm, fastMode=fm), ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C0,
                             m)
    gold = small[case_key("gemm", case)]
    assert bits_equal(out, gold), first_diff(out, gold)
    assert list(small[case_key("gemm", case) + "_split"]) == [info.nSplitA, info.nSplitB, info.nSplitC]


@pytest.mark.parametrize("n,phi", DOT_CASES)
@pytest.mark.parametrize("sm", [0, 1])
def test_dot_golden(n, phi, sm, oracle, small):
    x, y = oracle.phi_vector(n, phi, 1), oracle.phi_vector(n, phi, 2)
    d, _ = oracle.ddot(make_flags(sumMode=sm), x, y)
    r, _ = oracle.dnrm2(make_flags(sumMode=sm), x)
    assert bits_equal(np.array([d, r]), small[f"dot_{n}_{phi}_{sm}"])


@pytest.mark.parametrize("case", GEMV_CASES)
def test_gemv_golden(case, oracle, small):
    m, n, tr, sm, fm = case
    A = oracle.phi_matrix(m, n, 1.0, 1)
    xl, yl = (n, m) if tr == "n" else (m, n)
    x, y0 = oracle.phi_vector(xl, 1.0, 2), oracle.phi_vector(yl, 1.0, 3)
    out, _ = oracle.dgemv(make_flags(sumMode=sm, fastMode=fm), tr, m, n, 0.75, A, m, x, 0.5, y0)
    assert bits_equal(out, small[f"gemv_{m}_{n}_{tr}_{sm}_{fm}"])


@pytest.mark.parametrize("g", CSR_GRIDS)
@pytest.mark.parametrize("sm", [0, 1])
def test_csrmv_golden(g, sm, oracle, small):
    rowptr, colind = oracle.stencil7(*g)
    nn = len(rowptr) - 1
    val = oracle.phi_vector(len(colind), 1.0, 1)
    x, y0 = oracle.phi_vector(nn, 1.0, 2), oracle.phi_vector(nn, 1.0, 3)
    for al, be in [(1.0, 0.0), (-1.0, 1.0), (0.5, 2.0)]:
        out, _ = oracle.dcsrmv(make_flags(sumMode=sm), nn, nn, al, val, colind, rowptr, x, be, y0)
        gold = small[f"csrmv_{g[0]}x{g[1]}x{g[2]}_{sm}_{al}_{be}"]
        assert bits_equal(out, gold), first_diff(out, gold)


@pytest.mark.parametrize("sm", [0, 1])
def test_cg_golden(sm, oracle, small):
    nx = 12
    rowptr, colind = oracle.stencil7(nx, nx, nx)
    nn = len(rowptr) - 1
    val = oracle.poisson_shift(nx, nx, nx, 3, rowptr, colind)
    b = oracle.csrmv_fma(val, colind, rowptr, oracle.normal(nn, 4))
    x, h, _ = oracle.dcg(make_flags(sumMode=sm), val, colind, rowptr, b, np.zeros(nn), 60, 0.0)
    assert bits_equal(h, small[f"cg12_{sm}_hist"]) and bits_equal(x, small[f"cg12_{sm}_x"])


@pytest.mark.slow
def test_gemm1024_golden_hash(oracle):
    """BASELINE config 1 (1024^3, phi=1): the restatement reproduces the reference's output hash."""
    with open(os.path.join(GOLD, "full.json")) as f:
        full = json.load(f)
    A, B = oracle.phi_matrix(1024, 1024, 1.0, 1), oracle.phi_matrix(1024, 1024, 1.0, 2)
    # the restatement's naive triple loop is slow at 1024^3; check one 64-row block of the hash's sample
    m = 64
    Ab = np.ascontiguousarray(A[:, :m])  # first 64 rows of A (column-major slice)
    out, info = oracle.dgemm(make_flags(), "n", "n", m, 1024, 1024, 1.0, Ab, m, B, 1024, 0.0,
                             np.zeros((1024, m)), m)
    assert float(out[0, 0]).hex() == full["gemm1024_0"]["sample"][0]
    assert float(out[700, 5]).hex() == full["gemm1024_0"]["sample"][2]


def test_dot_full_golden(oracle):
    with open(os.path.join(GOLD, "full.json")) as f:
        full = json.load(f)
    n = 1 << 24
    x, y = oracle.phi_vector(n, 2.0, 1), oracle.phi_vector(n, 2.0, 2)
    for sm in (0, 1):
        d, info = oracle.ddot(make_flags(sumMode=sm), x, y)
        assert float(d).hex() == full[f"dot2p24_{sm}"]["dot"]
        assert [info.nSplitA, info.nSplitB] == full[f"dot2p24_{sm}"]["nSplit"]


# ---- live reference (only where oracle/_ref exists) ----

@pytest.mark.parametrize("seed", range(6))
def test_restatement_vs_reference_random_shapes(seed, oracle, reference):
    rng = np.random.default_rng(100 + seed)
    m, n, k = (int(v) for v in rng.integers(1, 90, 3))
    k = int(rng.integers(1, 700))
    ta, tb = rng.choice(["n", "t"]), rng.choice(["n", "t"])
    sm, fm = int(rng.integers(0, 2)), int(rng.integers(0, 3))
    nsplit = int(rng.choice([0, 0, 2, 5]))
    phi = float(rng.choice([0.5, 1.0, 2.0, 4.0]))
    case = (m, n, k, ta, tb, sm, fm, 1.25, -0.5, phi)
    A, B, C0, lda, ldb = gemm_inputs(oracle, case)
    out, info = oracle.dgemm(make_flags(sumMode=sm, fastMode=fm, nSplitMax=nsplit), ta, tb, m, n, k, 1.25, A, lda,
                             B, ldb, -0.5, C0, m)
    reference.set_flags(sumMode=sm, fastMode=fm, nSplitMax=nsplit)
    gold = reference.dgemm(ta, tb, m, n, k, 1.25, A, lda, B, ldb, -0.5, C0, m)
    assert bits_equal(out, gold), (case, nsplit, first_diff(out, gold))
    inf = reference.info()
    assert [info.nSplitA, info.nSplitB, info.nSplitC] == [inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]]


@pytest.mark.parametrize("n,phi", [(1, 1.0), (37, 1.0), (1000, 2.0), (20000, 1.0), (65537, 4.0)])
@pytest.mark.parametrize("sm", [0, 1])
def test_dot2_dot_vs_reference_one_thread(n, phi, sm, oracle, reference):
    """Dot2 (splitEpsMode 2) DOT: the restatement follows the reference run by one OpenMP thread
    (its double-double partials are combined in critical-section order, so only one thread is
    reproducible)."""
    x = oracle.phi_vector(n, phi, 1)
    y = oracle.phi_vector(n, phi, 2)
    r, info = oracle.ddot(make_flags(sumMode=sm, splitEpsMode=2), x, y)
    prev = reference.threads()
    reference.threads(1)
    try:
        reference.set_flags(sumMode=sm, splitEpsMode=2)
        gold = reference.ddot(x, y)
    finally:
        reference.threads(prev)
    assert np.float64(r).view(np.int64) == np.float64(gold).view(np.int64), (n, phi, sm, r, gold)
    inf = reference.info()
    assert [info.nSplitA, info.nSplitB] == [inf["nSplitA"], inf["nSplitB"]]


@pytest.mark.parametrize("sm", [0, 1])
def test_dot2_csrmv_vs_reference(sm, oracle, reference):
    """Dot2 CSRMV: Dot2i along each row (deterministic for any thread count), hi terms then lo
    terms in the sum."""
    rowptr, colind = oracle.stencil7(9, 8, 7)
    n = len(rowptr) - 1
    val = oracle.phi_vector(len(colind), 2.0, 1)
    x = oracle.phi_vector(n, 2.0, 2)
    y0 = oracle.phi_vector(n, 1.0, 3)
    for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
        out, info = oracle.dcsrmv(make_flags(sumMode=sm, splitEpsMode=2), n, n, alpha, val, colind, rowptr, x,
                                  beta, y0)
        reference.set_flags(sumMode=sm, splitEpsMode=2)
        gold = reference.dcsrmv(n, n, alpha, val, colind, rowptr, x, beta, y0)
        assert bits_equal(out, gold), first_diff(out, gold)
        inf = reference.info()
        assert [info.nSplitA, info.nSplitB, info.nSplitC] == [inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]]


@pytest.mark.parametrize("seed", range(10))
def test_mixed_f32_gemm_vs_reference(seed, oracle, reference):
    """<double, float, float> (FP32 slices with per-line exponents, exact FP32 products, scaled FSum):
    the restatement against ozblasRgemm<double, float, float>, bit-exact with the split counts."""
    rng = np.random.default_rng(300 + seed)
    m, n = (int(v) for v in rng.integers(1, 60, 2))
    k = int(rng.integers(1, 500))
    if seed == 0:
        m = n = 1
    if seed in (1, 2):
        n = 1
    ta, tb = rng.choice(["n", "t"]), rng.choice(["n", "t"])
    fm = int(rng.integers(0, 3)) if seed != 2 else 0
    nsplit = int(rng.choice([0, 0, 2, 5]))
    phi = float(rng.choice([0.5, 1.0, 2.0, 4.0]))
    case = (m, n, k, ta, tb, 0, fm, 1.25, -0.5, phi)
    A, B, C0, lda, ldb = gemm_inputs(oracle, case)
    out, info = oracle.dgemm_f32(make_flags(fastMode=fm, nSplitMax=nsplit), ta, tb, m, n, k, 1.25, A, lda, B, ldb,
                                 -0.5, C0, m)
    reference.set_flags(fastMode=fm, nSplitMax=nsplit)
    gold = reference.dgemm_f32(ta, tb, m, n, k, 1.25, A, lda, B, ldb, -0.5, C0, m)
    assert bits_equal(out, gold), (case, nsplit, first_diff(out, gold))
    inf = reference.info()
    assert [info.nSplitA, info.nSplitB, info.nSplitC] == [inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]]


def test_mixed_f32_skinny_vs_reference(oracle, reference):
    """The mixed DOT, NRM2 and GEMV are the mixed GEMM with m = n = 1 / n = 1
    (src/cpu/ozblas_dot.cpp:25, ozblas_nrm2.cpp:22-29, ozblas_gemv.cpp:22-26); long vectors and
    tiny / huge magnitudes included."""
    reference.set_flags()
    f = make_flags()
    for n, phi, scale in ((1, 1.0, 1.0), (1000, 2.0, 1.0), (100003, 1.0, 1.0), (5000, 4.0, 2.0 ** -1000),
                          (5000, 1.0, 2.0 ** 900), (3000, 1.0, 2.0 ** -1060)):
        x = oracle.phi_vector(n, phi, 1) * scale
        y = oracle.phi_vector(n, phi, 2)
        r, _ = oracle.dgemm_f32(f, "t", "n", 1, 1, n, 1.0, x, n, y, n, 0.0, np.zeros(1), 1)
        gold = reference.ddot_f32(x, y)
        assert bits_equal(r, np.array([gold])), (n, phi, scale, r[0], gold)
        r2, _ = oracle.dgemm_f32(f, "t", "n", 1, 1, n, 1.0, x, n, x, n, 0.0, np.zeros(1), 1)
        assert bits_equal(np.sqrt(r2), np.array([reference.dnrm2_f32(x)]))
    for ta, (m, n) in (("n", (70, 300)), ("t", (300, 70))):
        A = oracle.phi_matrix(m, n, 2.0, 3)
        xl = n if ta == "n" else m
        yl = m if ta == "n" else n
        x = oracle.phi_vector(xl, 2.0, 4)
        y0 = oracle.phi_vector(yl, 1.0, 5)
        if ta == "n":
            out, _ = oracle.dgemm_f32(f, "n", "n", m, 1, n, 0.75, A, m, x, n, 1.5, y0, m)
        else:
            out, _ = oracle.dgemm_f32(f, "t", "n", n, 1, m, 0.75, A, m, x, m, 1.5, y0, n)
        gold = reference.dgemv_f32(ta, m, n, 0.75, A, m, x, 1.5, y0)
        assert bits_equal(out, gold), (ta, first_diff(out, gold))


def test_mixed_f32_split_exactness(oracle):
    """Every FP32 slice is scalbn(FP64 slice, -tau) exactly: at most 53 - rho significant bits, so
    a k-term slice product stays within FP32's 24 bits."""
    for k in (1, 7, 64, 1000, 4096, 1 << 20):
        rho = oracle.rho_f32(k)
        assert 2 * (53 - rho) + np.log2(k) <= 24 + 1e-9, (k, rho)
    x = oracle.phi_matrix(40, 3, 4.0, 9).reshape(3, 40)
    ns, sl, ex = oracle.split_cols_f32(make_flags(), x)
    ns64, sl64 = oracle.split_cols(make_flags(), x)
    # FP64 slices differ (rho differs); the FP32 ones rebuild the input exactly
    rec = np.zeros_like(x)
    for s in range(ns):
        rec += np.ldexp(sl[s].astype(np.float64), ex[s][:, None].astype(np.int64))
    assert np.array_equal(rec, x)
    assert ns > ns64


def f32_bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.int32), b.view(np.int32))


@pytest.mark.parametrize("seed", range(12))
def test_mixed_sd_gemm_vs_reference(seed, oracle, reference):
    """<float, double, double> (float data split in float arithmetic, FP64 slices, each pair product
    rounded and scaled in float, float sum): the restatement against ozblasRgemm<float, double,
    double>, bit-exact with the split counts."""
    rng = np.random.default_rng(500 + seed)
    m, n = (int(v) for v in rng.integers(1, 50, 2))
    k = int(rng.integers(1, 600))
    if seed == 0:
        m = n = 1
    if seed in (1, 2):
        n = 1
    ta, tb = rng.choice(["n", "t"]), rng.choice(["n", "t"])
    fm = int(rng.integers(0, 3))
    nsplit = int(rng.choice([0, 0, 2, 5]))
    phi = float(rng.choice([0.5, 1.0, 2.0, 4.0]))
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1).astype(np.float32)
    B = oracle.phi_matrix(br, bc, phi, 2).astype(np.float32)
    C0 = oracle.phi_matrix(m, n, 1.0, 3).astype(np.float32)
    out, info = oracle.sgemm_d(make_flags(fastMode=fm, nSplitMax=nsplit), ta, tb, m, n, k, 1.25, A, ar, B, br, -0.5,
                               C0, m)
    reference.set_flags(fastMode=fm, nSplitMax=nsplit)
    gold = reference.sgemm_d(ta, tb, m, n, k, 1.25, A, ar, B, br, -0.5, C0, m)
    assert f32_bits_equal(out, gold), (seed, m, n, k, ta, tb, fm, nsplit, phi)
    inf = reference.info()
    assert [info.nSplitA, info.nSplitB, info.nSplitC] == [inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]]


def test_mixed_sd_skinny_vs_reference(oracle, reference):
    """The <float, double, double> DOT, NRM2 and GEMV, including data scaled near the ends of the
    float range (the float scaling then rounds or overflows as the reference's does)."""
    reference.set_flags()
    f = make_flags()
    for n, phi, scale in ((1, 1.0, 1.0), (1000, 2.0, 1.0), (100003, 1.0, 1.0), (5000, 4.0, 2.0 ** -120),
                          (5000, 1.0, 2.0 ** 60), (3000, 1.0, 2.0 ** -140)):
        x = (oracle.phi_vector(n, phi, 1) * scale).astype(np.float32)
        y = oracle.phi_vector(n, phi, 2).astype(np.float32)
        r, _ = oracle.sgemm_d(f, "t", "n", 1, 1, n, 1.0, x, n, y, n, 0.0, np.zeros(1, np.float32), 1)
        gold = reference.sdot_d(x, y)
        assert f32_bits_equal(r, np.array([gold], np.float32)), (n, phi, scale, r[0], gold)
        r2, _ = oracle.sgemm_d(f, "t", "n", 1, 1, n, 1.0, x, n, x, n, 0.0, np.zeros(1, np.float32), 1)
        nr = np.float32(np.sqrt(np.float64(r2[0])))
        assert f32_bits_equal(np.array([nr]), np.array([reference.snrm2_d(x)], np.float32))
    for ta, (m, n) in (("n", (70, 300)), ("t", (300, 70))):
        A = oracle.phi_matrix(m, n, 2.0, 3).astype(np.float32)
        xl, yl = (n, m) if ta == "n" else (m, n)
        x = oracle.phi_vector(xl, 2.0, 4).astype(np.float32)
        y0 = oracle.phi_vector(yl, 1.0, 5).astype(np.float32)
        if ta == "n":
            out, _ = oracle.sgemm_d(f, "n", "n", m, 1, n, 0.75, A, m, x, n, 1.5, y0, m)
        else:
            out, _ = oracle.sgemm_d(f, "t", "n", n, 1, m, 0.75, A, m, x, m, 1.5, y0, n)
        gold = reference.sgemv_d(ta, m, n, 0.75, A, m, x, 1.5, y0)
        assert f32_bits_equal(out, gold), ta


def test_tau_of_float_data_vs_reference(oracle, reference):
    """The restatement's float tau, (short)ceil((float)log2((double)v)), against the reference's
    log21<float> on every binary exponent (mantissas 0..400 and the top ones) and random floats."""
    import math
    vals = []
    for e in range(-149, 128):
        for j in list(range(0, 400)) + [4095, (1 << 22), (1 << 23) - 1]:
            if e >= -126:
                vals.append(math.ldexp(1.0 + j * 2.0 ** -23, e))
            elif j % (1 << min(-126 - e, 30)) == 0:
                vals.append(math.ldexp(1.0 + j * 2.0 ** -23, e))
    rng = np.random.default_rng(3)
    vals += list(rng.integers(1, 0x7F800000, 20000, dtype=np.int64).astype(np.uint32).view(np.float32).astype(float))
    bad = [v for v in vals if oracle.tau_sd_libm(v) != math.ceil(reference.log21f(v))]
    assert not bad, bad[:5]


@pytest.mark.parametrize("seed", range(8))
def test_quad_gemm_vs_reference(seed, oracle, reference):
    """<__float128, double, double> (binary128 split, FP64 slices, binary128 ordered sum and fmaq): the
    restatement against ozblasRgemm<__float128, double, double>, bit-exact with the split counts.  The
    reference library needs MPLAPACK (not built) to split a one-column panel, so m, n >= 2 here."""
    rng = np.random.default_rng(700 + seed)
    m, n = (int(v) for v in rng.integers(2, 30, 2))
    k = int(rng.integers(1, 300))
    ta, tb = rng.choice(["n", "t"]), rng.choice(["n", "t"])
    fm = int(rng.integers(0, 3))
    nsplit = int(rng.choice([0, 0, 2, 5]))
    phi = float(rng.choice([0.5, 1.0, 2.0, 4.0]))
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix_q(ar, ac, phi, 1)
    B = oracle.phi_matrix_q(br, bc, phi, 2)
    C0 = oracle.phi_matrix_q(m, n, 1.0, 3)
    al, be = oracle.q(1.25), oracle.q(-0.5)
    out, info = oracle.qgemm_d(make_flags(fastMode=fm, nSplitMax=nsplit), ta, tb, m, n, k, al, A, ar, B, br, be, C0,
                               m)
    reference.set_flags(fastMode=fm, nSplitMax=nsplit)
    gold = reference.qgemm_d(ta, tb, m, n, k, al, A, ar, B, br, be, C0, m)
    assert np.array_equal(out, gold), (seed, m, n, k, ta, tb, fm, nsplit, phi)
    inf = reference.info()
    assert [info.nSplitA, info.nSplitB, info.nSplitC] == [inf["nSplitA"], inf["nSplitB"], inf["nSplitC"]]


def test_split_slices_vs_reference(oracle, reference):
    """Slice-level parity of the column-panel and CSR splits."""
    for phi, k, ncol in [(1.0, 100, 7), (4.0, 333, 5), (2.0, 1, 3), (1.0, 64, 1)]:
        X = oracle.phi_matrix(k, ncol, phi, 9)
        reference.set_flags()
        s_ref, sl_ref = reference.split_panel(X)
        s, sl = oracle.split_cols(make_flags(), X)
        assert s == s_ref and bits_equal(sl, sl_ref)
    rowptr, colind = oracle.stencil7(6, 5, 4)
    val = oracle.phi_vector(len(colind), 1.0, 3)
    s_ref, sl_ref = reference.split_sparse(val, rowptr)
    s, sl = oracle.split_csr(make_flags(), val, rowptr)
    assert s == s_ref and bits_equal(sl, sl_ref)


def test_zero_and_tiny_inputs_vs_reference(oracle, reference):
    m, n, k = 9, 7, 40
    A = oracle.phi_matrix(m, k, 1.0, 1)
    A[3, :] = 0.0  # a zero column of A
    A[:, 2] = 0.0  # a zero row
    B = oracle.phi_matrix(k, n, 1.0, 2) * 1e-300
    for sm in (0, 1):
        out, _ = oracle.dgemm(make_flags(sumMode=sm), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
        reference.set_flags(sumMode=sm)
        gold = reference.dgemm("n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
        assert bits_equal(out, gold), first_diff(out, gold)


def test_tau_libm_matches_reference(oracle, reference):
    for v in [1.0, 1.5, 2.0 ** 100 * (1 + 2.0 ** -52), 3.0e-310, 7.0, 2.0 ** -1000]:
        assert oracle.tau_libm(v) == reference.tau(v)


# ---- exact accumulator ----

def test_exact_dot_vs_mpmath(oracle):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 4000
    rng = np.random.default_rng(3)
    for trial in range(20):
        n = int(rng.integers(1, 200))
        x = (rng.random(n) - 0.5) * np.exp(rng.normal(0, 30, n))
        y = (rng.random(n) - 0.5) * np.exp(rng.normal(0, 30, n))
        if trial == 0:
            x[0], y[0] = 1e300, 1e300
            x[1], y[1] = 5e-324, 3.0
        exact = mpmath.fsum(mpmath.mpf(float(a)) * mpmath.mpf(float(b)) for a, b in zip(x, y))
        rn = oracle.exact_dot(x, y)
        assert rn == float(exact) or (np.isinf(rn) and abs(exact) > 1.79e308), (trial, rn, exact)
        if abs(exact) > 1e308:
            continue
        c = float(exact) * (1 + 2.0 ** -50)
        _, rel = oracle.exact_dot_err(x, y, c)
        if exact != 0:
            ref_rel = abs((mpmath.mpf(c) - exact) / exact)
            assert abs(rel - float(ref_rel)) <= 1e-12 * float(ref_rel)


# ---- C ABI ----

def test_c_abi_exports_every_declared_symbol():
    lib = os.path.join(ROOT, "ozblas_b200", "libcuozblas_b200.so")
    assert os.path.exists(lib), "libcuozblas_b200.so is not built"
    hdr = open(os.path.join(ROOT, "include", "cuozblas.h")).read()
    c_part = hdr.split('extern "C" {', 1)[1]
    declared = set(re.findall(r"^\s*(?:int|double|const char \*)\s*(cuozblas\w+)\s*\(", c_part, re.M))
    assert len(declared) >= 15
    syms = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)$", syms, re.M))
    assert declared <= exported, declared - exported
    # the reference's C++ instantiations (include/cuozblas.h:66-80) for drop-in linking
    for mangled in ["_Z14cuozblasCreateP16cuozblasHandle_tm", "_Z15cuozblasDestroyP16cuozblasHandle_t",
                    "_Z13cuozblasRgemmIdddEiP16cuozblasHandle_tccPKiiiT_PKS3_iS5_iS3_PS3_i"[:0] or "cuozblasRgemmIdddE",
                    "cuozblasRdotIdddE", "cuozblasRnrm2IdddE", "cuozblasRgemvIdddE", "cuozblasRaxpyIdE",
                    "cuozblasRcsrmvIddE", "cuozblasRcsrmvSplitAIddE", "cuozblasRcgIddE", "cuozblasRgemmIdaiE"]:
        assert any(mangled in s for s in exported), mangled


def test_python_binding_lists_c_abi():
    import importlib
    # the package refuses to load without its library; the list must match the header
    ozb = importlib.import_module("ozblas_b200")
    hdr = open(os.path.join(ROOT, "include", "cuozblas.h")).read()
    c_part = hdr.split('extern "C" {', 1)[1]
    declared = set(re.findall(r"^\s*(?:int|double|const char \*)\s*(cuozblas\w+)\s*\(", c_part, re.M))
    assert declared == set(ozb.C_ABI_SYMBOLS)
