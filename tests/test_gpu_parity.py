"""Plain form (FP64 slices) on the GPU vs the CPU oracle: bit-exact.

Every case calls the library through its C ABI (ozblas_b200 -> ctypes ->
libcuozblas_b200.so) with device buffers, and compares all output bits with
the C restatement of the reference CPU path (oracle/ozoracle.c), which is
itself pinned to the reference library by tests/test_oracle.py and the
golden files.  Inputs come from the reference harness's phi generator
(testing/testing_common.cpp:703-717), seeds 1 (A, x) and 2 (B, y).
"""
import numpy as np
import pytest

from oracle.oracle import make_flags
from tests.conftest import bits_equal, first_diff

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


GEMM_CASES = [
    # m, n, k, ta, tb, sumMode, fastMode, alpha, beta, phi
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


@pytest.mark.parametrize("case", GEMM_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-{c[3]}{c[4]}-s{c[5]}f{c[6]}")
def test_dgemm_small(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, sm, fm, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1)
    B = oracle.phi_matrix(br, bc, phi, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    ref, info = oracle.dgemm(make_flags(sumMode=sm, fastMode=fm), ta, tb, m, n, k, alpha, A, ar, B, br, beta, C0, m)
    dA, dB, dC = dev(cuda, A), dev(cuda, B), dev(cuda, C0)
    handle.sumMode, handle.fastMode = sm, fm
    ozb.dgemm(handle, ta, tb, m, n, k, alpha, dA, ar, dB, br, beta, dC, m)
    out = host(dC)
    assert bits_equal(out, ref), first_diff(out, ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


def test_dgemm_run_to_run_identical(oracle, handle, ozb, cuda):
    m = n = k = 256
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    dA, dB = dev(cuda, A), dev(cuda, B)
    outs = []
    for _ in range(3):
        dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
        ozb.dgemm(handle, "n", "n", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m)
        outs.append(host(dC))
    assert bits_equal(outs[0], outs[1]) and bits_equal(outs[0], outs[2])
    ref, _ = oracle.dgemm(make_flags(), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
    assert bits_equal(outs[0], ref), first_diff(outs[0], ref)


def test_phase_timers(oracle, handle, ozb, cuda):
    """The exec-info phase timers (t_SplitA, t_SplitB, t_comp, t_sum) of the plain form are filled,
    as the reference's drivers print them."""
    m = n = k = 256
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
    handle.sumMode = 1
    ozb.dgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    t = [handle.t_SplitA, handle.t_SplitB, handle.t_comp, handle.t_sum]
    assert all(v > 0 for v in t) and sum(t) <= handle.t_total * 1.01, (t, handle.t_total)


@pytest.mark.parametrize("sum_mode", [0, 1])
def test_kernel_span_timer(oracle, handle, ozb, cuda, sum_mode):
    """t_comp holds the device span of the call's kernels on every DOT and GEMV path: positive and no longer
    than the whole call."""
    handle.sumMode = sum_mode
    n = 1 << 16
    x = dev(cuda, oracle.phi_vector(n, 2.0, 1))
    y = dev(cuda, oracle.phi_vector(n, 2.0, 2))
    ozb.ddot(handle, n, x, y)
    assert 0 < handle.t_comp <= handle.t_total * 1.01, (handle.t_comp, handle.t_total)
    m = k = 512
    A = dev(cuda, oracle.phi_matrix(m, k, 1.0, 3))
    xv = dev(cuda, oracle.phi_vector(k, 1.0, 4))
    yv = cuda.zeros(m, dtype=cuda.float64, device="cuda")
    ozb.dgemv(handle, "n", m, k, 1.0, A, m, xv, 0.0, yv)
    assert 0 < handle.t_comp <= handle.t_total * 1.01, (handle.t_comp, handle.t_total)


def test_dgemm_beta0_propagates_nan(oracle, handle, ozb, cuda):
    """C = fma(alpha, t, beta*C) with beta = 0 keeps NaN from C, as the reference does."""
    m = n = k = 8
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    C0 = np.zeros((n, m))
    C0[2, 3] = np.nan
    ref, _ = oracle.dgemm(make_flags(), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, C0, m)
    dC = dev(cuda, C0)
    ozb.dgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    out = host(dC)
    assert np.isnan(out[2, 3]) and bits_equal(out, ref)


@pytest.mark.parametrize("nsplit", [1, 2, 3])
def test_dgemm_truncated_split(nsplit, oracle, handle, ozb, cuda):
    m, n, k = 40, 30, 200
    A = oracle.phi_matrix(m, k, 2.0, 1)
    B = oracle.phi_matrix(k, n, 2.0, 2)
    ref, _ = oracle.dgemm(make_flags(nSplitMax=nsplit), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
    handle.nSplitMax = nsplit
    dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
    ozb.dgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    assert bits_equal(host(dC), ref), first_diff(host(dC), ref)


@pytest.mark.parametrize("n,phi", [(1, 1.0), (7, 1.0), (1000, 2.0), (100003, 2.0), (1 << 20, 2.0)])
@pytest.mark.parametrize("sm", [0, 1])
def test_ddot_dnrm2(n, phi, sm, oracle, handle, ozb, cuda):
    x = oracle.phi_vector(n, phi, 1)
    y = oracle.phi_vector(n, phi, 2)
    handle.sumMode = sm
    d = ozb.ddot(handle, n, dev(cuda, x), dev(cuda, y))
    r, info = oracle.ddot(make_flags(sumMode=sm), x, y)
    assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (d, r)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)
    nr = ozb.dnrm2(handle, n, dev(cuda, x))
    nr_ref, _ = oracle.dnrm2(make_flags(sumMode=sm), x)
    assert np.float64(nr).view(np.int64) == np.float64(nr_ref).view(np.int64), (nr, nr_ref)
    if sm == 1:
        assert d == oracle.exact_dot(x, y)  # NearSum with a complete split = correctly rounded


@pytest.mark.parametrize("m,n,trans,sm,fm", [(50, 70, "n", 0, 0), (50, 70, "t", 1, 0), (300, 257, "n", 1, 0),
                                              (64, 1000, "n", 0, 1), (1, 33, "t", 0, 0)])
def test_dgemv(m, n, trans, sm, fm, oracle, handle, ozb, cuda):
    A = oracle.phi_matrix(m, n, 1.0, 1)
    xl = n if trans == "n" else m
    yl = m if trans == "n" else n
    x = oracle.phi_vector(xl, 1.0, 2)
    y0 = oracle.phi_vector(yl, 1.0, 3)
    ref, info = oracle.dgemv(make_flags(sumMode=sm, fastMode=fm), trans, m, n, 0.75, A, m, x, 0.5, y0)
    handle.sumMode, handle.fastMode = sm, fm
    dy = dev(cuda, y0)
    ozb.dgemv(handle, trans, m, n, 0.75, dev(cuda, A), m, dev(cuda, x), 0.5, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)


def stencil_case(oracle, nx, ny, nz, seed=1):
    rowptr, colind = oracle.stencil7(nx, ny, nz)
    val = oracle.phi_vector(len(colind), 1.0, seed)
    return rowptr, colind, val


@pytest.mark.parametrize("grid", [(4, 3, 2), (12, 10, 9), (32, 32, 32)])
@pytest.mark.parametrize("sm", [0, 1])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (-1.0, 1.0), (0.5, 2.0)])
def test_dcsrmv(grid, sm, ab, oracle, handle, ozb, cuda):
    rowptr, colind, val = stencil_case(oracle, *grid)
    n = len(rowptr) - 1
    x = oracle.phi_vector(n, 1.0, 2)
    y0 = oracle.phi_vector(n, 1.0, 3)
    ref, info = oracle.dcsrmv(make_flags(sumMode=sm), n, n, ab[0], val, colind, rowptr, x, ab[1], y0)
    handle.sumMode = sm
    dy = dev(cuda, y0)
    ozb.dcsrmv(handle, "n", n, n, len(val), ab[0], dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr),
               dev(cuda, x), ab[1], dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


def test_dcsrmv_empty_rows(oracle, handle, ozb, cuda):
    rowptr = np.array([0, 2, 2, 5, 5, 6], dtype=np.int32)
    colind = np.array([0, 3, 1, 2, 4, 0], dtype=np.int32)
    val = oracle.phi_vector(6, 1.0, 5)
    x = oracle.phi_vector(5, 1.0, 6)
    y0 = np.zeros(5)
    ref, _ = oracle.dcsrmv(make_flags(), 5, 5, 1.0, val, colind, rowptr, x, 0.0, y0)
    dy = dev(cuda, y0)
    ozb.dcsrmv(handle, "n", 5, 5, 6, 1.0, dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, x), 0.0, dy)
    assert bits_equal(host(dy), ref)


@pytest.mark.parametrize("sm", [0, 1])
def test_split_a_and_cg(sm, oracle, handle, ozb, cuda):
    nx = ny = nz = 12
    rowptr, colind = oracle.stencil7(nx, ny, nz)
    n = len(rowptr) - 1
    val = oracle.poisson_shift(nx, ny, nz, 3, rowptr, colind)
    b = oracle.csrmv_fma(val, colind, rowptr, oracle.normal(n, 4))
    iters = 60
    xr, hr, info = oracle.dcg(make_flags(sumMode=sm), val, colind, rowptr, b, np.zeros(n), iters, 0.0)
    handle.sumMode = sm
    handle.verbose = 1
    dx = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    h1 = np.zeros(iters + 1)
    h2 = np.zeros(iters + 1)
    it = ozb.dcg(handle, "n", n, len(val), dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, b), dx,
                 iters, 0.0, h1, h2)
    assert it == iters
    assert bits_equal(h1, hr), first_diff(h1, hr)
    assert bits_equal(host(dx), xr), first_diff(host(dx), xr)


@pytest.mark.parametrize("K", [60, 120])
@pytest.mark.parametrize("sm", [0, 1])
def test_cg_deep_rows(K, sm, oracle, handle, ozb, cuda):
    """Columns scaled by 2^[-K, K]: rows need 5 (K=60) or 7 (K=120) levels, so
    the CG's SpMV runs the deep-row kernel (and defers rows beyond it); the
    later, wide CG vectors take the general x path."""
    nx = ny = nz = 8
    rowptr, colind = oracle.stencil7(nx, ny, nz)
    n = len(rowptr) - 1
    val = oracle.poisson_shift(nx, ny, nz, 3, rowptr, colind)
    val = val * 2.0 ** np.random.default_rng(K).integers(-K, K + 1, n)[colind]
    b = oracle.normal(n, 4)
    iters = 4
    xr, hr, info = oracle.dcg(make_flags(sumMode=sm), val, colind, rowptr, b, np.zeros(n), iters, 0.0)
    handle.sumMode = sm
    handle.verbose = 1
    dx = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    h1 = np.zeros(iters + 1)
    h2 = np.zeros(iters + 1)
    ozb.dcg(handle, "n", n, len(val), dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, b), dx,
            iters, 0.0, h1, h2)
    assert bits_equal(h1, hr), first_diff(h1, hr)
    assert bits_equal(host(dx), xr), first_diff(host(dx), xr)


@pytest.mark.parametrize("n", [1, 2, 3, 4097, 100003])
@pytest.mark.parametrize("sm", [0, 1])
def test_ddot_unaligned_and_odd(n, sm, oracle, handle, ozb, cuda):
    """Vectors 8 bytes off a 16-byte boundary take the scalar-load kernels;
    odd lengths leave one element outside the paired stream."""
    x = oracle.phi_vector(n, 2.0, 1)
    y = oracle.phi_vector(n, 2.0, 2)
    handle.sumMode = sm
    r, info = oracle.ddot(make_flags(sumMode=sm), x, y)
    bx = cuda.zeros(n + 1, dtype=cuda.float64, device="cuda")
    by = cuda.zeros(n + 1, dtype=cuda.float64, device="cuda")
    bx[1:] = dev(cuda, x)
    by[1:] = dev(cuda, y)
    for xv, yv in ((bx[1:], by[1:]), (bx[1:], dev(cuda, y)), (dev(cuda, x), dev(cuda, y))):
        d = ozb.ddot(handle, n, xv, yv)
        assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (n, sm, d, r)
        assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)
    nr_ref, _ = oracle.dnrm2(make_flags(sumMode=sm), x)
    for xv in (bx[1:], dev(cuda, x)):
        nr = ozb.dnrm2(handle, n, xv)
        assert np.float64(nr).view(np.int64) == np.float64(nr_ref).view(np.int64), (n, sm, nr, nr_ref)


@pytest.mark.parametrize("n,phi", [((1 << 23) + 12345, 1.0), (5000001, 1.0)])
@pytest.mark.parametrize("sm", [0, 1])
def test_ddot_tensor_core_pass(n, phi, sm, oracle, handle, ozb, cuda):
    """Long vectors (2 and 3 digits per level): with FSum pass 2 runs on the INT8 tensor cores; with NearSum the
    one-pass exact DOT answers and its last block proves the predicted chains from the blocks' witness
    candidates.  The chains of these vectors are the predicted ones, so the fused paths must be the ones that
    answer: two launches (scan, tensor-core pass) with FSum, one with NearSum."""
    x = oracle.phi_vector(n, phi, 1)
    y = oracle.phi_vector(n, phi, 2)
    handle.sumMode = sm
    dx, dy = dev(cuda, x), dev(cuda, y)
    l0 = handle.launch_count()
    d = ozb.ddot(handle, n, dx, dy)
    assert handle.launch_count() - l0 == (2 if sm == 0 else 1)  # no fallback to the general path
    r, info = oracle.ddot(make_flags(sumMode=sm), x, y)
    assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (d, r)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)
    nr = ozb.dnrm2(handle, n, dx)
    nr_ref, _ = oracle.dnrm2(make_flags(sumMode=sm), x)
    assert np.float64(nr).view(np.int64) == np.float64(nr_ref).view(np.int64), (nr, nr_ref)


@pytest.mark.parametrize("case", ["n_at_threshold", "one_element_tail", "zero_block", "same_vector", "nan_inf",
                                  "unaligned", "wide_range"])
def test_ddot_tensor_core_pass_edges(case, oracle, handle, ozb, cuda):
    """Edge cases around the tensor-core pass: its length threshold, a last job holding one element,
    jobs of zeros, x = y, Inf/NaN (the general path answers), a vector 8 bytes off a 16-byte
    boundary (the tree pass answers) and a range too wide for 8 levels."""
    n = (1 << 22) + (1 if case == "one_element_tail" else 0)
    x = oracle.phi_vector(n, 1.0, 5)
    y = oracle.phi_vector(n, 1.0, 6)
    if case == "zero_block":
        x[100000:900000] = 0.0
    if case == "nan_inf":
        x[12345] = np.inf
        y[777] = np.nan
    if case == "wide_range":
        x[::1000] *= 2.0 ** 200
    for sm in (0, 1):
        handle.sumMode = sm
        if case == "unaligned":
            bx = cuda.zeros(n + 1, dtype=cuda.float64, device="cuda")
            bx[1:] = dev(cuda, x)
            dx = bx[1:]
        else:
            dx = dev(cuda, x)
        dy = dx if case == "same_vector" else dev(cuda, y)
        yy = x if case == "same_vector" else y
        d = ozb.ddot(handle, n, dx, dy)
        r, info = oracle.ddot(make_flags(sumMode=sm), x, yy)
        if case == "nan_inf":
            # IEEE 754 leaves the sign and payload of a NaN result open: x86 makes inf - inf a
            # negative NaN and keeps an input NaN's sign, and which one survives depends on the
            # order of the additions.  The result must be a NaN; its bits are not compared.
            assert np.isnan(d) and np.isnan(r), (sm, d, r)
        else:
            assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (case, sm, d, r)
        assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)


def test_ddot_tensor_core_pass_matches_tree(oracle, handle, ozb, cuda, monkeypatch):
    """The INT8 tensor-core pass (vectors of 2^22 elements and more) and the FP64 tree pass give the same
    bits, with 3 and 2 digits per level."""
    for n, phi in (((1 << 22) + 5, 1.0), ((1 << 23) + 3, 0.5), ((1 << 23) + 77, 2.0), ((1 << 24) + 9, 1.0)):
        x = dev(cuda, oracle.phi_vector(n, phi, 3))
        y = dev(cuda, oracle.phi_vector(n, phi, 4))
        for sm in (0, 1):
            handle.sumMode = sm
            monkeypatch.delenv("OZBLAS_DOT_TREE", raising=False)
            handle.read_env()
            a = (ozb.ddot(handle, n, x, y), ozb.dnrm2(handle, n, x), ozb.ddot(handle, n, y, y))
            monkeypatch.setenv("OZBLAS_DOT_TREE", "1")
            handle.read_env()
            b = (ozb.ddot(handle, n, x, y), ozb.dnrm2(handle, n, x), ozb.ddot(handle, n, y, y))
            monkeypatch.delenv("OZBLAS_DOT_TREE", raising=False)
            handle.read_env()
            assert np.array(a).view(np.int64).tolist() == np.array(b).view(np.int64).tolist(), (n, phi, sm, a, b)


def test_invalid_arguments(handle, ozb, cuda):
    x = cuda.zeros(8, dtype=cuda.float64, device="cuda")
    with pytest.raises(ozb.OzblasError) as e:
        ozb.ddot(handle, 8, x, x, incx=2)
    assert e.value.code == 2
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dcsrmv(handle, "t", 1, 1, 0, 1.0, x, x, x, x, 0.0, x)
    assert e.value.code == 2
    handle.splitEpsMode = 2  # Dot2 exists for DOT, NRM2, CSRMV and CG, with fastMode 0
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dgemm(handle, "n", "n", 2, 2, 2, 1.0, x, 2, x, 2, 0.0, x, 2)
    assert e.value.code == 4
    handle.fastMode = 1
    with pytest.raises(ozb.OzblasError) as e:
        ozb.ddot(handle, 8, x, x)
    assert e.value.code == 4


# ---- Dot2 (splitEpsMode 2) ----

@pytest.mark.parametrize("grid", [(4, 3, 2), (12, 10, 9), (30, 20, 25)])
@pytest.mark.parametrize("sm", [0, 1])
def test_dcsrmv_dot2(grid, sm, oracle, handle, ozb, cuda):
    """Dot2 CSRMV is sequential per row in the reference, so it is bit-exact here."""
    rowptr, colind = oracle.stencil7(*grid)
    n = len(rowptr) - 1
    val = oracle.phi_vector(len(colind), 2.0, 1)
    x = oracle.phi_vector(n, 2.0, 2)
    y0 = oracle.phi_vector(n, 1.0, 3)
    handle.sumMode, handle.splitEpsMode = sm, 2
    for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
        ref, info = oracle.dcsrmv(make_flags(sumMode=sm, splitEpsMode=2), n, n, alpha, val, colind, rowptr, x, beta,
                                  y0)
        dy = dev(cuda, y0)
        ozb.dcsrmv(handle, "n", n, n, len(val), alpha, dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr),
                   dev(cuda, x), beta, dy)
        assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
        assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("n,phi", [(1, 1.0), (1000, 2.0), (100003, 1.0), (1 << 20, 2.0)])
@pytest.mark.parametrize("sm", [0, 1])
def test_ddot_dot2(n, phi, sm, oracle, handle, ozb, cuda):
    """Dot2 DOT: the reference's double-double partials meet in OpenMP order, so only its one-thread
    run is reproducible; this library uses a fixed parallel order instead.  Tolerance: the result
    is within one unit in the last place of the one-thread reference (restatement), identical run
    to run, and the split counts agree."""
    x = oracle.phi_vector(n, phi, 1)
    y = oracle.phi_vector(n, phi, 2)
    handle.sumMode, handle.splitEpsMode = sm, 2
    dx, dy = dev(cuda, x), dev(cuda, y)
    d = ozb.ddot(handle, n, dx, dy)
    assert ozb.ddot(handle, n, dx, dy) == d
    r, info = oracle.ddot(make_flags(sumMode=sm, splitEpsMode=2), x, y)
    assert abs(d - r) <= np.spacing(abs(r)), (d, r)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)
    nr = ozb.dnrm2(handle, n, dx)
    nr_ref, _ = oracle.dnrm2(make_flags(sumMode=sm, splitEpsMode=2), x)
    assert abs(nr - nr_ref) <= np.spacing(nr_ref), (nr, nr_ref)


def test_cg_dot2(oracle, handle, ozb, cuda):
    """CG in Dot2 mode (host loop): CSRMV bit-exact, DOT within an ulp, so the residual history
    follows the one-thread reference closely."""
    nx = ny = nz = 10
    rowptr, colind = oracle.stencil7(nx, ny, nz)
    n = len(rowptr) - 1
    val = oracle.poisson_shift(nx, ny, nz, 3, rowptr, colind)
    b = oracle.csrmv_fma(val, colind, rowptr, oracle.normal(n, 4))
    iters = 25
    xr, hr, _ = oracle.dcg(make_flags(sumMode=1, splitEpsMode=2), val, colind, rowptr, b, np.zeros(n), iters, 0.0)
    handle.sumMode, handle.splitEpsMode, handle.verbose = 1, 2, 1
    dx = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    h1 = np.zeros(iters + 1)
    h2 = np.zeros(iters + 1)
    it = ozb.dcg(handle, "n", n, len(val), dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, b), dx,
                 iters, 0.0, h1, h2)
    assert it == iters
    assert np.allclose(h1, hr, rtol=1e-9, atol=0), np.max(np.abs(h1 - hr) / np.abs(hr))
    assert np.allclose(host(dx), xr, rtol=1e-9, atol=1e-12)


# ---- fused DOT / CSRMV: the paths that must hand over to the general algorithm ----

def test_ddot_chain_prediction_fails(oracle, handle, ozb, cuda):
    """A remainder maximum below the predicted binade: the fused DOT must fall back."""
    n = 4096
    x = oracle.phi_vector(n, 1.0, 1) * 2.0 ** -40
    x[0] = 1.0  # the only large entry: after level 0 every remainder is tiny
    y = oracle.phi_vector(n, 1.0, 2)
    for sm in (0, 1):
        handle.sumMode = sm
        d = ozb.ddot(handle, n, dev(cuda, x), dev(cuda, y))
        r, info = oracle.ddot(make_flags(sumMode=sm), x, y)
        assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (sm, d, r)
        assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)


@pytest.mark.parametrize("phi", [6.0, 10.0])
def test_ddot_many_levels(phi, oracle, handle, ozb, cuda):
    """More levels than the fused pass holds (wide exponent range)."""
    n = 20000
    x, y = oracle.phi_vector(n, phi, 1), oracle.phi_vector(n, phi, 2)
    for sm in (0, 1):
        handle.sumMode = sm
        d = ozb.ddot(handle, n, dev(cuda, x), dev(cuda, y))
        r, info = oracle.ddot(make_flags(sumMode=sm), x, y)
        assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (phi, sm, d, r, info.nSplitA)


def _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, alpha, beta, sm, fm=0):
    n = len(rowptr) - 1
    ref, info = oracle.dcsrmv(make_flags(sumMode=sm, fastMode=fm), n, len(x), alpha, val, colind, rowptr, x, beta, y0)
    handle.sumMode, handle.fastMode = sm, fm
    dy = dev(cuda, y0)
    ozb.dcsrmv(handle, "n", n, len(x), len(val), alpha, dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr),
               dev(cuda, x), beta, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("sm", [0, 1])
def test_dcsrmv_long_rows_and_deep_rows(sm, oracle, handle, ozb, cuda):
    """Rows longer than 8 entries and rows needing many levels go to the per-row kernel."""
    rng = np.random.default_rng(5)
    n = 300
    lens = rng.integers(0, 20, n)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    colind = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    val = oracle.phi_vector(len(colind), 1.0, 7)
    for r in range(0, n, 37):  # some rows with a huge in-row exponent range
        lo, hi = rowptr[r], rowptr[r + 1]
        if hi - lo >= 2:
            val[lo] *= 2.0 ** 150
            val[hi - 1] *= 2.0 ** -150
    x = oracle.phi_vector(n, 1.0, 8)
    y0 = oracle.phi_vector(n, 1.0, 9)
    _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 0.5, -2.0, sm)


@pytest.mark.parametrize("sm", [0, 1])
def test_dcsrmv_special_rows(sm, oracle, handle, ozb, cuda):
    """Rows of exact powers of two, zero entries and rows, subnormal entries and a wide in-row range."""
    rowptr, colind, val = stencil_case(oracle, 10, 9, 8)
    n = len(rowptr) - 1
    rng = np.random.default_rng(15)
    for r in range(0, n, 7):
        lo, hi = rowptr[r], rowptr[r + 1]
        kind = (r // 7) % 5
        if kind == 0:
            val[lo:hi] = rng.choice([-1.0, 1.0], hi - lo) * 2.0 ** rng.integers(-3, 4, hi - lo)
        elif kind == 1:
            val[lo:hi] = 0.0
        elif kind == 2:
            val[lo] = 0.0
            val[hi - 1] = -0.0
        elif kind == 3:
            val[lo:hi] *= 2.0 ** -1060
        else:
            val[lo] *= 2.0 ** 40
    x = oracle.phi_vector(n, 1.0, 2)
    y0 = oracle.phi_vector(n, 1.0, 3)
    for beta in (0.0, 1.5):
        _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 1.0, beta, sm)


@pytest.mark.parametrize("sm", [0, 1])
def test_dcsrmv_x_chain_general_path(sm, oracle, handle, ozb, cuda):
    """x whose chain is not the predicted one, and x needing more than 8 levels."""
    rowptr, colind, val = stencil_case(oracle, 10, 9, 8)
    n = len(rowptr) - 1
    y0 = oracle.phi_vector(n, 1.0, 3)
    x = oracle.phi_vector(n, 1.0, 2) * 2.0 ** -40
    x[5] = 1.0
    _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 1.0, 0.0, sm)
    x = oracle.phi_vector(n, 9.0, 2)
    _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 1.0, 0.0, sm)


def test_dcsrmv_fastmode_uses_general_path(oracle, handle, ozb, cuda):
    rowptr, colind, val = stencil_case(oracle, 6, 5, 4)
    n = len(rowptr) - 1
    x = oracle.phi_vector(n, 1.0, 2)
    y0 = np.zeros(n)
    # fastMode = 1 drops only the last level: pair sets agree with the reference's storage
    _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 1.0, 0.0, 0, fm=1)


@pytest.mark.parametrize("sm", [0, 1])
@pytest.mark.parametrize("m,n,k,ta,tb,scale", [(600, 500, 4096, "n", "n", 1.0), (257, 300, 1000, "t", "t", 2.0 ** -900),
                                                (130, 129, 2000, "n", "t", 2.0 ** 700)])
def test_dgemm_tensor_core_pairs_equal_dmma(sm, m, n, k, ta, tb, scale, oracle, handle, ozb, cuda, monkeypatch):
    """The plain form's exact slice-pair products on the INT8 tensor cores (slices cut into int8
    digits, exact INT32 digit products combined exactly in FP64, scaled by 2^(tauA + tauB)) give the
    DMMA kernel's bits under FSum and NearSum, also for data far from 1."""
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, 2.0, 1) * scale
    B = oracle.phi_matrix(br, bc, 1.0, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    handle.sumMode = sm
    outs = []
    for dmma in (False, True):
        if dmma:
            monkeypatch.setenv("OZBLAS_PLAIN_DMMA", "1")
            handle.read_env()
        dC = dev(cuda, C0)
        ozb.dgemm(handle, ta, tb, m, n, k, 1.25, dev(cuda, A), ar, dev(cuda, B), br, -0.5, dC, m)
        outs.append((host(dC), handle.nSplitC))
    assert bits_equal(outs[0][0], outs[1][0]), first_diff(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


@pytest.mark.parametrize("sm", [0, 1])
@pytest.mark.parametrize("m,n,fm,phi,scale", [(1000, 3000, 0, 1.0, 1.0), (777, 513, 1, 2.0, 2.0 ** -1000),
                                               (64, 9000, 0, 4.0, 2.0 ** 900), (33, 1, 0, 1.0, 1.0),
                                               (300, 700, 0, 0.0, 1.0), (96, 200, 0, -1.0, 1.0)])
def test_dgemv_fused_equals_materialised(sm, m, n, fm, phi, scale, oracle, handle, ozb, cuda, monkeypatch):
    """GEMV 'n' with the split and the slice products fused gives the bits of the path that writes
    every slice, in both sum modes: the two-read path on predicted tau chains, the path with one read
    of A per level, and the materialised one.  phi = 0 builds rows 1 + 2^-45 s (s = +-1), whose
    remainders after the first level fall far below the predicted chain, so the two-read path has
    to detect the wrong prediction and take the level passes."""
    if phi == 0.0:
        rng = np.random.default_rng(5)
        A = 1.0 + 2.0 ** -45 * rng.choice([-1.0, 1.0], size=(m, n))
        x = oracle.phi_vector(n, 1.0, 2)
    elif phi < 0.0:  # a zero row and an infinite x entry: 0 * Inf makes NaN on every path
        A = oracle.phi_matrix(m, n, 1.0, 1)
        A[:, 7] = 0.0  # row 7 of the column-major m x n matrix (array rows are columns)
        x = oracle.phi_vector(n, 1.0, 2)
        x[n // 2] = np.inf
    else:
        A = oracle.phi_matrix(m, n, phi, 1) * scale
        x = oracle.phi_vector(n, phi, 2)
    y0 = oracle.phi_vector(m, 1.0, 3)
    handle.sumMode, handle.fastMode = sm, fm
    outs = []
    for env in (None, "OZBLAS_GEMV_LEVELS", "OZBLAS_GEMV_SPLIT"):
        if env:
            monkeypatch.setenv(env, "1")
        dy = dev(cuda, y0)
        ozb.dgemv(handle, "n", m, n, 0.75, dev(cuda, A), m, dev(cuda, x), 0.5, dy)
        outs.append((host(dy), (handle.nSplitA, handle.nSplitB, handle.nSplitC)))
    for o in outs[1:]:
        if phi < 0.0:  # IEEE leaves the sign of a NaN open
            assert np.array_equal(np.isnan(outs[0][0]), np.isnan(o[0])) and np.isnan(o[0][7])
            assert bits_equal(np.nan_to_num(outs[0][0]), np.nan_to_num(o[0]))
        else:
            assert bits_equal(outs[0][0], o[0]), first_diff(outs[0][0], o[0])
        assert outs[0][1] == o[1]
    if phi < 0.0:
        return
    if m * n <= 4_000_000:
        ref, info = oracle.dgemv(make_flags(sumMode=sm, fastMode=fm), "n", m, n, 0.75, A, m, x, 0.5, y0)
        assert bits_equal(outs[0][0], ref), first_diff(outs[0][0], ref)


@pytest.mark.parametrize("nsplit", [2, 3])
@pytest.mark.parametrize("m,n", [(200, 300), (64, 4096)])
def test_dgemv_truncated_split(nsplit, m, n, oracle, handle, ozb, cuda):
    """GEMV 'n' with the slice count capped below what the split needs (nSplitMax): the fused paths
    keep the first levels of each row's chain, as the reference's split does."""
    A = oracle.phi_matrix(m, n, 2.0, 1)
    x = oracle.phi_vector(n, 2.0, 2)
    y0 = oracle.phi_vector(m, 1.0, 3)
    ref, info = oracle.dgemv(make_flags(nSplitMax=nsplit), "n", m, n, 1.0, A, m, x, 0.25, y0)
    handle.nSplitMax = nsplit
    dy = dev(cuda, y0)
    ozb.dgemv(handle, "n", m, n, 1.0, dev(cuda, A), m, dev(cuda, x), 0.25, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)


# One-column op(B) stored as a 1 x k row (tb = 't', ldb > 1) and a one-row
# op(A) of a 1 x 1 product stored with lda > 1 (ta = 'n'): the operand's
# elements are strided, the slots between them hold NaN so a contiguous read
# would show.  The oracle reads the same strided storage.
STRIDED_CASES = [
    # m, n, k, ta, tb, lda_extra, ldb, sumMode
    (37, 1, 300, "n", "t", 0, 5, 0),
    (37, 1, 300, "t", "t", 0, 3, 1),
    (1, 1, 257, "n", "n", 3, None, 0),
    (1, 1, 257, "n", "t", 2, 4, 1),
    (1, 1, 64, "t", "t", 0, 2, 0),
]


def _strided_operands(oracle, m, n, k, ta, tb, lda_extra, ldb, phi=1.0):
    if ta == "n":
        lda = m + lda_extra
        A = np.full(lda * k, np.nan)
        A.reshape(k, lda)[:, :m] = oracle.phi_matrix(m, k, phi, 1)[:, :m]
    else:
        lda = k
        A = oracle.phi_matrix(k, m, phi, 1).ravel()
    if tb == "t":
        B = np.full(ldb * k, np.nan)
        B.reshape(k, ldb)[:, 0] = oracle.phi_vector(k, phi, 2)
    else:
        ldb = k
        B = oracle.phi_vector(k, phi, 2).copy()
    return A, lda, B, ldb


@pytest.mark.parametrize("case", STRIDED_CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}{c[4]}-s{c[7]}")
def test_dgemm_strided_vector_operands(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, lda_extra, ldb, sm = case
    A, lda, B, ldb = _strided_operands(oracle, m, n, k, ta, tb, lda_extra, ldb)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    ref, info = oracle.dgemm(make_flags(sumMode=sm), ta, tb, m, n, k, 1.0, A, lda, B, ldb, 0.5, C0, m)
    assert np.all(np.isfinite(ref))
    handle.sumMode = sm
    dC = dev(cuda, C0)
    ozb.dgemm(handle, ta, tb, m, n, k, 1.0, dev(cuda, A), lda, dev(cuda, B), ldb, 0.5, dC, m)
    out = host(dC)
    assert bits_equal(out, ref), first_diff(out, ref)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)


def test_daxpy_public_entry(oracle, handle, ozb, cuda):
    """cuozblasDaxpy: y = fma(alpha, x, y) elementwise (src/cuda/cuozblas_axpy.cu:5-16, reproMode 1), bit for bit;
    incx/incy other than 1 are rejected with INVALID_VALUE (the reference's stride-1 kernel)."""
    n = 20011
    x = oracle.phi_vector(n, 2.0, 1)
    y = oracle.phi_vector(n, 2.0, 2)
    alpha = -1.2345678901234567
    dy = dev(cuda, y)
    ozb.daxpy(handle, n, alpha, dev(cuda, x), dy)
    out = host(dy)
    from fractions import Fraction
    fa = Fraction(alpha)
    ref = np.array([float(fa * Fraction(a) + Fraction(b)) for a, b in zip(x.tolist(), y.tolist())])  # one rounding
    assert bits_equal(out, ref), first_diff(out, ref)
    ozb.daxpy(handle, 0, alpha, dev(cuda, x), dy)  # n = 0: nothing changes
    assert bits_equal(host(dy), ref)
    for incx, incy in ((2, 1), (1, 2), (0, 1), (-1, 1)):
        with pytest.raises(ozb.OzblasError) as e:
            ozb.daxpy(handle, 8, alpha, dev(cuda, x), dy, incx=incx, incy=incy)
        assert e.value.code == 2


# ---- the one-pass NearSum DOT (exact bins, certified rounding, proven counts) ----

ONE_PASS_CASES = [
    # name, n, builder(oracle, n) -> (x, y)
    ("phi1", 1 << 20, lambda o, n: (o.phi_vector(n, 1.0, 1), o.phi_vector(n, 1.0, 2))),
    ("phi4_wide", 300001, lambda o, n: (o.phi_vector(n, 4.0, 1), o.phi_vector(n, 4.0, 2))),
    ("odd_tiny", 7, lambda o, n: (o.phi_vector(n, 2.0, 1), o.phi_vector(n, 2.0, 2))),
    ("cancel", 100000, lambda o, n: (np.concatenate([o.phi_vector(n // 2, 1.0, 1)] * 2),
                                      np.concatenate([o.phi_vector(n // 2, 1.0, 2), -o.phi_vector(n // 2, 1.0, 2)]))),
    ("zeros_and_scale", 65536, lambda o, n: (np.where(np.arange(n) % 3 == 0, 0.0, o.phi_vector(n, 2.0, 1) * 2.0 ** 300),
                                             o.phi_vector(n, 2.0, 2) * 2.0 ** -350)),
    ("huge", 4096, lambda o, n: (o.phi_vector(n, 1.0, 1) * 2.0 ** 500, o.phi_vector(n, 1.0, 2) * 2.0 ** 510)),
    ("tiny", 4096, lambda o, n: (o.phi_vector(n, 1.0, 1) * 2.0 ** -500, o.phi_vector(n, 1.0, 2) * 2.0 ** -480)),
]


@pytest.mark.parametrize("case", ONE_PASS_CASES, ids=lambda c: c[0])
def test_ddot_nearsum_one_pass(case, oracle, handle, ozb, cuda, monkeypatch):
    """NearSum DOT and NRM2: the one-pass path (one or two launches when it answers) gives the oracle's bits and exec-info
    counts, equal to the two-pass DOT's; wide ranges, cancellation, zeros, and products beyond the bins' range
    (which hand the call to the two-pass DOT) included."""
    name, n, build = case
    x, y = build(oracle, n)
    x, y = np.ascontiguousarray(x), np.ascontiguousarray(y)
    dx, dy = dev(cuda, x), dev(cuda, y)
    handle.sumMode = 1
    l0 = handle.launch_count()
    d = ozb.ddot(handle, n, dx, dy)
    launches = handle.launch_count() - l0
    r, info = oracle.ddot(make_flags(sumMode=1), x, y)
    assert np.float64(d).view(np.int64) == np.float64(r).view(np.int64), (name, d, r)
    assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)
    nr = ozb.dnrm2(handle, n, dx)
    nr_ref, _ = oracle.dnrm2(make_flags(sumMode=1), x)
    assert np.float64(nr).view(np.int64) == np.float64(nr_ref).view(np.int64), (name, nr, nr_ref)
    monkeypatch.setenv("OZBLAS_DOT_TWO_PASS", "1")
    handle.read_env()
    d2 = ozb.ddot(handle, n, dx, dy)
    monkeypatch.delenv("OZBLAS_DOT_TWO_PASS")
    handle.read_env()
    assert np.float64(d2).view(np.int64) == np.float64(d).view(np.int64)
    if name in ("phi1", "odd_tiny"):
        # answered by the one-pass kernels: the streaming kernel alone when its last block proves the chains
        # from the witness candidates, with the proof kernel otherwise (or for unaligned vectors)
        assert launches <= 2, launches
    # "cancel" sums to exactly zero while the bins hold the products' lowest bits only up to a bound: the
    # rounding of a sum within that bound of zero is not certified, so the two-pass DOT answers (same bits)


@pytest.mark.parametrize("phi", [1.0, 4.0])
def test_dcsrmv_nearsum_rows_equal_slices(phi, oracle, handle, ozb, cuda, monkeypatch):
    """NearSum CSRMV: the correctly rounded exact row dots give the bits of the slice-pair path (and of the
    oracle), with rows that the kernel must defer (longer than 8, deep splits) mixed in."""
    g = 24
    rowptr, colind = oracle.stencil7(g, g, g)
    m = len(rowptr) - 1
    val = oracle.phi_vector(len(colind), phi, 3)
    val[::97] *= 2.0 ** -600  # rows spanning many levels
    x = oracle.phi_vector(m, phi, 4)
    y0 = oracle.phi_vector(m, 1.0, 5)
    _csr_run(oracle, handle, ozb, cuda, rowptr, colind, val, x, y0, 1.5, -0.5, 1)
    a = (handle.nSplitA, handle.nSplitB, handle.nSplitC)
    dy = dev(cuda, y0)
    monkeypatch.setenv("OZBLAS_CSR_SLICES", "1")
    handle.read_env()
    ozb.dcsrmv(handle, "n", m, m, len(val), 1.5, dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, x),
               -0.5, dy)
    monkeypatch.delenv("OZBLAS_CSR_SLICES")
    handle.read_env()
    ref, _ = oracle.dcsrmv(make_flags(sumMode=1), m, m, 1.5, val, colind, rowptr, x, -0.5, y0)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == a


@pytest.mark.parametrize("m,n,phi", [(300, 1000, 1.0), (1024, 8192, 2.0), (77, 513, 4.0)])
def test_dgemv_nearsum_rows_equal_slices(m, n, phi, oracle, handle, ozb, cuda, monkeypatch):
    """NearSum GEMV 'n': the correctly rounded exact row dots give the oracle's bits and exec-info counts, and the
    bits of the slice path; rows spanning many levels (which hand the call back to the slice path) included."""
    A = oracle.phi_matrix(m, n, phi, 1)
    x = oracle.phi_vector(n, phi, 2)
    y0 = oracle.phi_vector(m, 1.0, 3)
    if phi == 4.0:
        A[5, 3] *= 2.0 ** -700  # a deep row: its split needs more levels than the cap allows
    ref, info = oracle.dgemv(make_flags(sumMode=1), "n", m, n, 0.75, A, m, x, -1.5, y0)
    handle.sumMode = 1
    dy = dev(cuda, y0)
    ozb.dgemv(handle, "n", m, n, 0.75, dev(cuda, A), m, dev(cuda, x), -1.5, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)
    monkeypatch.setenv("OZBLAS_GEMV_SLICES", "1")
    handle.read_env()
    dy2 = dev(cuda, y0)
    ozb.dgemv(handle, "n", m, n, 0.75, dev(cuda, A), m, dev(cuda, x), -1.5, dy2)
    monkeypatch.delenv("OZBLAS_GEMV_SLICES")
    handle.read_env()
    assert bits_equal(host(dy2), host(dy))


def test_dgemv_nearsum_rows_steep_chain(oracle, handle, ozb, cuda):
    """NearSum GEMV 'n' where the row with the largest predicted split count splits in fewer levels (its second
    level already takes the tiny element): the rows' correctly rounded dots are written and the exec-info count
    comes from every row's own split; both equal the oracle's."""
    m, n = 300, 64
    A = oracle.phi_matrix(m, n, 1.0, 11)
    A[7, :] = 0.0
    A[7, 0], A[7, 1] = 1.0, 2.0 ** -100
    x = oracle.phi_vector(n, 1.0, 12)
    y0 = oracle.phi_vector(m, 1.0, 13)
    ref, info = oracle.dgemv(make_flags(sumMode=1), "n", m, n, 0.75, A, m, x, -1.5, y0)
    handle.sumMode = 1
    dy = dev(cuda, y0)
    ozb.dgemv(handle, "n", m, n, 0.75, dev(cuda, A), m, dev(cuda, x), -1.5, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)
