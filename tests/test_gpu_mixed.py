"""Mixed and quad I/O forms on the GPU vs the CPU oracle: bit-exact.

<double, float, float>: FP64 data, FP32 slices (scalbn(slice, -tau) with tau
per line and level), exact FP32 slice products and the scaled FSum
(src/cpu/ozblas_gemm.cpp with TYPE2 = TYPE3 = float, src/cpu/ozblas_sum.cpp:382-432),
through cuozblasDSgemm / DSgemv / DSdot / DSnrm2.

<float, double, double>: float data split in float arithmetic, FP64 slices,
exact FP64 slice products, each rounded to float, scaled and summed in float
(TYPE1 = float), through cuozblasSDgemm / SDgemv / SDdot / SDnrm2.

<__float128, double, double>: binary128 data (16-byte values, held here as
uint64 pairs) split in binary128, FP64 slices, exact FP64 products, the
ordered sum and fmaq in binary128, through cuozblasQgemm / Qgemv / Qdot /
Qnrm2 (the library's software binary128, q128.cuh).

The oracle's restatements of these forms are pinned to the reference library's
ozblasRgemm/Rgemv/Rdot/Rnrm2 instantiations by tests/test_oracle.py.
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


CASES = [
    # m, n, k, ta, tb, fastMode, nSplitMax, alpha, beta, phi
    (1, 2, 1, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (2, 3, 7, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "t", "n", 1, 0, 1.0, 0.0, 1.0),
    (7, 9, 130, "n", "t", 0, 0, -0.5, 2.0, 1.0),
    (20, 20, 64, "t", "t", 2, 0, 1.0, 1.0, 2.0),
    (130, 260, 300, "n", "n", 0, 0, 1.5, -1.0, 2.0),
    (129, 127, 33, "t", "t", 0, 3, 1.0, 0.0, 4.0),
    (64, 64, 1, "n", "n", 0, 0, 1.0, 0.0, 0.5),
    (256, 200, 600, "n", "t", 0, 0, 1.0, 0.5, 1.0),
    (40, 300, 2000, "t", "n", 1, 0, 1.0, 0.0, 1.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-{c[3]}{c[4]}-f{c[5]}s{c[6]}")
def test_dsgemm(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, fm, ns, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1)
    B = oracle.phi_matrix(br, bc, phi, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    ref, info = oracle.dgemm_f32(make_flags(fastMode=fm, nSplitMax=ns), ta, tb, m, n, k, alpha, A, ar, B, br, beta,
                                 C0, m)
    handle.fastMode, handle.nSplitMax = fm, ns
    dC = dev(cuda, C0)
    ozb.dsgemm(handle, ta, tb, m, n, k, alpha, dev(cuda, A), ar, dev(cuda, B), br, beta, dC, m)
    out = host(dC)
    assert bits_equal(out, ref), first_diff(out, ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


DS_TC_CASES = [
    # k > 1024: every FP32 slice is an int8 times a power of two, and the products run on tcgen05 kind::i8
    (130, 100, 1500, "n", "n", 0, 0, 1.5, -1.0, 2.0),
    (129, 70, 3000, "t", "t", 2, 0, 1.0, 0.5, 1.0),
    (64, 200, 1025, "n", "t", 0, 3, -0.75, 0.0, 4.0),
    (1, 300, 2048, "t", "n", 0, 0, 1.0, 0.0, 1.0),
]


@pytest.mark.parametrize("case", DS_TC_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-{c[3]}{c[4]}-f{c[5]}")
def test_dsgemm_tensor_core_path(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, fm, ns, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1)
    B = oracle.phi_matrix(br, bc, phi, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    ref, info = oracle.dgemm_f32(make_flags(fastMode=fm, nSplitMax=ns), ta, tb, m, n, k, alpha, A, ar, B, br, beta,
                                 C0, m)
    handle.fastMode, handle.nSplitMax = fm, ns
    dC = dev(cuda, C0)
    ozb.dsgemm(handle, ta, tb, m, n, k, alpha, dev(cuda, A), ar, dev(cuda, B), br, beta, dC, m)
    out = host(dC)
    assert bits_equal(out, ref), first_diff(out, ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("scale", [1.0, 2.0 ** -1040, 2.0 ** 950])
def test_dsgemm_tensor_core_equals_simt(scale, oracle, handle, ozb, cuda, monkeypatch):
    """At a size the oracle cannot afford, the INT8 tensor-core path gives the FP32 SIMT path's bits
    (both are the reference's exact slice products and ordered sum), also with the scaling in the
    subnormal range and near overflow."""
    m, n, k = 700, 600, 4096
    A = oracle.phi_matrix(m, k, 1.0, 1) * scale
    B = oracle.phi_matrix(k, n, 1.0, 2)
    dA, dB = dev(cuda, A), dev(cuda, B)
    outs = []
    for simt in (False, True):
        if simt:
            monkeypatch.setenv("OZBLAS_DS_SIMT", "1")
            handle.read_env()
        dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
        ozb.dsgemm(handle, "n", "n", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m)
        outs.append((host(dC), handle.nSplitC))
    assert bits_equal(outs[0][0], outs[1][0]), first_diff(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


def test_dsgemm_run_to_run_identical(oracle, handle, ozb, cuda):
    m, n, k = 300, 200, 256
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    dA, dB = dev(cuda, A), dev(cuda, B)
    outs = []
    for _ in range(3):
        dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
        ozb.dsgemm(handle, "n", "n", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m)
        outs.append(host(dC))
    assert bits_equal(outs[0], outs[1]) and bits_equal(outs[0], outs[2])
    ref, _ = oracle.dgemm_f32(make_flags(), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
    assert bits_equal(outs[0], ref), first_diff(outs[0], ref)


@pytest.mark.parametrize("n,phi", [(1, 1.0), (7, 1.0), (1000, 2.0), (100003, 2.0), (1 << 20, 1.0)])
def test_dsdot_dsnrm2(n, phi, oracle, handle, ozb, cuda):
    x = oracle.phi_vector(n, phi, 1)
    y = oracle.phi_vector(n, phi, 2)
    d = ozb.dsdot(handle, n, dev(cuda, x), dev(cuda, y))
    r, info = oracle.dgemm_f32(make_flags(), "t", "n", 1, 1, n, 1.0, x, n, y, n, 0.0, np.zeros(1), 1)
    assert bits_equal(np.array([d]), r), (d, r[0])
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, 1.0)
    nr = ozb.dsnrm2(handle, n, dev(cuda, x))
    r2, _ = oracle.dgemm_f32(make_flags(), "t", "n", 1, 1, n, 1.0, x, n, x, n, 0.0, np.zeros(1), 1)
    assert bits_equal(np.array([nr]), np.sqrt(r2)), (nr, np.sqrt(r2[0]))


@pytest.mark.parametrize("m,n,trans,fm", [(50, 70, "n", 0), (50, 70, "t", 0), (300, 257, "n", 1), (1, 33, "t", 0),
                                           (700, 2000, "t", 2)])
def test_dsgemv(m, n, trans, fm, oracle, handle, ozb, cuda):
    A = oracle.phi_matrix(m, n, 2.0, 1)
    xl, yl = (n, m) if trans == "n" else (m, n)
    x = oracle.phi_vector(xl, 2.0, 2)
    y0 = oracle.phi_vector(yl, 1.0, 3)
    f = make_flags(fastMode=fm)
    if trans == "n":
        ref, info = oracle.dgemm_f32(f, "n", "n", m, 1, n, 0.75, A, m, x, n, 0.5, y0, m)
    else:
        ref, info = oracle.dgemm_f32(f, "t", "n", n, 1, m, 0.75, A, m, x, m, 0.5, y0, n)
    handle.fastMode = fm
    dy = dev(cuda, y0)
    ozb.dsgemv(handle, trans, m, n, 0.75, dev(cuda, A), m, dev(cuda, x), 0.5, dy)
    assert bits_equal(host(dy), ref), first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("scale", [2.0 ** -1060, 2.0 ** -540, 2.0 ** 900])
def test_mixed_extreme_magnitudes(scale, oracle, handle, ozb, cuda):
    """Products scaled into the subnormal range (scalbn rounds once there) and near overflow."""
    m, n, k = 45, 37, 200
    A = oracle.phi_matrix(m, k, 1.0, 1) * scale
    B = oracle.phi_matrix(k, n, 1.0, 2)
    ref, _ = oracle.dgemm_f32(make_flags(), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m)), m)
    dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
    ozb.dsgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    assert bits_equal(host(dC), ref), first_diff(host(dC), ref)
    x = oracle.phi_vector(5000, 1.0, 4) * scale
    y = oracle.phi_vector(5000, 1.0, 5)
    d = ozb.dsdot(handle, 5000, dev(cuda, x), dev(cuda, y))
    r, _ = oracle.dgemm_f32(make_flags(), "t", "n", 1, 1, 5000, 1.0, x, 5000, y, 5000, 0.0, np.zeros(1), 1)
    assert bits_equal(np.array([d]), r), (d, r[0])


def test_mixed_zero_and_special_lines(oracle, handle, ozb, cuda):
    """Zero rows / columns (tau of a zero line) and an all-zero operand."""
    m, n, k = 70, 50, 96
    A = oracle.phi_matrix(m, k, 2.0, 1)
    B = oracle.phi_matrix(k, n, 2.0, 2)
    A.reshape(k, m)[:, 5] = 0.0    # row 5 of A
    B.reshape(n, k)[7, :] = 0.0    # column 7 of B
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    for a in (A, np.zeros_like(A)):
        ref, info = oracle.dgemm_f32(make_flags(), "n", "n", m, n, k, 1.0, a, m, B, k, -1.0, C0, m)
        dC = dev(cuda, C0)
        ozb.dsgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, a), m, dev(cuda, B), k, -1.0, dC, m)
        assert bits_equal(host(dC), ref), first_diff(host(dC), ref)
        assert (handle.nSplitA, handle.nSplitB) == (info.nSplitA, info.nSplitB)


def test_mixed_unsupported_flags(handle, ozb, cuda):
    """NearSum (sumMode 1) and Dot2 do not exist for mixed types in the reference."""
    x = cuda.zeros(8, dtype=cuda.float64, device="cuda")
    handle.sumMode = 1
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dsgemm(handle, "n", "n", 2, 2, 2, 1.0, x, 2, x, 2, 0.0, x, 2)
    assert e.value.code == 4
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dsdot(handle, 8, x, x)
    assert e.value.code == 4
    handle.sumMode, handle.splitEpsMode = 0, 2
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dsdot(handle, 8, x, x)
    assert e.value.code == 4
    handle.splitEpsMode = 0
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dsdot(handle, 8, x, x, incx=2)
    assert e.value.code == 2


# ---- <float, double, double>: float data, FP64 slices, float-scaled sum ----

def f32_bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.int32), b.view(np.int32))


def f32_first_diff(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32).ravel()
    b = np.ascontiguousarray(b, dtype=np.float32).ravel()
    d = np.nonzero(a.view(np.int32) != b.view(np.int32))[0]
    return None if len(d) == 0 else (int(d[0]), len(d), float(a[d[0]]), float(b[d[0]]))


SD_CASES = [
    # m, n, k, ta, tb, fastMode, nSplitMax, alpha, beta, phi
    (1, 2, 1, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (2, 3, 7, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "t", "n", 1, 0, 1.0, 0.0, 4.0),
    (7, 9, 130, "n", "t", 0, 0, -0.5, 2.0, 2.0),
    (20, 20, 64, "t", "t", 2, 0, 1.0, 1.0, 2.0),
    (130, 260, 300, "n", "n", 0, 0, 1.5, -1.0, 4.0),
    (129, 127, 33, "t", "t", 0, 2, 1.0, 0.0, 4.0),
    (64, 64, 1, "n", "n", 0, 0, 1.0, 0.0, 0.5),
    (300, 200, 2000, "n", "t", 0, 0, 1.0, 0.5, 1.0),
]


@pytest.mark.parametrize("case", SD_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-{c[3]}{c[4]}-f{c[5]}s{c[6]}")
def test_sdgemm(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, fm, ns, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1).astype(np.float32)
    B = oracle.phi_matrix(br, bc, phi, 2).astype(np.float32)
    C0 = oracle.phi_matrix(m, n, 1.0, 3).astype(np.float32)
    ref, info = oracle.sgemm_d(make_flags(fastMode=fm, nSplitMax=ns), ta, tb, m, n, k, alpha, A, ar, B, br, beta,
                               C0, m)
    handle.fastMode, handle.nSplitMax = fm, ns
    dC = dev(cuda, C0)
    ozb.sdgemm(handle, ta, tb, m, n, k, alpha, dev(cuda, A), ar, dev(cuda, B), br, beta, dC, m)
    out = host(dC)
    assert f32_bits_equal(out, ref), f32_first_diff(out, ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("n,phi,scale", [(1, 1.0, 1.0), (7, 1.0, 1.0), (1000, 2.0, 1.0), (100003, 2.0, 1.0),
                                         (1 << 20, 1.0, 1.0), (5000, 4.0, 2.0 ** -120), (5000, 1.0, 2.0 ** 60),
                                         (3000, 1.0, 2.0 ** -140)])
def test_sddot_sdnrm2(n, phi, scale, oracle, handle, ozb, cuda):
    x = (oracle.phi_vector(n, phi, 1) * scale).astype(np.float32)
    y = oracle.phi_vector(n, phi, 2).astype(np.float32)
    d = ozb.sddot(handle, n, dev(cuda, x), dev(cuda, y))
    r, info = oracle.sgemm_d(make_flags(), "t", "n", 1, 1, n, 1.0, x, n, y, n, 0.0, np.zeros(1, np.float32), 1)
    assert f32_bits_equal(np.array([d], np.float32), r), (d, r[0])
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, 1.0)
    nr = ozb.sdnrm2(handle, n, dev(cuda, x))
    r2, _ = oracle.sgemm_d(make_flags(), "t", "n", 1, 1, n, 1.0, x, n, x, n, 0.0, np.zeros(1, np.float32), 1)
    assert f32_bits_equal(np.array([nr], np.float32), np.array([np.sqrt(np.float64(r2[0]))], np.float32))


@pytest.mark.parametrize("m,n,trans,fm", [(50, 70, "n", 0), (50, 70, "t", 0), (300, 257, "n", 1), (1, 33, "t", 0),
                                           (700, 2000, "t", 2)])
def test_sdgemv(m, n, trans, fm, oracle, handle, ozb, cuda):
    A = oracle.phi_matrix(m, n, 2.0, 1).astype(np.float32)
    xl, yl = (n, m) if trans == "n" else (m, n)
    x = oracle.phi_vector(xl, 2.0, 2).astype(np.float32)
    y0 = oracle.phi_vector(yl, 1.0, 3).astype(np.float32)
    f = make_flags(fastMode=fm)
    if trans == "n":
        ref, info = oracle.sgemm_d(f, "n", "n", m, 1, n, 0.75, A, m, x, n, 0.5, y0, m)
    else:
        ref, info = oracle.sgemm_d(f, "t", "n", n, 1, m, 0.75, A, m, x, m, 0.5, y0, n)
    handle.fastMode = fm
    dy = dev(cuda, y0)
    ozb.sdgemv(handle, trans, m, n, 0.75, dev(cuda, A), m, dev(cuda, x), 0.5, dy)
    assert f32_bits_equal(host(dy), ref), f32_first_diff(host(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("scale", [2.0 ** -140, 2.0 ** -70, 2.0 ** 62])
def test_sd_extreme_magnitudes(scale, oracle, handle, ozb, cuda):
    """Products scaled into float's subnormal range (the float scaling rounds there) and to its top."""
    m, n, k = 45, 37, 200
    A = (oracle.phi_matrix(m, k, 1.0, 1) * scale).astype(np.float32)
    B = oracle.phi_matrix(k, n, 1.0, 2).astype(np.float32)
    ref, _ = oracle.sgemm_d(make_flags(), "n", "n", m, n, k, 1.0, A, m, B, k, 0.0, np.zeros((n, m), np.float32), m)
    dC = cuda.zeros((n, m), dtype=cuda.float32, device="cuda")
    ozb.sdgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    assert f32_bits_equal(host(dC), ref), f32_first_diff(host(dC), ref)


def test_sd_unsupported_flags(handle, ozb, cuda):
    x = cuda.zeros(8, dtype=cuda.float32, device="cuda")
    handle.sumMode = 1
    with pytest.raises(ozb.OzblasError) as e:
        ozb.sdgemm(handle, "n", "n", 2, 2, 2, 1.0, x, 2, x, 2, 0.0, x, 2)
    assert e.value.code == 4
    handle.sumMode, handle.splitEpsMode = 0, 2
    with pytest.raises(ozb.OzblasError) as e:
        ozb.sddot(handle, 8, x, x)
    assert e.value.code == 4


# ---- <__float128, double, double>: binary128 data (uint64 pairs), FP64 slices, binary128 sum ----

def qdev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


def qhost(t):
    return t.cpu().numpy().view(np.uint64)


Q_CASES = [
    # m, n, k, ta, tb, fastMode, nSplitMax, alpha, beta, phi
    (2, 2, 1, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (1, 5, 40, "t", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "n", "n", 0, 0, 1.0, 0.0, 1.0),
    (33, 17, 100, "t", "n", 1, 0, 1.25, -0.5, 4.0),
    (7, 9, 130, "n", "t", 0, 0, -0.5, 2.0, 2.0),
    (20, 20, 64, "t", "t", 2, 0, 1.0, 1.0, 2.0),
    (130, 150, 300, "n", "n", 0, 0, 1.5, -1.0, 1.0),
    (65, 70, 33, "t", "t", 0, 2, 1.0, 0.0, 4.0),
]


@pytest.mark.parametrize("case", Q_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-{c[3]}{c[4]}-f{c[5]}s{c[6]}")
def test_qgemm(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, fm, ns, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix_q(ar, ac, phi, 1)
    B = oracle.phi_matrix_q(br, bc, phi, 2)
    C0 = oracle.phi_matrix_q(m, n, 1.0, 3)
    al, be = oracle.q(alpha), oracle.q(beta)
    ref, info = oracle.qgemm_d(make_flags(fastMode=fm, nSplitMax=ns), ta, tb, m, n, k, al, A, ar, B, br, be, C0, m)
    handle.fastMode, handle.nSplitMax = fm, ns
    dC = qdev(cuda, C0)
    ozb.qgemm(handle, ta, tb, m, n, k, al, qdev(cuda, A), ar, qdev(cuda, B), br, be, dC, m)
    out = qhost(dC)
    assert np.array_equal(out, ref), np.argwhere(np.any(out != ref, axis=-1))[:3]
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("n,phi", [(1, 1.0), (7, 1.0), (1000, 2.0), (100003, 1.0)])
def test_qdot_qnrm2(n, phi, oracle, handle, ozb, cuda):
    import math
    x = oracle.phi_vector_q(n, phi, 1)
    y = oracle.phi_vector_q(n, phi, 2)
    d = ozb.qdot(handle, n, qdev(cuda, x), qdev(cuda, y))
    one, zero = oracle.q(1.0), oracle.q(0.0)
    r, info = oracle.qgemm_d(make_flags(), "t", "n", 1, 1, n, one, x, n, y, n, zero, np.zeros((1, 2), np.uint64), 1)
    assert tuple(int(v) for v in r[0]) == tuple(int(v) for v in d)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, 1.0)
    nr = ozb.qnrm2(handle, n, qdev(cuda, x))
    r2, _ = oracle.qgemm_d(make_flags(), "t", "n", 1, 1, n, one, x, n, x, n, zero, np.zeros((1, 2), np.uint64), 1)
    want = oracle.q(math.sqrt(oracle.q_to_double(r2[0])))  # the reference's double sqrt of the binary128 dot
    assert tuple(int(v) for v in want) == tuple(int(v) for v in nr)


@pytest.mark.parametrize("m,n,trans,fm", [(50, 70, "n", 0), (50, 70, "t", 0), (300, 257, "n", 1), (1, 33, "t", 0)])
def test_qgemv(m, n, trans, fm, oracle, handle, ozb, cuda):
    A = oracle.phi_matrix_q(m, n, 2.0, 1)
    xl, yl = (n, m) if trans == "n" else (m, n)
    x = oracle.phi_vector_q(xl, 2.0, 2)
    y0 = oracle.phi_vector_q(yl, 1.0, 3)
    al, be = oracle.q(0.75), oracle.q(0.5)
    f = make_flags(fastMode=fm)
    if trans == "n":
        ref, info = oracle.qgemm_d(f, "n", "n", m, 1, n, al, A, m, x, n, be, y0, m)
    else:
        ref, info = oracle.qgemm_d(f, "t", "n", n, 1, m, al, A, m, x, m, be, y0, n)
    handle.fastMode = fm
    dy = qdev(cuda, y0)
    ozb.qgemv(handle, trans, m, n, al, qdev(cuda, A), m, qdev(cuda, x), be, dy)
    assert np.array_equal(qhost(dy), ref)
    assert (handle.nSplitA, handle.nSplitB, handle.nSplitC) == (info.nSplitA, info.nSplitB, info.nSplitC)


@pytest.mark.parametrize("e", [-16350, -8000, 9000, 16200])
def test_q_extreme_magnitudes(e, oracle, handle, ozb, cuda):
    """Data scaled toward the ends of binary128's range: products land in its subnormal range (the
    binary128 scaling rounds there) or near overflow."""
    m, n, k = 20, 17, 90
    A = oracle.q_scale(oracle.phi_matrix_q(m, k, 1.0, 1), e)
    B = oracle.phi_matrix_q(k, n, 1.0, 2)
    one, zero = oracle.q(1.0), oracle.q(0.0)
    ref, _ = oracle.qgemm_d(make_flags(), "n", "n", m, n, k, one, A, m, B, k, zero, np.zeros((n, m, 2), np.uint64), m)
    dC = qdev(cuda, np.zeros((n, m, 2), np.uint64))
    ozb.qgemm(handle, "n", "n", m, n, k, one, qdev(cuda, A), m, qdev(cuda, B), k, zero, dC, m)
    assert np.array_equal(qhost(dC), ref)


def test_q_unsupported_flags(oracle, handle, ozb, cuda):
    x = qdev(cuda, np.zeros((8, 2), np.uint64))
    handle.sumMode = 1
    with pytest.raises(ozb.OzblasError) as e:
        ozb.qdot(handle, 8, x, x)
    assert e.value.code == 4


@pytest.mark.parametrize("m,n,k,ta,tb", [(300, 260, 1000, "n", "n"), (129, 400, 4096, "t", "n"), (257, 130, 60, "n", "t")])
def test_qgemm_tensor_core_equals_dmma(m, n, k, ta, tb, oracle, handle, ozb, cuda, monkeypatch):
    """The quad form's pair products on the INT8 tensor cores (slices cut into int8 digits, exact
    INT32 digit products combined exactly in FP64) give the DMMA kernel's bits, beta C included."""
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix_q(ar, ac, 2.0, 1)
    B = oracle.phi_matrix_q(br, bc, 1.0, 2)
    C0 = oracle.phi_matrix_q(m, n, 1.0, 3)
    al, be = oracle.q(1.25), oracle.q(-0.5)
    outs = []
    for dmma in (False, True):
        if dmma:
            monkeypatch.setenv("OZBLAS_Q_DMMA", "1")
            handle.read_env()
        dC = qdev(cuda, C0)
        ozb.qgemm(handle, ta, tb, m, n, k, al, qdev(cuda, A), ar, qdev(cuda, B), br, be, dC, m)
        outs.append((qhost(dC), handle.nSplitC))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


@pytest.mark.parametrize("m,n,k,ta,tb,scale", [(300, 260, 1000, "n", "n", 1.0), (129, 400, 4096, "t", "t", 1.0),
                                                (257, 130, 200, "n", "t", 2.0 ** -120), (200, 200, 3000, "n", "n", 2.0 ** 60)])
def test_sdgemm_tensor_core_equals_dmma(m, n, k, ta, tb, scale, oracle, handle, ozb, cuda, monkeypatch):
    """The <float,double,double> pair products on the INT8 tensor cores (k > 128: FP64 slices cut into
    int8 digits) give the DMMA kernel's bits, with products scaled near the ends of float's range."""
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = (oracle.phi_matrix(ar, ac, 2.0, 1) * scale).astype(np.float32)
    B = oracle.phi_matrix(br, bc, 1.0, 2).astype(np.float32)
    C0 = oracle.phi_matrix(m, n, 1.0, 3).astype(np.float32)
    outs = []
    for dmma in (False, True):
        if dmma:
            monkeypatch.setenv("OZBLAS_SD_DMMA", "1")
            handle.read_env()
        dC = dev(cuda, C0)
        ozb.sdgemm(handle, ta, tb, m, n, k, 1.25, dev(cuda, A), ar, dev(cuda, B), br, -0.5, dC, m)
        outs.append((host(dC), handle.nSplitC))
    assert f32_bits_equal(outs[0][0], outs[1][0]), f32_first_diff(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


# Strided vector operands in the mixed and quad forms: a one-column op(B)
# stored as a 1 x k row (tb = 't', ldb > 1) and the one-row op(A) of a 1 x 1
# product with lda > 1; the slots between the elements hold NaN, the oracle
# reads the same storage.
MIXED_STRIDED = [
    # m, n, k, ta, tb, lda, ldb
    (37, 1, 300, "n", "t", 37, 5),
    (1, 1, 257, "n", "n", 3, 257),
    (1, 1, 257, "n", "t", 2, 4),
]


def _strided_f64(oracle, m, k, ta, tb, lda, ldb):
    if ta == "n":
        A = np.full(lda * k, np.nan)
        A.reshape(k, lda)[:, :m] = oracle.phi_matrix(m, k, 1.0, 1)[:, :m]
    else:
        A = oracle.phi_matrix(k, m, 1.0, 1).ravel()
    if tb == "t":
        B = np.full(ldb * k, np.nan)
        B.reshape(k, ldb)[:, 0] = oracle.phi_vector(k, 1.0, 2)
    else:
        B = oracle.phi_vector(k, 1.0, 2).copy()
    return A, B


@pytest.mark.parametrize("case", MIXED_STRIDED, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}{c[4]}")
def test_mixed_strided_vector_operands(case, oracle, handle, ozb, cuda):
    m, n, k, ta, tb, lda, ldb = case
    A, B = _strided_f64(oracle, m, k, ta, tb, lda, ldb)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    # <double, float, float>
    ref, _ = oracle.dgemm_f32(make_flags(), ta, tb, m, n, k, 1.0, A, lda, B, ldb, 0.5, C0, m)
    dC = dev(cuda, C0)
    ozb.dsgemm(handle, ta, tb, m, n, k, 1.0, dev(cuda, A), lda, dev(cuda, B), ldb, 0.5, dC, m)
    out = host(dC)
    assert np.all(np.isfinite(ref)) and bits_equal(out, ref), first_diff(out, ref)
    # <float, double, double>
    Af, Bf, Cf = A.astype(np.float32), B.astype(np.float32), C0.astype(np.float32)
    ref, _ = oracle.sgemm_d(make_flags(), ta, tb, m, n, k, 1.0, Af, lda, Bf, ldb, 0.5, Cf, m)
    dC = dev(cuda, Cf)
    ozb.sdgemm(handle, ta, tb, m, n, k, 1.0, dev(cuda, Af), lda, dev(cuda, Bf), ldb, 0.5, dC, m)
    out = host(dC)
    assert np.all(np.isfinite(ref)) and f32_bits_equal(out, ref), f32_first_diff(out, ref)
    # <__float128, double, double>: NaN slots become binary128 NaNs
    qnan = oracle.q(float("nan"))
    Aq = np.tile(qnan, (A.size, 1))
    Bq = np.tile(qnan, (B.size, 1))
    fa, fb = np.isfinite(A), np.isfinite(B)
    Aq[fa] = np.array([oracle.q(v) for v in A[fa]])
    Bq[fb] = np.array([oracle.q(v) for v in B[fb]])
    Cq = np.array([oracle.q(v) for v in C0.ravel()])
    al, be = oracle.q(1.0), oracle.q(0.5)
    ref, _ = oracle.qgemm_d(make_flags(), ta, tb, m, n, k, al, Aq, lda, Bq, ldb, be, Cq, m)
    dC = qdev(cuda, Cq)
    ozb.qgemm(handle, ta, tb, m, n, k, al, qdev(cuda, Aq), lda, qdev(cuda, Bq), ldb, be, dC, m)
    out = qhost(dC)
    assert np.array_equal(out, ref)
