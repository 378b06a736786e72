"""Plain form at the full configuration sizes vs the reference library's own
outputs (SHA-256 of the FP64 result bytes in tests/golden/full.json and
cg100.json, produced by tests/golden/make_golden.py from oracle/_ref).

Inputs are rebuilt on the host from the same seeds with the reference
harness's generator, copied to the device, and the library is called through
its C ABI.  Bit-exact: the hash of our output must equal the reference's.
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def full():
    with open(os.path.join(GOLD, "full.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def big_handle(ozb):
    h = ozb.Handle(work_bytes=24 << 30)
    yield h
    h.close()


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("sm", [0, 1])
def test_gemm_1024_phi1(sm, full, oracle, big_handle, ozb, cuda):
    """Plain Ozaki DGEMM, m=n=k=1024, phi=1, split until exact."""
    A, B = oracle.phi_matrix(1024, 1024, 1.0, 1), oracle.phi_matrix(1024, 1024, 1.0, 2)
    big_handle.sumMode = sm
    dC = cuda.zeros((1024, 1024), dtype=cuda.float64, device="cuda")
    ozb.dgemm(big_handle, "n", "n", 1024, 1024, 1024, 1.0, dev(cuda, A), 1024, dev(cuda, B), 1024, 0.0, dC, 1024)
    C = dC.cpu().numpy()
    g = full[f"gemm1024_{sm}"]
    assert [big_handle.nSplitA, big_handle.nSplitB, big_handle.nSplitC] == g["nSplit"]
    assert float(C[0, 0]).hex() == g["sample"][0]
    assert sha(C) == g["sha256"]


@pytest.mark.parametrize("sm", [0, 1])
def test_dot_nrm2_2p24(sm, full, oracle, big_handle, ozb, cuda):
    n = 1 << 24
    x, y = oracle.phi_vector(n, 2.0, 1), oracle.phi_vector(n, 2.0, 2)
    big_handle.sumMode = sm
    dx, dy = dev(cuda, x), dev(cuda, y)
    d = ozb.ddot(big_handle, n, dx, dy)
    g = full[f"dot2p24_{sm}"]
    assert float(d).hex() == g["dot"]
    assert [big_handle.nSplitA, big_handle.nSplitB] == g["nSplit"]
    assert float(ozb.dnrm2(big_handle, n, dx)).hex() == g["nrm2"]


@pytest.mark.parametrize("sm", [0, 1])
def test_gemv_8192(sm, full, oracle, big_handle, ozb, cuda):
    A = oracle.phi_matrix(8192, 8192, 1.0, 1)
    x = oracle.phi_vector(8192, 1.0, 2)
    big_handle.sumMode = sm
    dy = cuda.zeros(8192, dtype=cuda.float64, device="cuda")
    ozb.dgemv(big_handle, "n", 8192, 8192, 1.0, dev(cuda, A), 8192, dev(cuda, x), 0.0, dy)
    assert sha(dy.cpu().numpy()) == full[f"gemv8192_{sm}"]["sha256"]


@pytest.mark.parametrize("sm", [0, 1])
def test_csrmv_stencil_128(sm, full, oracle, big_handle, ozb, cuda):
    rowptr, colind = oracle.stencil7(128, 128, 128)
    n = len(rowptr) - 1
    val = oracle.phi_vector(len(colind), 1.0, 1)
    x = oracle.phi_vector(n, 1.0, 2)
    big_handle.sumMode = sm
    dy = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    ozb.dcsrmv(big_handle, "n", n, n, len(val), 1.0, dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr),
               dev(cuda, x), 0.0, dy)
    g = full[f"csrmv128_{sm}"]
    assert [big_handle.nSplitA, big_handle.nSplitB, big_handle.nSplitC] == g["nSplit"]
    assert sha(dy.cpu().numpy()) == g["sha256"]


def test_cg_poisson_100_2000(oracle, big_handle, ozb, cuda):
    """CG, 100^3 Poisson + 0.01 U shift, NearSum, 2000 iterations: residual history bit-identical."""
    with open(os.path.join(GOLD, "cg100.json")) as f:
        g = json.load(f)
    nx = 100
    rowptr, colind = oracle.stencil7(nx, nx, nx)
    n = len(rowptr) - 1
    val = oracle.poisson_shift(nx, nx, nx, 3, rowptr, colind)
    b = oracle.csrmv_fma(val, colind, rowptr, oracle.normal(n, 4))
    big_handle.sumMode = 1
    big_handle.verbose = 1
    it = g["iters"]
    h1 = np.zeros(it + 1)
    h2 = np.zeros(it + 1)
    dx = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    ozb.dcg(big_handle, "n", n, len(val), dev(cuda, val), dev(cuda, colind), dev(cuda, rowptr), dev(cuda, b), dx, it,
            0.0, h1, h2)
    assert big_handle.cg_numiter == g["cg_numiter"]
    assert [float(v).hex() for v in h1[:5]] == g["hist_head"]
    assert sha(h1) == g["hist_sha256"]
    assert sha(dx.cpu().numpy()) == g["x_sha256"]
