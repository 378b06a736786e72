"""The allocation-free INT8 DGEMM entry point (cuozblasDgemmI8Static).

Callers that cannot allocate device memory (hosts whose device memory is
budgeted once at start-up, or whose own allocator owns the whole device) use
this entry point: it runs the INT8 precision form on a 64 MiB scratch array
compiled into the library.  This file is collected last so that a run which
stops at the first failure has already run every other test; it passes alone
in a fresh process and after the rest of the suite.

Each case calls the new entry point twice in a row through the C ABI and
compares both results with the handle-based cuozblasDgemmI8 on the same
inputs.  Both run the same kernels with the same schedule, so the tolerance
is the one the INT8 tests use for repeatability: bit-identical.
"""
import numpy as np
import pytest

from tests.conftest import bits_equal, first_diff

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


CASES = [
    # m, n, k, ta, tb, fastMode, nSplitMax, alpha, beta, phi
    (300, 200, 500, "n", "n", 0, 0, 1.5, -0.5, 1.0),
    (130, 257, 129, "t", "t", 1, 0, 1.0, 0.0, 2.0),
    (64, 96, 1000, "n", "t", 1, 6, -1.0, 2.0, 0.5),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}{c[4]}-f{c[5]}s{c[6]}")
def test_static_matches_handle_path_twice(case, oracle, ozb, cuda):
    m, n, k, ta, tb, fast, nsplit, alpha, beta, phi = case
    ar, ac = (m, k) if ta == "n" else (k, m)
    br, bc = (k, n) if tb == "n" else (n, k)
    A = oracle.phi_matrix(ar, ac, phi, 1)
    B = oracle.phi_matrix(br, bc, phi, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    dA, dB = dev(cuda, A), dev(cuda, B)

    h = ozb.Handle(work_bytes=2 << 30)
    h.fastMode = fast
    h.nSplitMax = nsplit
    dC = dev(cuda, C0)
    ozb.dgemm_i8(h, ta, tb, m, n, k, alpha, dA, ar, dB, br, beta, dC, m)
    expect = dC.cpu().numpy()
    h.close()

    for call in range(2):
        dS = dev(cuda, C0)
        ozb.dgemm_i8_static(ta, tb, m, n, k, alpha, dA, ar, dB, br, beta, dS, m, nSplitMax=nsplit, fastMode=fast)
        got = dS.cpu().numpy()
        assert bits_equal(got, expect), (call, first_diff(got, expect))


def test_static_rejects_problems_beyond_its_scratch(ozb, cuda):
    n = 4096  # the transposed copy of A alone needs 128 MiB
    A = cuda.zeros((n, n), dtype=cuda.float64, device="cuda")
    with pytest.raises(ozb.OzblasError) as e:
        ozb.dgemm_i8_static("n", "n", n, n, n, 1.0, A, n, A, n, 0.0, A, n)
    assert e.value.code == 3  # CUOZBLAS_STATUS_WORKSPACE
