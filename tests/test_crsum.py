"""The certified fast path of the correctly rounded sum against NearSum.

NearSum (src/cpu/ozblas_sum.cpp:10-112) returns the double nearest to the
exact sum of its terms; the library first tries a cascade of TwoSums with an
error certificate (crsum.h) and runs NearSum only when the certificate fails.
Whenever the certificate holds, its result must equal the oracle's NearSum and
the oracle's exact rounding; it must also hold for almost every ordinary term
set, or the fast path buys nothing.  The exported host entry point runs the
same code the kernels run.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ozblas_b200", "libcuozblas_b200.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail("libcuozblas_b200.so is not built")
    L = C.CDLL(LIB)
    L.cuozblasRuleCrSum.argtypes = [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.cuozblasRuleCrSum.restype = C.c_int
    return L


def crsum(lib, v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = C.c_double(0.0)
    ok = lib.cuozblasRuleCrSum(len(v), v.ctypes.data_as(C.POINTER(C.c_double)), C.byref(out))
    return ok, out.value


def same(a, b):
    return np.float64(a).view(np.int64) == np.float64(b).view(np.int64)


def check(lib, oracle, v):
    """Returns whether the certificate held; fails if it held on a wrong value."""
    ok, r = crsum(lib, v)
    if ok:
        ns = oracle.nearsum(list(v))
        ex = oracle.exact_sum(v)
        assert same(r, ns), (list(v), r, ns)
        assert same(r, ex), (list(v), r, ex)
    return ok


def test_random_magnitudes(lib, oracle):
    """Random signs, exponents over 120 binades and lengths 1..48: all agree; almost all certified."""
    rng = np.random.default_rng(11)
    certified = 0
    trials = 4000
    for t in range(trials):
        n = int(rng.integers(1, 49))
        spread = int(rng.integers(0, 120))
        v = rng.uniform(-1, 1, n) * np.exp2(rng.integers(-spread // 2 - 1, spread // 2 + 1, n))
        certified += check(lib, oracle, v)
    assert certified >= trials * 0.99, certified


def test_slice_pair_like_terms(lib, oracle):
    """Terms like the pair products of a split: geometric levels, exact on their grids."""
    rng = np.random.default_rng(12)
    certified = 0
    trials = 3000
    for _ in range(trials):
        na, nb = int(rng.integers(1, 7)), int(rng.integers(1, 9))
        d = int(rng.integers(14, 27))
        terms = []
        for ik in range(na + nb - 1):
            for ia in range(max(0, ik - nb + 1), min(ik, na - 1) + 1):
                k = int(rng.integers(-(1 << 40), 1 << 40))
                terms.append(math.ldexp(float(k), -d * ik - 40))
        certified += check(lib, oracle, np.array(terms))
    assert certified >= trials * 0.98, certified


def test_midpoints_and_near_midpoints(lib, oracle):
    """Exact ties are never certified; near ties either are (correctly) or fall back."""
    cases = [
        [1.0, 2.0 ** -53],
        [1.0 + 2.0 ** -52, 2.0 ** -53],
        [1.0, 2.0 ** -53, 2.0 ** -200],
        [1.0, 2.0 ** -53, -(2.0 ** -200)],
        [1.0, -(2.0 ** -54)],
        [1.0, -(2.0 ** -54), 2.0 ** -300],
        [-1.0, -(2.0 ** -53)],
        [3.0, 2.0 ** -52, 2.0 ** -52],
        [2.0 ** 600, 2.0 ** 547, 2.0 ** 100, -(2.0 ** 100)],
    ]
    for v in cases:
        check(lib, oracle, np.array(v))
    # generated: r + ulp/2 (and the power-of-two side) nudged by 2^-k ulp
    rng = np.random.default_rng(14)
    for _ in range(300):
        r = float(rng.uniform(1, 2)) * 2.0 ** int(rng.integers(-200, 200))
        if rng.integers(0, 4) == 0:
            r = 2.0 ** int(rng.integers(-200, 200))
        r = -r if rng.integers(0, 2) else r
        u = math.ulp(r)
        for half in (u / 2, -u / 4, -u / 2):
            for k in (1, 2, 10, 30, 52, 53, 60, 100):
                for sgn in (1.0, -1.0):
                    check(lib, oracle, np.array([r, half, sgn * u * 2.0 ** -k]))
    ok, _ = crsum(lib, np.array([1.0, 2.0 ** -53]))
    assert not ok
    ok, _ = crsum(lib, np.array([1.0 + 2.0 ** -52, 2.0 ** -53]))
    assert not ok


def test_fallback_cases(lib, oracle):
    """Zero sums, tiny sums, subnormal error terms, overflow and NaN are left to NearSum."""
    for v in ([], [0.0], [1.0, -1.0], [-0.0, 0.0], [5e-324, 5e-324], [1e-300, -1e-300, 1e-310],
              [1.0, 5e-324], [1.7e308, 1.7e308], [float("inf"), 1.0], [float("nan")], [2.0 ** -970, 2.0 ** -1000]):
        ok, _ = crsum(lib, np.array(v, dtype=np.float64))
        assert not ok, v


def test_cancellation(lib, oracle):
    """Heavy cancellation: a large pair that cancels exactly plus ordinary terms."""
    rng = np.random.default_rng(13)
    for _ in range(1000):
        big = float(rng.uniform(1, 2)) * 2.0 ** int(rng.integers(30, 200))
        rest = list(rng.uniform(-1, 1, int(rng.integers(1, 10))))
        v = np.array([big] + rest + [-big])
        rng.shuffle(v)
        check(lib, oracle, v)
