"""The integer rules the GPU split uses, pinned against glibc on the host.

tau = (short)ceil(log2(max)) and rho = ceil(53 - (53 - log2 dim)/2) fix the
bits of every slice (src/cpu/ozblas_split.cpp:19-34,145).  The library
evaluates both without libm (ozb_rules.cuh); its exported host entry points
run the same code the kernels run.
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
    L.cuozblasRuleTau.argtypes = [C.c_double]
    L.cuozblasRuleTau.restype = C.c_int
    L.cuozblasRuleRho.argtypes = [C.c_int32, C.c_int32]
    L.cuozblasRuleRho.restype = C.c_int
    return L


def test_tau_every_exponent_near_binade_start(lib, oracle):
    """For every binary exponent, the mantissas where glibc rounds log2 down onto e."""
    bad = []
    for e in range(-1074, 1024):
        for j in list(range(0, 400)) + [1000, 4095, (1 << 51), (1 << 52) - 1]:
            if e >= -1022:
                v = math.ldexp(1.0 + j * 2.0 ** -52, e)
            else:
                sh = -1022 - e
                if j % (1 << min(sh, 62)):
                    continue
                v = math.ldexp(1.0 + j * 2.0 ** -52, e)
            if v == 0.0 or math.isinf(v):
                continue
            t_ref = oracle.tau_libm(v)
            t = lib.cuozblasRuleTau(v)
            if t != t_ref:
                bad.append((e, j, v, t, t_ref))
    assert not bad, bad[:10]


def test_tau_random_doubles(lib, oracle):
    rng = np.random.default_rng(7)
    bits = rng.integers(1, 0x7FF0000000000000, size=200000, dtype=np.int64)
    vals = bits.view(np.float64)
    bad = [v for v in vals if lib.cuozblasRuleTau(float(v)) != oracle.tau_libm(float(v))]
    assert not bad, bad[:5]


def test_tau_subnormals(lib, oracle):
    for j in list(range(1, 5000)) + [(1 << 52) - 1, (1 << 51) + 1, 1 << 40]:
        v = float(np.array([j], dtype=np.int64).view(np.float64)[0])
        assert lib.cuozblasRuleTau(v) == oracle.tau_libm(v), (j, v)


@pytest.mark.parametrize("mode", [0, 9, 2])
def test_rho_rule(lib, oracle, mode):
    dims = list(range(1, 70000)) + [2 ** p + d for p in range(16, 31) for d in (-1, 0, 1)]
    bad = [(d, lib.cuozblasRuleRho(d, mode), oracle.rho(d, mode)) for d in dims
           if lib.cuozblasRuleRho(d, mode) != oracle.rho(d, mode)]
    assert not bad, bad[:10]


def test_tau_of_float_data_sweep(lib, oracle):
    """The library's integer float tau rule (the device code, exported as cuozblasRuleTauF32) against
    (short)ceil((float)log2((double)v)) on every 61st positive finite float bit pattern, plus every
    exponent's first 400 mantissas through the per-value entry point."""
    import ctypes
    addr = ctypes.cast(lib.cuozblasRuleTauF32, ctypes.c_void_p).value
    bad, first = oracle.tau_sd_sweep(addr, 61)
    assert bad == 0, (bad, hex(first))
    lib.cuozblasRuleTauF32.argtypes = [ctypes.c_float]
    lib.cuozblasRuleTauF32.restype = ctypes.c_int
    mism = []
    for e in range(-149, 128):
        for j in range(0, 400):
            if e < -126 and j % (1 << min(-126 - e, 30)):
                continue
            v = math.ldexp(1.0 + j * 2.0 ** -23, e)
            if lib.cuozblasRuleTauF32(v) != oracle.tau_sd_libm(v):
                mism.append((e, j))
    assert not mism, mism[:10]


def _qrule(lib):
    import ctypes
    lib.cuozblasRuleQ128.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
    lib.cuozblasRuleQ128.restype = ctypes.c_int
    return ctypes.cast(lib.cuozblasRuleQ128, ctypes.c_void_p).value


@pytest.mark.parametrize("op,name", [(0, "add"), (1, "mul"), (2, "fma"), (3, "tau"), (4, "split")])
def test_software_binary128(op, name, lib, oracle):
    """The library's binary128 (q128.cuh, the code the quad-form kernels run) against gcc's
    __float128 and libquadmath's fmaq on 200,000 random operands per operation: random and close
    exponents (cancellation), short significands (ties to even), signed zeros and subnormals.
    tau is compared with the restatement's ceil((double)log2q(v)), the split with the reference's
    (x + sigma) - sigma in binary128."""
    addr = _qrule(lib)
    for seed in (op + 1, op + 101):
        bad, first = oracle.q128_check(addr, op, 100000, seed=seed)
        assert bad == 0, (name, bad, [hex(int(v)) for v in first])


def _q_bits(e, j):
    be = e + 16383
    hi = (be << 48) | (j >> 64)
    return np.array([j & ((1 << 64) - 1), hi], dtype=np.uint64)


def test_tau_of_binary128_every_exponent(lib, oracle, reference):
    """The quad tau rule (threshold table) against the reference's own expression on every normal
    binary128 exponent, at the last mantissa that keeps tau = e and the first that gives e + 1, and
    on random subnormals."""
    import ctypes
    _qrule(lib)
    out = ctypes.c_int(0)

    def lib_tau(v):
        lib.cuozblasRuleQ128(3, v.ctypes.data, None, None, ctypes.byref(out))
        return out.value

    bad = []
    for e in range(-16382, 16384):
        for j in (0, 1, (1 << 112) - 1):
            v = _q_bits(e, j)
            if lib_tau(v) != reference.tau_q(v):
                bad.append((e, j))
        # the switch point: tau(j) == e for j <= T, e + 1 above
        lo, hi = 0, (1 << 112) - 1
        if e % 97 == 0:  # bisection on a sample of exponents, every binade class included
            while hi - lo > 1:
                mid = (lo + hi) // 2
                if reference.tau_q(_q_bits(e, mid)) == e:
                    lo = mid
                else:
                    hi = mid
            for j in (lo, hi):
                if lib_tau(_q_bits(e, j)) != reference.tau_q(_q_bits(e, j)):
                    bad.append((e, j))
    rng = np.random.default_rng(5)
    for _ in range(2000):
        j = int(rng.integers(1, 1 << 62)) << int(rng.integers(0, 50))
        j &= (1 << 112) - 1
        if j == 0:
            continue
        v = np.array([j & ((1 << 64) - 1), j >> 64], dtype=np.uint64)  # subnormal
        if lib_tau(v) != reference.tau_q(v):
            bad.append(("sub", j))
    assert not bad, bad[:10]


def test_scale2_matches_ldexp(lib):
    """scale2 (the scaling the mixed forms add in their ordered sums, in integer arithmetic so that
    nothing can be fused with the addition) = ldexp, correctly rounded, on integer-valued,
    float-valued and general doubles across the normal, subnormal and overflow ranges (numpy's
    ldexp is the C one)."""
    import ctypes
    lib.cuozblasRuleScale2.argtypes = [ctypes.c_double, ctypes.c_int32]
    lib.cuozblasRuleScale2.restype = ctypes.c_double
    rng = np.random.default_rng(9)
    vals = list(rng.integers(-(1 << 31), 1 << 31, 3000).astype(float))
    vals += list(rng.standard_normal(3000).astype(np.float32).astype(float) * np.exp2(rng.integers(-140, 120, 3000)))
    vals += list(rng.standard_normal(3000) * np.exp2(rng.integers(-1070, 1020, 3000)))
    vals += [0.0, -0.0, 1.0, -1.0, 5e-324, -5e-324, 2.0 ** -1022, 1.7976931348623157e308, float("inf")]
    bad = []
    for v in vals:
        for e in (int(rng.integers(-2200, 2200)), int(rng.integers(-1100, -1000)), int(rng.integers(-60, 60)), -1074,
                  -1075, 1023, 2000):
            with np.errstate(over="ignore", under="ignore"):
                want = float(np.ldexp(np.float64(v), e))
            got = lib.cuozblasRuleScale2(v, e)
            if np.float64(got).view(np.int64) != np.float64(want).view(np.int64):
                bad.append((v, e, got, want))
    assert not bad, bad[:5]
