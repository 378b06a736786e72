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
