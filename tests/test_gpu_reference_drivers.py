"""The reference's own test drivers run on this library.

oracle/Makefile (target `drivers`) compiles the reference's testing/testing_level3.cpp,
testing_level2.cpp and testing_level1b.cpp — unmodified, with MPLAPACK off — against this
library's include/cuozblas.h and libcuozblas_b200.so.  They call the reference's C++ API
(cuozblasCreate, cuozblasRgemm<double,double,double>, ...), allocate their own device buffers
with cudaMallocPitch and check the result against a double-precision CBLAS product.  A driver
that links, runs and reports a small error shows that a program written for the reference
switches to this library without source changes.  The CSRMV and CG drivers need BeBOP (absent)
and are not built.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRV = os.path.join(ROOT, "oracle", "_ref", "drivers")

CASES = [
    ("testing_cuozblas_dgemm", ["--mnk=256", "--phi=1"]),
    ("testing_cuozblas_dgemm", ["--mnk=300", "--transa=t", "--transb=n"]),
    ("testing_cuozblas_dgemv", ["--mnk=512"]),
    ("testing_cuozblas_dgemv", ["--mnk=333", "--transa=t"]),
    ("testing_cuozblas_ddot", ["--mnk=100000"]),
]


def result_line(text):
    """The driver's data line: three size columns (GEMM "M N K", GEMV "M N --", DOT "-- N --"),
    err(rlt.max), num-err, then the handle's exec-info columns."""
    rows = [l.split() for l in text.splitlines() if l and not l.startswith("#")]
    rows = [r for r in rows if len(r) >= 5 and (r[0].isdigit() or r[0] == "--") and r[1].isdigit()]
    assert rows, text[-2000:]
    return rows[-1]


@pytest.mark.parametrize("exe,args", CASES, ids=lambda v: v if isinstance(v, str) else " ".join(v))
@pytest.mark.parametrize("summode", [0, 1])
def test_reference_driver_runs_on_this_library(exe, args, summode):
    path = os.path.join(DRV, exe)
    if not os.path.exists(path):
        pytest.skip("reference drivers not built (oracle/Makefile target drivers needs the reference sources)")
    cmd = [path, "--mode=c", "--repromode=1", f"--summode={summode}", "--nodisp=1"] + args
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (cmd, r.stdout[-2000:], r.stderr[-2000:])
    assert "error" not in r.stderr.lower(), r.stderr[-2000:]
    row = result_line(r.stdout)
    err = float(row[3])
    assert "Nan/Inf" not in r.stdout
    # against a double-precision CBLAS product: the Ozaki result is (near) exact, so the
    # difference is CBLAS's own rounding error, which cancellation in the drivers' "erange"
    # inputs magnifies (2e-12 at 256^3); a wrong result would be off by far more
    assert err < 1e-8, row
    # exec-info columns of the handle: split counts (#sA, #sB) and the number of products
    nums = [float(v) for v in row[5:] if v.replace(".", "", 1).replace("e-", "", 1).replace("e+", "", 1).isdigit()]
    assert len(nums) >= 9 and nums[6] >= 1 and nums[7] >= 1, row
