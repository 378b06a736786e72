"""Shared fixtures.

Markers: ``gpu`` tests need a CUDA device (they call the library through its
C ABI); everything else runs on the CPU.  The oracle (oracle/) is the checker
only: tests compare the library's results against it, never route through it.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size configuration")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Restatement

    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference library oracle/_ref not built (only the restatement and golden files pin parity)")
    r = Reference(work_bytes=int(24e9))
    yield r
    r.close()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def ozb(cuda):
    import ozblas_b200

    return ozblas_b200


@pytest.fixture()
def handle(ozb):
    h = ozb.Handle(work_bytes=8 << 30)
    yield h
    h.close()


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def first_diff(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    b = np.ascontiguousarray(b, dtype=np.float64).ravel()
    d = np.nonzero(a.view(np.int64) != b.view(np.int64))[0]
    if len(d) == 0:
        return "identical"
    i = d[0]
    return f"{len(d)} of {a.size} differ; first at {i}: {a[i]!r} vs {b[i]!r}"
