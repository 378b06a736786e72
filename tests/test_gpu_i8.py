"""INT8 precision form (tcgen05) vs the exact oracle.

There is no reference implementation of this form, so its oracle is the exact
dot product (oracle/ozoracle.c, an exact fixed-point accumulator, pinned
against mpmath in tests/test_oracle.py).  Tolerances are written per test:
with a complete split and the full pair set every product is exact and only
the final FP64 level sum rounds, so the componentwise error stays within
2 units of 2^-53 relative; the plain FP64-slice form is run on the same
inputs as the comparison point.
"""
import numpy as np
import pytest

from tests.conftest import bits_equal

pytestmark = pytest.mark.gpu

U = 2.0 ** -53


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def errors(oracle, A, B, C, m, n, k, rows=None, cols=None):
    """max |c - exact| / |exact| over the sampled entries (A m x k, B k x n column-major)."""
    rows = range(m) if rows is None else rows
    cols = range(n) if cols is None else cols
    At = np.ascontiguousarray(A.reshape(k, m).T) if A.ndim == 2 else A  # A stored (k, m): row j = column j
    worst = 0.0
    for j in cols:
        b = np.ascontiguousarray(B[j, :k])
        for i in rows:
            _, rel = oracle.exact_dot_err(np.ascontiguousarray(At[i]), b, float(C[j, i]), n=k)
            worst = max(worst, rel)
    return worst


def run_i8(ozb, handle, cuda, A, B, m, n, k, ta="n", tb="n", nsplit=0, fast=0, alpha=1.0, beta=0.0, C0=None):
    handle.nSplitMax = nsplit
    handle.fastMode = fast
    dC = dev(cuda, C0) if C0 is not None else cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
    lda = A.shape[1]
    ldb = B.shape[1]
    ozb.dgemm_i8(handle, ta, tb, m, n, k, alpha, dev(cuda, A), lda, dev(cuda, B), ldb, beta, dC, m)
    return dC.cpu().numpy()


@pytest.mark.parametrize("m,n,k,phi", [(128, 128, 128, 1.0), (200, 130, 300, 1.0), (1, 1, 1, 1.0),
                                       (64, 256, 1000, 0.5), (256, 256, 512, 2.0), (300, 77, 129, 4.0)])
def test_i8_full_pairs_accuracy(m, n, k, phi, oracle, handle, ozb, cuda):
    A = oracle.phi_matrix(m, k, phi, 1)  # shape (k, m): column-major m x k
    B = oracle.phi_matrix(k, n, phi, 2)  # shape (n, k)
    C = run_i8(ozb, handle, cuda, A, B, m, n, k)
    rows = range(m) if m <= 128 else np.linspace(0, m - 1, 64).astype(int)
    cols = range(n) if n <= 128 else np.linspace(0, n - 1, 64).astype(int)
    err = errors(oracle, A, B, C, m, n, k, rows, cols)
    assert err <= 2 * U, (err, handle.nSplitA, handle.nSplitB)


def test_i8_transposes(oracle, handle, ozb, cuda):
    m, n, k = 150, 90, 260
    A = oracle.phi_matrix(k, m, 1.0, 1)  # stored k x m: op(A) = A^T with ta='t'
    B = oracle.phi_matrix(n, k, 1.0, 2)  # stored n x k: op(B) = B^T with tb='t'
    Cn = run_i8(ozb, handle, cuda, A, B, m, n, k, ta="t", tb="t")
    An = np.ascontiguousarray(A.T)  # m x k column-major -> shape (k, m)
    Bn = np.ascontiguousarray(B.T)
    Cr = run_i8(ozb, handle, cuda, An, Bn, m, n, k)
    assert bits_equal(Cn, Cr)


def test_i8_alpha_beta_and_repeatability(oracle, handle, ozb, cuda):
    m, n, k = 257, 129, 384
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    C1 = run_i8(ozb, handle, cuda, A, B, m, n, k, alpha=-0.5, beta=2.0, C0=C0)
    C2 = run_i8(ozb, handle, cuda, A, B, m, n, k, alpha=-0.5, beta=2.0, C0=C0)
    assert bits_equal(C1, C2)
    Cp = run_i8(ozb, handle, cuda, A, B, m, n, k)
    expect = np.fma(-0.5, Cp, 2.0 * C0) if hasattr(np, "fma") else -0.5 * Cp + 2.0 * C0
    assert np.allclose(C1, expect, rtol=4 * U, atol=0)


@pytest.mark.parametrize("nsplit", [4, 6, 8])
def test_i8_truncated_triangular(nsplit, oracle, handle, ozb, cuda):
    """Fewer digits / triangular pairs: the error follows the dropped digit weight 2^-7S."""
    m, n, k = 128, 128, 256
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    C = run_i8(ozb, handle, cuda, A, B, m, n, k, nsplit=nsplit, fast=1)
    assert handle.nSplitA == nsplit and handle.nSplitC == nsplit * (nsplit + 1) // 2
    err = errors(oracle, A, B, C, m, n, k, range(0, m, 8), range(0, n, 8))
    assert err < 2.0 ** (-7 * nsplit + 24), err


def test_i8_vs_plain_error(oracle, handle, ozb, cuda):
    """At a complete split the INT8 form is at least as accurate as the plain FP64-slice form."""
    m, n, k = 128, 128, 1024
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    Ci8 = run_i8(ozb, handle, cuda, A, B, m, n, k)
    handle.nSplitMax = 0
    handle.fastMode = 0
    dC = cuda.zeros((n, m), dtype=cuda.float64, device="cuda")
    ozb.dgemm(handle, "n", "n", m, n, k, 1.0, dev(cuda, A), m, dev(cuda, B), k, 0.0, dC, m)
    Cp = dC.cpu().numpy()
    rows, cols = range(0, m, 4), range(0, n, 4)
    e8 = errors(oracle, A, B, Ci8, m, n, k, rows, cols)
    ep = errors(oracle, A, B, Cp, m, n, k, rows, cols)
    assert e8 <= max(ep, U), (e8, ep)


# ---- grouped launch of many uneven problems (cuozblasDgemmI8Batched) ----

def _batch_case(oracle, shapes, ta, tb, seed):
    """Column-major inputs for each (m, n, k, phi); A stored for op(A) = A ('n') or A^T ('t')."""
    rng = np.random.default_rng(seed)
    probs = []
    for i, (m, n, k, phi) in enumerate(shapes):
        ar, ac = (m, k) if ta == "n" else (k, m)   # A is ar x ac column-major
        br, bc = (k, n) if tb == "n" else (n, k)
        A = oracle.phi_matrix(ar, ac, phi, 100 + i) if ar * ac else np.zeros((max(ac, 1), max(ar, 1)))
        B = oracle.phi_matrix(br, bc, phi, 200 + i) if br * bc else np.zeros((max(bc, 1), max(br, 1)))
        C0 = rng.standard_normal((max(n, 1), max(m, 1)))
        probs.append((m, n, k, A, max(ar, 1), B, max(br, 1), C0, float(rng.choice([1.0, -0.5])),
                      float(rng.choice([0.0, 2.0]))))
    return probs


@pytest.mark.parametrize("ta,tb", [("n", "n"), ("t", "n"), ("n", "t"), ("t", "t")])
@pytest.mark.parametrize("fast", [0, 1])
@pytest.mark.parametrize("split", ["one launch", "three launches"])
def test_i8_batched_matches_single(ta, tb, fast, split, oracle, handle, ozb, cuda, monkeypatch):
    """Every problem of a grouped launch is bit-identical to its own cuozblasDgemmI8 call, with the split of all
    operands as one cooperative launch (then the whole call is two launches: split and products) or as three."""
    if split == "three launches":
        monkeypatch.setenv("OZBLAS_GROUPED_SPLIT3", "1")
    handle.read_env()
    shapes = [(1, 1, 1, 1.0), (64, 300, 129, 0.5), (130, 70, 1000, 2.0), (200, 256, 512, 4.0), (7, 129, 33, 1.0),
              (256, 3, 256, 1.0), (129, 129, 128, 2.0), (90, 40, 0, 1.0), (0, 5, 10, 1.0), (300, 200, 64, 0.5)]
    probs = _batch_case(oracle, shapes, ta, tb, 7 + fast)
    handle.nSplitMax, handle.fastMode = 0, fast
    Cs = [dev(cuda, p[7]) for p in probs]

    def grouped():
        ozb.dgemm_i8_batched(handle, ta, tb, [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                             [p[8] for p in probs], [dev(cuda, p[3]) for p in probs], [p[4] for p in probs],
                             [dev(cuda, p[5]) for p in probs], [p[6] for p in probs], [p[9] for p in probs], Cs,
                             [max(p[0], 1) for p in probs])

    grouped()  # settles the dealing order's measurement
    for c, p in zip(Cs, probs):
        c.copy_(dev(cuda, p[7]))
    l0 = handle.launch_count()
    grouped()
    assert handle.launch_count() - l0 == (2 if split == "one launch" else 4)
    monkeypatch.delenv("OZBLAS_GROUPED_SPLIT3", raising=False)
    handle.read_env()
    for i, p in enumerate(probs):
        m, n, k, A, lda, B, ldb, C0, al, be = p
        dC = dev(cuda, C0)
        if m and n:
            ozb.dgemm_i8(handle, ta, tb, m, n, k, al, dev(cuda, A), lda, dev(cuda, B), ldb, be, dC, max(m, 1))
        assert bits_equal(Cs[i].cpu().numpy(), dC.cpu().numpy()), (i, m, n, k)


@pytest.mark.parametrize("fast", [0, 1])
@pytest.mark.parametrize("ta,tb", [("n", "n"), ("t", "t")])
def test_i8_batched_kernels_match_single(fast, ta, tb, oracle, handle, ozb, cuda, monkeypatch):
    """The grouped launch's product kernel forced to the level-blocked form (widths 4, 3 and 1 within the runs of
    levels, 4 and 3 cut across them) and to the level-wise form: every problem bit-identical to its own cuozblasDgemmI8 call in each case (a K-chunked
    problem, ragged tiles, k = 0 and an empty problem included)."""
    shapes = [(300, 200, 20000, 1.0), (129, 257, 500, 4.0), (1, 1, 1, 1.0), (64, 64, 0, 1.0), (0, 9, 9, 1.0),
              (700, 130, 128, 0.5), (33, 500, 1000, 2.0)]
    probs = _batch_case(oracle, shapes, ta, tb, 21 + fast)
    handle.nSplitMax, handle.fastMode = 0, fast
    singles = []
    for p in probs:
        m, n, k, A, lda, B, ldb, C0, al, be = p
        dC = dev(cuda, C0)
        if m and n:
            ozb.dgemm_i8(handle, ta, tb, m, n, k, al, dev(cuda, A), lda, dev(cuda, B), ldb, be, dC, max(m, 1))
        singles.append(dC.cpu().numpy())
    for var, val in [("OZBLAS_I8_BLOCK", "4"), ("OZBLAS_I8_BLOCK", "3"), ("OZBLAS_I8_BLOCK", "1"),
                     ("OZBLAS_I8_BLOCK", "-4"), ("OZBLAS_I8_BLOCK", "-3"), ("OZBLAS_I8_LEVELWISE", "1")]:
        monkeypatch.setenv(var, val)
        handle.read_env()
        Cs = [dev(cuda, p[7]) for p in probs]
        ozb.dgemm_i8_batched(handle, ta, tb, [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                             [p[8] for p in probs], [dev(cuda, p[3]) for p in probs], [p[4] for p in probs],
                             [dev(cuda, p[5]) for p in probs], [p[6] for p in probs], [p[9] for p in probs], Cs,
                             [max(p[0], 1) for p in probs])
        monkeypatch.delenv(var)
        for i, p in enumerate(probs):
            assert bits_equal(Cs[i].cpu().numpy(), singles[i]), (var, val, i, p[:3])
    handle.read_env()


def test_i8_batched_accuracy_uneven(oracle, handle, ozb, cuda):
    """48 log-uniform shapes in [16, 400], phi from {0.5, 1, 2, 4}: within 2 units of 2^-53 of the exact product."""
    rng = np.random.default_rng(5)
    shapes = [(int(a), int(b), int(c), float(rng.choice([0.5, 1.0, 2.0, 4.0])))
              for a, b, c in np.exp(rng.uniform(np.log(16), np.log(400), (48, 3))).astype(int)]
    probs = _batch_case(oracle, shapes, "n", "n", 11)
    handle.nSplitMax, handle.fastMode = 0, 0
    Cs = [cuda.zeros((p[1], p[0]), dtype=cuda.float64, device="cuda") for p in probs]
    ozb.dgemm_i8_batched(handle, "n", "n", [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                         [1.0] * len(probs), [dev(cuda, p[3]) for p in probs], [p[4] for p in probs],
                         [dev(cuda, p[5]) for p in probs], [p[6] for p in probs], [0.0] * len(probs), Cs,
                         [p[0] for p in probs])
    for i, p in enumerate(probs[:12]):
        m, n, k, A, _, B = p[:6]
        C = Cs[i].cpu().numpy()
        err = errors(oracle, A, B, C, m, n, k, np.linspace(0, m - 1, min(m, 16)).astype(int),
                     np.linspace(0, n - 1, min(n, 16)).astype(int))
        assert err <= 2 * U, (i, m, n, k, err)


# ---- autotuned launch choices: speed only, never bits ----

def test_autotune_changes_no_bits(oracle, handle, ozb, cuda, tmp_path, monkeypatch):
    """Product kernel, block width and strip height (single) and dealing order (grouped) are measured per shape;
    the results equal the untuned defaults bit for bit, and a choice is recorded in $OZBLAS_TUNE_CACHE."""
    m, n, k = 700, 520, 300  # a shape no other test uses (6 tile rows: two strip heights to try)
    A = oracle.phi_matrix(m, k, 1.0, 31)
    B = oracle.phi_matrix(k, n, 1.0, 32)
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("OZBLAS_TUNE_CACHE", str(cache))
    monkeypatch.setenv("OZBLAS_TUNE", "1")
    tuned = run_i8(ozb, handle, cuda, A, B, m, n, k, fast=1)
    monkeypatch.setenv("OZBLAS_TUNE", "0")
    plain = run_i8(ozb, handle, cuda, A, B, m, n, k, fast=1)
    assert bits_equal(tuned, plain)
    text = cache.read_text()
    assert "i8s0:" in text  # the product's launch shape: kernel, block width and strip measured together
    shapes = [(100, 260, 300, 1.0), (390, 70, 129, 2.0), (64, 64, 64, 0.5), (257, 129, 513, 4.0)]
    probs = _batch_case(oracle, shapes, "n", "n", 3)
    outs = []
    for tune in ("1", "0"):
        monkeypatch.setenv("OZBLAS_TUNE", tune)
        Cs = [cuda.zeros((p[1], p[0]), dtype=cuda.float64, device="cuda") for p in probs]
        ozb.dgemm_i8_batched(handle, "n", "n", [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                             [1.0] * 4, [dev(cuda, p[3]) for p in probs], [p[4] for p in probs],
                             [dev(cuda, p[5]) for p in probs], [p[6] for p in probs], [0.0] * 4, Cs,
                             [p[0] for p in probs])
        outs.append([c.cpu().numpy() for c in Cs])
    assert all(bits_equal(a, b) for a, b in zip(*outs))
    assert "i8grouped:" in cache.read_text()


@pytest.mark.parametrize("fast", [0, 1], ids=["full", "triangular"])
@pytest.mark.parametrize("phi", [1.0, 4.0])
def test_i8_correctly_rounded_2048(fast, phi, oracle, handle, ozb, cuda):
    """m = n = k = 2048: every checked entry equals the correctly rounded exact product (RN of the exact dot, from
    the oracle's exact accumulator): 64 x 64 sampled entries plus all of row 0 and column 0, for the full and the
    triangular pair set.  Tolerance: none (bit equality with RN(exact))."""
    n = 2048
    A = oracle.phi_matrix(n, n, phi, 1)  # (k, m): row j is column j of A
    B = oracle.phi_matrix(n, n, phi, 2)  # (n, k): row j is column j of B
    C = run_i8(ozb, handle, cuda, A, B, n, n, n, fast=fast)
    assert handle.nSplitA < 19 and handle.nSplitB < 19, "split must be complete (below the default digit cap)"
    g = np.random.default_rng(11)
    rows = np.sort(g.choice(n, 64, replace=False))
    cols = np.sort(g.choice(n, 64, replace=False))
    At = np.ascontiguousarray(A.T)  # row i of A
    checks = [(At[rows], B[cols], C[np.ix_(cols, rows)]),  # sampled block, (nc, nr) = column-major nr x nc
              (At[0:1], B, C[:, 0:1]),                    # row 0
              (At, B[0:1], C[0:1, :])]                    # column 0
    for Ar, Bc, Cb in checks:
        rn, _ = oracle.exact_gemm_block(Ar, Bc, Cb)
        bad = np.nonzero(rn.view(np.int64) != np.ascontiguousarray(Cb).view(np.int64))
        assert bad[0].size == 0, (bad[0].size, rn[bad][:3], np.ascontiguousarray(Cb)[bad][:3], handle.nSplitC)


def test_i8_wait_timeout_reports_and_recovers(oracle, handle, ozb, cuda):
    """A bounded device wait that runs out: the INT8 kernel's producer holds back its copies (a test switch) and
    the wait limit is 20 ms, so the tensor-core issuer's wait for its first stage gives up; the call returns
    CUOZBLAS_STATUS_DEVICE_TIMEOUT (6) instead of hanging or faulting (the kernel frees its tensor memory first),
    and with the switch and the default limit restored the same call on the same context returns the bits of the
    first call."""
    m = n = k = 1024
    A = oracle.phi_matrix(m, k, 1.0, 1)
    B = oracle.phi_matrix(k, n, 1.0, 2)
    ref = run_i8(ozb, handle, cuda, A, B, m, n, k)  # also settles the shape's launch tuning
    ozb.set_i8_wait_test(20_000_000, hold_copies=True)
    try:
        with pytest.raises(ozb.OzblasError) as e:
            run_i8(ozb, handle, cuda, A, B, m, n, k)
        assert e.value.code == 6
    finally:
        ozb.set_i8_wait_test(0, hold_copies=False)
    cuda.cuda.synchronize()
    again = run_i8(ozb, handle, cuda, A, B, m, n, k)
    assert bits_equal(again, ref)


def test_i8_batched_wait_timeout_reports_and_recovers(oracle, handle, ozb, cuda, monkeypatch):
    """The same bounded wait in the grouped level-blocked kernel: with its producer holding back every copy and a
    20 ms limit, cuozblasDgemmI8Batched returns CUOZBLAS_STATUS_DEVICE_TIMEOUT (6); restored, the same grouped call
    on the same context gives the bits of the first one."""
    monkeypatch.setenv("OZBLAS_I8_BLOCK", "4")
    handle.read_env()
    probs = _batch_case(oracle, [(200, 150, 300, 1.0), (64, 300, 129, 2.0), (1, 1, 1, 1.0)], "n", "n", 41)
    handle.nSplitMax, handle.fastMode = 0, 0

    def grouped():
        Cs = [dev(cuda, p[7]) for p in probs]
        ozb.dgemm_i8_batched(handle, "n", "n", [p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                             [p[8] for p in probs], [dev(cuda, p[3]) for p in probs], [p[4] for p in probs],
                             [dev(cuda, p[5]) for p in probs], [p[6] for p in probs], [p[9] for p in probs], Cs,
                             [max(p[0], 1) for p in probs])
        return [c.cpu().numpy() for c in Cs]

    ref = grouped()
    ozb.set_i8_wait_test(20_000_000, hold_copies=True)
    try:
        with pytest.raises(ozb.OzblasError) as e:
            grouped()
        assert e.value.code == 6
    finally:
        ozb.set_i8_wait_test(0, hold_copies=False)
    cuda.cuda.synchronize()
    again = grouped()
    monkeypatch.delenv("OZBLAS_I8_BLOCK")
    handle.read_env()
    assert all(bits_equal(a, b) for a, b in zip(again, ref))


@pytest.mark.parametrize("m,n,k,phi,fast,ta,tb", [
    (300, 260, 1000, 1.0, 0, "n", "n"),
    (300, 260, 1000, 1.0, 1, "t", "n"),
    (129, 513, 4096, 4.0, 0, "n", "t"),
    (256, 128, 20000, 1.0, 0, "n", "n"),   # K chunks: a level's INT32 sum is split over K
    (130, 200, 20000, 2.0, 1, "t", "t"),
    (1, 1, 7, 1.0, 0, "n", "n"),
    (1000, 900, 3000, 1.0, 1, "n", "n"),
])
def test_i8_level_blocked_equals_levelwise(m, n, k, phi, fast, ta, tb, oracle, handle, ozb, cuda, monkeypatch):
    """The level-blocked product kernel (k_i8_blk) gives the bits of the level-wise one (k_i8_gemm) at every block
    width (levels accumulated together), with blocks within the runs of levels and with equal cuts across them (a
    run flushed in the middle of a block): the same products and sums, in another order of the exact INT32
    accumulations."""
    A = oracle.phi_matrix(m, k, phi, 1) if ta == "n" else oracle.phi_matrix(k, m, phi, 1)
    B = oracle.phi_matrix(k, n, phi, 2) if tb == "n" else oracle.phi_matrix(n, k, phi, 2)
    C0 = oracle.phi_matrix(m, n, 1.0, 3)
    outs = {}
    for name, var, val in [("w4", "OZBLAS_I8_BLOCK", "4"), ("w3", "OZBLAS_I8_BLOCK", "3"),
                           ("w2", "OZBLAS_I8_BLOCK", "2"), ("w1", "OZBLAS_I8_BLOCK", "1"),
                           ("x4", "OZBLAS_I8_BLOCK", "-4"), ("x3", "OZBLAS_I8_BLOCK", "-3"),
                           ("levelwise", "OZBLAS_I8_LEVELWISE", "1")]:
        monkeypatch.setenv(var, val)
        handle.read_env()
        outs[name] = run_i8(ozb, handle, cuda, A, B, m, n, k, ta=ta, tb=tb, fast=fast, alpha=-0.75, beta=0.5, C0=C0)
        monkeypatch.delenv(var)
    handle.read_env()
    for w in ("w4", "w3", "w2", "w1", "x4", "x3"):
        assert bits_equal(outs[w], outs["levelwise"]), w
