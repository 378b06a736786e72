"""The INT8 form's level-blocked schedule (cuozblasRuleI8Schedule: the steps the product kernels run), checked on
the host against a restatement of its arithmetic contract.

Whatever the block width and whether the blocks are cut within or across the runs of levels, the kernels must
compute the same thing as the level-wise kernel: every level L accumulated over all K steps exactly once, scaled
by 2^(7 (run_hi(L) - L)) into its run, every run flushed once, in increasing level order, with flush exponent
-7 (run_hi + 2) and carry exponent 7 (next run_hi + 2), the first flush of a tile marked first and the last one
last, and every INT32 accumulator within 2^31 - 1.  The runs are the greedy runs of the level-wise schedule:
consecutive levels whose exact combination (bound pairs(L) x K x 127^2 per level, 7 bits apart) stays below 2^53.
"""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ozblas_b200", "libcuozblas_b200.so")


@pytest.fixture(scope="module")
def sched():
    if not os.path.exists(LIB):
        pytest.fail("libcuozblas_b200.so is not built")
    L = C.CDLL(LIB)
    f = L.cuozblasRuleI8Schedule
    f.argtypes = [C.c_int32] * 5 + [C.POINTER(C.c_int32), C.c_int32]
    f.restype = C.c_int

    def run(nA, nB, nkb, tri, width):
        buf = np.zeros(12 * 4096, dtype=np.int32)
        n = f(nA, nB, nkb, int(tri), width, buf.ctypes.data_as(C.POINTER(C.c_int32)), 4096)
        assert n != -2
        return None if n < 0 else buf[:12 * n].reshape(n, 12)

    return run


def pairs(L, nA, nB):
    return min(L, nA - 1) - max(L - (nB - 1), 0) + 1


def runs_of(nA, nB, nkb, tri):
    """The level-wise schedule's runs (restated): greedy, bound pairs(L) x 128 nkb x 127^2, 7 bits apart."""
    maxlevel = min(nA, nB) - 1 if tri else nA + nB - 2
    lb = [pairs(L, nA, nB) * nkb * 128 * 127 * 127 for L in range(maxlevel + 1)]
    runs, L0 = [], 0
    while L0 <= maxlevel:
        b, L1 = lb[L0], L0
        while L1 + 1 <= maxlevel and (b << 7) + lb[L1 + 1] < (1 << 53):
            b = (b << 7) + lb[L1 + 1]
            L1 += 1
        runs.append((L0, L1))
        L0 = L1 + 1
    return runs


def flush_events(steps, nkb):
    """Replay the epilogue: per flush (run_hi, fexp, cexp, first, last, {level: [(kb0, kb1, scale exponent)]})."""
    events, pending = [], {}

    def add(L, kb0, kb1, run_hi):
        pending.setdefault(L, []).append((kb0, kb1, 7 * (run_hi - L)))

    for (L0, L1, kb0, kb1, run_hi, flags, fexp, cexp, mid, fexp_mid, cexp_mid, first_mid) in steps.tolist():
        assert 0 <= kb0 < kb1 <= nkb and L0 <= mid <= L1
        if mid < L1:  # a block crossing a run boundary is its K range's only chunk
            assert (kb0, kb1) == (0, nkb)
            for L in range(L0, mid + 1):
                add(L, kb0, kb1, mid)
            events.append((mid, fexp_mid, cexp_mid, bool(first_mid), False, pending))
            pending = {}
        for L in range(mid + 1 if mid < L1 else L0, L1 + 1):
            add(L, kb0, kb1, run_hi)
        if flags & 1:
            events.append((run_hi, fexp, cexp, bool(flags & 2), bool(flags & 4), pending))
            pending = {}
    assert not pending, "levels accumulated after the last flush"
    assert steps[-1][5] & 4, "the last step is not marked last"
    return events


SHAPES = [(nA, nB) for nA in (1, 2, 3, 5, 8, 12, 13, 16, 19) for nB in (1, 4, 11, 13, 16, 20)]


@pytest.mark.parametrize("nkb", [1, 3, 16, 64, 80, 157, 600])
@pytest.mark.parametrize("tri", [False, True], ids=["full", "triangular"])
def test_schedules_compute_the_level_wise_sums(sched, nkb, tri):
    checked = 0
    for nA, nB in SHAPES:
        runs = runs_of(nA, nB, nkb, tri)
        for width in (4, 3, 2, 1, -4, -3, -2, -1):
            steps = sched(nA, nB, nkb, tri, width)
            if steps is None:
                # only a cut across runs may be refused, and only where a crossing block would need K chunks
                assert width < 0
                continue
            checked += 1
            events = flush_events(steps, nkb)
            assert [e[0] for e in events] == [hi for _, hi in runs], (nA, nB, width)
            for i, ((lo, hi), (run_hi, fexp, cexp, first, last, acc)) in enumerate(zip(runs, events)):
                assert fexp == -7 * (hi + 2)
                assert first == (i == 0) and last == (i == len(runs) - 1)
                if not last:
                    assert cexp == 7 * (runs[i + 1][1] + 2)
                assert sorted(acc) == list(range(lo, hi + 1))
                for L, parts in acc.items():
                    parts.sort()
                    assert parts[0][0] == 0 and parts[-1][1] == nkb
                    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:])), "K chunks overlap or leave gaps"
                    assert all(p[2] == 7 * (hi - L) for p in parts)
            for (L0, L1, kb0, kb1, *_rest) in steps.tolist():
                assert L1 - L0 + 1 <= abs(width)
                for L in range(L0, L1 + 1):  # every INT32 accumulator stays exact
                    assert pairs(L, nA, nB) * (kb1 - kb0) * 128 * 127 * 127 <= 2**31 - 1
    assert checked > 0


def test_cut_across_runs_has_no_one_level_block_at_8192(sched):
    """The headline shape (13 x 13 digits, 64 K steps, triangular): within the runs the blocks are 4, 4, 4 and 1
    levels; cut across them 3, 3, 3 and 4, each crossing block a single K chunk."""
    within = sched(13, 13, 64, True, 4)
    across = sched(13, 13, 64, True, -4)
    assert [(s[0], s[1]) for s in within.tolist()] == [(0, 3), (4, 7), (8, 11), (12, 12)]
    assert [(s[0], s[1]) for s in across.tolist()] == [(0, 2), (3, 5), (6, 8), (9, 12)]
    assert [s[8] for s in across.tolist()] == [2, 3, 7, 11]  # mid: the last level of the run ending inside
