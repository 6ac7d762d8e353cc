"""The oracle (oracle/saru_oracle.c) pinned against the reference.

1. Against the committed golden fixtures: batches the reference's own
   q-gram filter produced, with the outputs of the reference's own kernel and
   writer (tests/golden/make_golden.py).
2. Where the host build of the reference is present, against the reference
   kernel code on random batches that reach the corners: every flag, N and
   other bytes, non-unit costs, m <= 3k (tracebacks that walk into the
   previous matrix), candidate 0 of a call.
"""
from __future__ import annotations

import numpy as np
import pytest

import golden_io as G
import refkit as R
from saruman_b200 import workloads as W

FIXTURES = G.fixture_names()


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference_golden(name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    sc, ra, ga, st = R.oracle_align(b, nthreads=4)
    assert st == 0
    np.testing.assert_array_equal(sc, exp["scores"])
    assert np.array_equal(ra, exp["read_aln"]), "read alignment slots differ"
    assert np.array_equal(ga, exp["genome_aln"]), "genome alignment slots differ"
    tab = R.name_table(G.names_by_id(b, names))
    tsv, st2, (df, dr) = R.oracle_tsv(b, sc, ra, ga, tab, read_length=m)
    assert st2 == 0
    assert tsv == exp["tsv"]
    assert df + dr == int((sc <= b.k).sum())


def test_golden_fixtures_present():
    assert len(FIXTURES) >= 14


def test_oracle_serial_equals_threaded():
    b = W.random_batch(50, 4, 400, seed=3, err=0.1)
    a = R.oracle_align(b, nthreads=1)
    c = R.oracle_align(b, nthreads=8)
    for x, y in zip(a[:3], c[:3]):
        np.testing.assert_array_equal(x, y)


needs_ref = pytest.mark.skipif(not R.have_ref(), reason="host build of the reference not present")

CORNER_CASES = [
    # (m, k, n, err, alphabet, match, mismatch, flags)
    (36, 2, 300, 0.05, b"ACGT", 0, 1, (1, 3, 5, 7)),
    (36, 3, 300, 0.15, b"ACGTN", 0, 1, (1, 2, 3, 5, 6, 7)),
    (100, 5, 200, 0.08, b"ACGTN", 0, 1, (1, 2, 3, 5, 6, 7)),
    (250, 15, 60, 0.06, b"ACGT", 0, 1, (1, 3, 5, 7)),
    (20, 8, 200, 0.3, b"ACGT", 0, 1, (1, 2, 3, 5, 6, 7)),   # m <= 3k
    (12, 6, 200, 0.4, b"AC", 0, 1, (1, 2, 3, 5, 6, 7)),     # m <= 3k, low entropy
    (30, 3, 200, 0.1, b"ACGTNRY", 1, 2, (1, 2, 3, 5, 6, 7)),  # non-unit costs
    (30, 4, 200, 0.1, b"ACGT", 0, 2, (0, 1, 2, 3, 4, 5, 6, 7)),
    (25, 3, 200, 0.2, b"ACGT", 2, 1, (1, 3)),               # match dearer than mismatch
]


@needs_ref
@pytest.mark.parametrize("case", CORNER_CASES)
def test_oracle_matches_reference_kernel_code(case):
    m, k, n, err, alpha, mat, mis, flags = case
    for seed in range(3):
        b = W.random_batch(m, k, n, seed=seed + 17 * m, err=err, alphabet=alpha, flags=flags)
        b.match, b.mismatch = mat, mis
        rs, rra, rga = R.ref_align(b, strict=True)
        sc, ra, ga, st = R.oracle_align(b, nthreads=1)
        if st & 2:  # the reference reads outside its arrays here: undefined
            continue
        np.testing.assert_array_equal(sc, rs)
        assert np.array_equal(ra, rra) and np.array_equal(ga, rga), (case, seed)


@needs_ref
def test_reference_threaded_driver_equals_serial():
    """The multithreaded host run of the reference kernel (the CPU baseline)
    gives the serial bytes."""
    b = W.random_batch(100, 5, 2000, seed=9, err=0.04)
    a = R.ref_align(b, strict=True)
    c = R.ref_align(b, strict=False, nthreads=8, chunk=64)
    for x, y in zip(a, c):
        np.testing.assert_array_equal(x, y)


def test_whole_call_checker_agrees_with_the_oracle_and_finds_differences():
    """saru_oracle_check (sub-calls led by their predecessor) accepts the
    whole-call oracle's own outputs -- so the lead reproduces the row-0
    walks into the previous matrix -- and counts every planted difference:
    a score, a read-string byte, a window-string byte in a slot's zero tail."""
    for m, k, n, seed in ((36, 2, 9000, 1), (100, 5, 5000, 2), (150, 9, 4500, 3),
                          (250, 15, 2100, 4)):
        b = W.random_batch(m, k, n, seed=seed, err=0.05, alphabet=b"ACGTN")
        s1, ra1, ga1, st = R.oracle_align(b, nthreads=4)
        assert st == 0
        bad, first, cst = R.oracle_check(b, s1, ra1, ga1, nthreads=3)
        assert (bad, first, cst) == (0, -1, 0), (m, k)
        sc2, ra2, ga2 = s1.copy(), ra1.copy(), ga1.copy()
        hit = [t for t in range(n) if s1[t] <= k]
        t1, t2, t3 = hit[3], hit[len(hit) // 2], hit[-1]
        sc2[t1] = (sc2[t1] + 1) % (k + 1)
        slot2 = (int(b.genome_offsets[t2 - 1]) if t2 else 0) + k * t2
        ra2[slot2 + 1] ^= 0x20
        slot3 = (int(b.genome_offsets[t3 - 1]) if t3 else 0) + k * t3
        L3 = int(b.genome_offsets[t3]) - (int(b.genome_offsets[t3 - 1]) if t3 else 0)
        ga2[slot3 + L3 + k - 1] = ord("A")
        bad, first, cst = R.oracle_check(b, sc2, ra2, ga2, nthreads=3)
        assert (bad, first, cst) == (3, t1, 0), (m, k, bad, first)
