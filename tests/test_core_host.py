"""CPU check of the device alignment core (saruman_b200/csrc/saru_core.cuh).

The header is compiled for the host by g++ into a test-only library
(tests/harness/core_host.cpp) so that the bit-parallel banded fill, the
decision planes and the traceback can be compared with the oracle on many
inputs without a GPU.  The product runs the same header on the GPU only.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

import golden_io as G
import refkit as R
from saruman_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
SO = ROOT / "tests" / "_build" / "libcore_host.so"


@pytest.fixture(scope="module")
def core():
    SO.parent.mkdir(exist_ok=True)
    src = ROOT / "tests" / "harness" / "core_host.cpp"
    hdr = ROOT / "saruman_b200" / "csrc" / "saru_core.cuh"
    if not SO.exists() or SO.stat().st_mtime < max(src.stat().st_mtime, hdr.stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(SO), str(src)],
                       check=True)
    return C.CDLL(str(SO))


def run_core(lib, b, first=True):
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    tot = b.total_genome
    sc = np.zeros(max(b.n, 1), np.int32)
    ra = np.zeros(tot + 64, np.uint8)
    ga = np.zeros(tot + 64, np.uint8)
    wide = 1 if b.k > 7 else 0
    fl = lib.core_align_batch(P(b.genome), P(b.reads), P(b.genome_offsets), P(b.read_offsets),
                              P(b.dirs), C.c_int(b.n), C.c_int(b.k), C.c_int(wide),
                              C.c_int(1 if first else 0), P(sc), P(ra), P(ga))
    return sc[:b.n], ra[:tot], ga[:tot], fl


CASES = [(36, 2), (36, 3), (75, 5), (100, 5), (100, 6), (150, 9), (250, 15), (20, 1), (10, 0),
         (40, 7), (64, 15), (50, 10), (31, 10), (512, 15), (2, 0), (4, 1)]


@pytest.mark.parametrize("m,k", CASES)
def test_core_matches_oracle_random(core, m, k):
    for seed in range(4):
        for err in (0.02, 0.08, 0.2):
            alpha = b"ACGT" if seed % 2 else b"ACGTNX"
            b = W.random_batch(m, k, 200, seed=seed * 7 + m, err=err, alphabet=alpha)
            s1, ra1, ga1, st = R.oracle_align(b, nthreads=4)
            s2, ra2, ga2, fl = run_core(core, b)
            assert fl == 0
            np.testing.assert_array_equal(np.minimum(s1, k + 1), s2)
            assert np.array_equal(ra1, ra2) and np.array_equal(ga1, ga2), (m, k, seed, err)


@pytest.mark.parametrize("name", G.fixture_names())
def test_core_matches_golden(core, name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    s2, ra2, ga2, fl = run_core(core, b)
    assert fl == 0
    np.testing.assert_array_equal(np.minimum(exp["scores"], b.k + 1), s2)
    assert np.array_equal(exp["read_aln"], ra2) and np.array_equal(exp["genome_aln"], ga2)


def test_core_continuation_batch(core):
    """A batch that continues a call: its candidate 0 walks row 0 like any
    later candidate of the reference."""
    b = W.random_batch(40, 3, 300, seed=5, err=0.08)
    s1, ra1, ga1, st = R.oracle_align(b)
    # drop candidate 0 from the oracle's view by comparing candidates 1.. of
    # a continuation run of candidates 1..n-1
    from nwbio import sub_batch
    sb, _ = sub_batch(b, [b""] * b.n, 1, b.n - 1)
    s2, ra2, ga2, fl = run_core(core, sb, first=False)
    off = int(b.slot_starts()[1])
    np.testing.assert_array_equal(np.minimum(s1[1:], b.k + 1), s2)
    assert np.array_equal(ra1[off:], ra2) and np.array_equal(ga1[off:], ga2)
