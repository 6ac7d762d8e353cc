"""Autotuner of the banded kernel's launch shape: the tuning table (host
only), every shape of the search space gives the reference bytes, and the
tuner installs its fastest shape."""
from __future__ import annotations

import numpy as np
import pytest

import refkit as R
import saruman_b200 as S
from saruman_b200 import autotune as A
from saruman_b200 import workloads as W


def test_search_space():
    assert len(A.search_space(5)) == 24 and len(A.search_space(9)) == 12
    assert all(b == 64 for _, _, b in A.search_space(12))


def test_tuning_table_roundtrip_and_validation(saru_lib):
    S.clear_tuning()
    assert S.get_tuning(100, 5) is None
    S.set_tuning(100, 5, 2, 3, 64)
    assert S.get_tuning(100, 5) == (2, 3, 64)
    for bad in [(5, 0, 0), (1, 17, 0), (1, 0, 48)]:
        with pytest.raises(S.SaruError):
            S.set_tuning(100, 5, *bad)
    with pytest.raises(S.SaruError):  # 32-bit band words cannot hold a k = 9 band
        S.set_tuning(150, 9, 1, 0, 32)
    S.clear_tuning(100, 5)
    assert S.get_tuning(100, 5) is None
    S.set_tuning(100, 5, 1, 0, 0)
    S.clear_tuning()
    assert S.get_tuning(100, 5) is None


@pytest.mark.gpu
@pytest.mark.parametrize("m,k", [(36, 3), (100, 5), (150, 9)])
def test_every_shape_gives_the_reference_bytes(saru_lib, m, k):
    b = W.random_batch(m, k, 700, seed=m + k, err=0.05, alphabet=b"ACGTN")
    s1, ra1, ga1, _ = R.oracle_align(b, nthreads=8)
    try:
        for shape in A.search_space(k):
            S.set_tuning(m, k, *shape)
            r = S.align_host(b)
            np.testing.assert_array_equal(np.minimum(r.scores, k + 1), np.minimum(s1, k + 1))
            assert np.array_equal(r.read_aln, ra1), shape
            assert np.array_equal(r.genome_aln, ga1), shape
    finally:
        S.clear_tuning()


@pytest.mark.gpu
def test_tuner_installs_its_fastest_shape(saru_lib):
    sample = A.Sample.build(100, 5, 20_000, seed=3)
    try:
        res = A.tune_bin(sample, reps=3)
        assert S.get_tuning(100, 5) == tuple(res["best"])
        assert res["ms"][res["best"]] <= res["default_ms"]
        assert len(res["ms"]) == 25  # the search space and the default shape
    finally:
        S.clear_tuning()
