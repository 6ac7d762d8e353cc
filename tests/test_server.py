"""The request server (saru_server_*): every request's results are the ones
saru_align_host gives for each of its calls alone, whatever group it ran in,
in pipeline and plain mode and under a device budget that makes admission
wait; calls the banded kernel flags are redone on the exact path."""
from __future__ import annotations

import numpy as np
import pytest

import saruman_b200 as S
from saruman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def make_requests(nreq: int, seed: int) -> list[list[W.Batch]]:
    """Requests of 1-4 calls of mixed read length, k and alphabet; some
    calls have m <= 3k (exact path) or an N-rich alphabet."""
    rng = np.random.default_rng(seed)
    shapes = [(36, 3), (75, 5), (100, 6), (150, 9), (250, 15), (12, 5)]
    reqs = []
    for q in range(nreq):
        calls = []
        for c in range(int(rng.integers(1, 5))):
            m, k = shapes[int(rng.integers(len(shapes)))]
            n = int(rng.integers(1, 900))
            alpha = b"ACGTN" if rng.random() < 0.3 else b"ACGT"
            calls.append(W.random_batch(m, k, n, seed=seed * 1000 + q * 10 + c, err=0.05,
                                        alphabet=alpha))
        reqs.append(calls)
    return reqs


def alone(calls: list[W.Batch]) -> list[S.AlignResult]:
    return [S.align_host(b) for b in calls]


def assert_same(got: S.AlignResult, want: S.AlignResult):
    np.testing.assert_array_equal(got.scores, want.scores)
    np.testing.assert_array_equal(got.read_aln, want.read_aln)
    np.testing.assert_array_equal(got.genome_aln, want.genome_aln)


def run(server: S.Server, reqs: list[list[W.Batch]]):
    hrs = [S.HostRequest(calls) for calls in reqs]
    tickets = [server.submit(h) for h in hrs]
    out = []
    for h, t in zip(hrs, tickets):
        rc, st = server.wait(t)
        assert rc == S.SARU_OK, S.last_error()
        out.append((h, st))
    return out


@pytest.mark.parametrize("pipeline", [True, False])
def test_results_identical_alone_and_in_the_mix(saru_lib, pipeline):
    reqs = make_requests(24, seed=5)
    want = [alone(calls) for calls in reqs]
    with S.Server(pipeline=pipeline, max_requests_per_launch=8, max_inflight=2,
                  budget_bytes=1 << 30) as srv:
        done = run(srv, reqs)
        groups, launches = srv.counters()
    for (h, st), w in zip(done, want):
        for i in range(len(w)):
            assert_same(h.result(i), w[i])
        assert st.submit_us <= st.admit_us <= st.done_us
    redone = sum(st.redone_calls for _, st in done)
    n_exact = sum(1 for calls in reqs for b in calls if b.m <= 3 * b.k)
    assert redone >= n_exact > 0
    if pipeline:
        assert groups < len(reqs)  # requests shared launch groups
        assert max(st.group for _, st in done) == groups - 1
    else:
        assert groups == len(reqs)
        assert launches == sum(1 for calls in reqs for b in calls if b.n)


def test_small_budget_makes_admission_wait(saru_lib):
    """A budget of about two requests: the queue drains through arena reuse,
    with the same results."""
    reqs = make_requests(12, seed=9)
    probe = S.HostRequest(max(reqs, key=lambda c: sum(b.total_genome for b in c)))
    big = sum(b.total_genome * 3 + b.reads.size + 16 * b.n + 4096 for b in probe.batches)
    want = [alone(calls) for calls in reqs]
    with S.Server(pipeline=True, max_requests_per_launch=64, max_inflight=2,
                  budget_bytes=max(2 * big, 1 << 20)) as srv:
        done = run(srv, reqs)
        groups, _ = srv.counters()
    assert groups > 1
    for (h, _), w in zip(done, want):
        for i in range(len(w)):
            assert_same(h.result(i), w[i])


def test_submit_rejects_bad_requests(saru_lib):
    with S.Server(budget_bytes=1 << 20) as srv:
        b = W.random_batch(100, 5, 50, seed=1)
        bad = W.random_batch(100, 5, 50, seed=1)
        bad.mismatch = 2
        with pytest.raises(S.SaruError) as e:
            srv.submit(S.HostRequest([bad]))
        assert e.value.code == S.SARU_E_INVALID
        huge = W.random_batch(100, 5, 20000, seed=2)
        with pytest.raises(S.SaruError) as e:
            srv.submit(S.HostRequest([huge]))
        assert e.value.code == S.SARU_E_NOMEM
        t = srv.submit(S.HostRequest([b]))
        rc, _ = srv.wait(t)
        assert rc == S.SARU_OK
