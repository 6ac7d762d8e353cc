"""GPU parity of libsaruman_b200.so against the reference and the oracle.

Every comparison is bit-exact: scores (the library reports k + 1 for any
score above k, where the reference's exact value is never printed), both
alignment-slot arrays byte for byte, and the printed TSV.
"""
from __future__ import annotations

import os
import subprocess
import sys
import threading
from pathlib import Path

import numpy as np
import pytest

import golden_io as G
import refkit as R
import saruman_b200 as S
from nwbio import sub_batch
from saruman_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def check_equal(b, exp_scores, exp_ra, exp_ga, r, exact_scores=False):
    """Scores above k are reported as k + 1 by the banded path and exactly
    by the full-rectangle path; both print nothing for them."""
    if exact_scores:
        np.testing.assert_array_equal(r.scores, exp_scores)
    else:
        np.testing.assert_array_equal(np.minimum(r.scores, b.k + 1),
                                      np.minimum(exp_scores, b.k + 1))
    ra = np.asarray(r.read_aln)
    ga = np.asarray(r.genome_aln)
    bad = np.nonzero(ra != exp_ra)[0]
    assert bad.size == 0, f"read slots differ at {bad[:5]}"
    bad = np.nonzero(ga != exp_ga)[0]
    assert bad.size == 0, f"genome slots differ at {bad[:5]}"


@pytest.mark.parametrize("name", G.fixture_names())
def test_golden_batches(saru_lib, name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    r = S.align_host(b, lane=do_rev and 1)
    check_equal(b, exp["scores"], exp["read_aln"], exp["genome_aln"], r)


@pytest.mark.parametrize("name", G.fixture_names())
def test_legacy_entry_prints_reference_tsv(saru_lib, name):
    """cuda_needleman_wunsch, called as the reference's host C calls it,
    prints exactly the reference writer's lines."""
    b, names, do_rev, m, exp = G.load_fixture(name)
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "legacy_call.py"),
                        str(G.GOLDEN / f"{name}.nwb.gz")], capture_output=True, check=True)
    assert r.stdout == exp["tsv"]
    done = int(r.stderr.split(b"DONE ")[1].split()[0])
    assert done == int((exp["scores"] <= b.k).sum())


def test_legacy_entry_large_call_and_new_name_table(saru_lib):
    """A call of 120k candidates (its lines formatted on several host
    threads, written in candidate order) through the drop-in entry prints
    the oracle writer's lines; a second call against another read_names
    table prints that table's names."""
    m, k, n, seed = 100, 5, 120_000, 77
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "legacy_big.py"), str(m), str(k),
                        str(n), str(seed)], capture_output=True, check=True)
    first, second = r.stdout.split(b"==== second call ====\n")
    b = W.random_batch(m, k, n, seed=seed, err=0.05, alphabet=b"ACGTN")
    s1, ra1, ga1, st = R.oracle_align(b, nthreads=8)
    assert st == 0
    n_ids = int(b.ids.max()) + 1
    for out, tag in ((first, b"A"), (second, b"B")):
        names = R.name_table([b"%s_read%d" % (tag, i) for i in range(n_ids)])
        exp, st, _ = R.oracle_tsv(b, s1, ra1, ga1, names, read_length=m)
        assert st == 0 and out == exp, tag
    assert first.count(b"\n") == int((s1 <= k).sum()) > 30_000


RANDOM = [(36, 2), (36, 3), (75, 5), (100, 5), (100, 6), (150, 9), (250, 15), (20, 1),
          (10, 0), (40, 7), (64, 15), (50, 10), (31, 10), (512, 15), (300, 12)]


@pytest.mark.parametrize("m,k", RANDOM)
def test_random_batches_vs_oracle(saru_lib, m, k):
    for seed in range(3):
        for err in (0.02, 0.1, 0.25):
            alpha = b"ACGT" if seed != 1 else b"ACGTNRY"
            b = W.random_batch(m, k, 400 if m < 200 else 120, seed=seed * 31 + m + k, err=err,
                               alphabet=alpha)
            s1, ra1, ga1, st = R.oracle_align(b, nthreads=8)
            r = S.align_host(b)
            check_equal(b, s1, ra1, ga1, r)


GENERAL = [
    # (m, k, err, alphabet, match, mismatch, flags): exact full-rectangle path
    (30, 3, 0.1, b"ACGTNRY", 1, 2, (1, 2, 3, 5, 6, 7)),
    (30, 4, 0.1, b"ACGT", 0, 2, (0, 1, 2, 3, 4, 5, 6, 7)),
    (25, 3, 0.2, b"ACGT", 2, 1, (1, 3)),
    (20, 8, 0.3, b"ACGT", 0, 1, (1, 2, 3, 5, 6, 7)),   # m <= 3k
    (12, 6, 0.4, b"AC", 0, 1, (1, 2, 3, 5, 6, 7)),
    (40, 16, 0.3, b"ACGT", 0, 1, (1, 3, 5, 7)),         # k > 15
    (36, 2, 0.05, b"ACGTNRYKMSWBDHV", 0, 1, (1, 3)),     # > 2 distinct non-ACGT read bytes
]


@pytest.mark.parametrize("case", GENERAL)
def test_general_path_vs_oracle(saru_lib, case):
    m, k, err, alpha, mat, mis, flags = case
    for seed in range(3):
        b = W.random_batch(m, k, 300, seed=seed + 101 * m, err=err, alphabet=alpha, flags=flags)
        b.match, b.mismatch = mat, mis
        s1, ra1, ga1, st = R.oracle_align(b, nthreads=8)
        if st:
            continue  # overflow or undefined bytes in the reference: not comparable
        r = S.align_host(b)
        if (mat, mis) != (0, 1) or m <= 3 * k or k > 15:
            np.testing.assert_array_equal(r.scores, s1)  # full path reports exact scores
        check_equal(b, s1, ra1, ga1, r, exact_scores=(mat, mis) != (0, 1) or m <= 3 * k or k > 15)


def test_irregular_windows_use_exact_path(saru_lib):
    """Windows whose length is not m + so + eo (a caller not built like
    src/hash.c) still give the reference's bytes."""
    rng = np.random.default_rng(7)
    m, k, n = 40, 3, 200
    reads = W.BASES[rng.integers(0, 4, size=(n, m))]
    wins = [W.BASES[rng.integers(0, 4, size=int(rng.integers(m - 5, m + 12)))] for _ in range(n)]
    for t in range(n):  # plant the read so some align
        L = len(wins[t])
        wins[t][:min(L, m)] = reads[t][:min(L, m)]
    b = W.make_batch(m, k, wins, reads, rng.choice([1, 3, 5, 7], size=n).astype(np.int8))
    s1, ra1, ga1, st = R.oracle_align(b)
    r = S.align_host(b)
    np.testing.assert_array_equal(r.scores, s1)
    check_equal(b, s1, ra1, ga1, r, exact_scores=True)


def test_empty_and_single(saru_lib):
    b = W.random_batch(36, 2, 1, seed=1)
    s1, ra1, ga1, _ = R.oracle_align(b)
    check_equal(b, s1, ra1, ga1, S.align_host(b))
    e = W.make_batch(36, 2, [], np.zeros((0, 36), np.uint8), np.zeros(0, np.int8))
    r = S.align_host(e)
    assert r.scores.size == 0


def test_invalid_batch_is_an_error_not_a_crash(saru_lib):
    b = W.random_batch(36, 2, 10, seed=2)
    b.genome_offsets = b.genome_offsets.copy()
    b.genome_offsets[3] = b.genome_offsets[2]  # empty window
    with pytest.raises(S.SaruError) as ei:
        S.align_host(b)
    assert ei.value.code == S.SARU_E_INVALID


def test_two_lanes_concurrently(saru_lib):
    """The forward and reverse reference threads call in parallel."""
    b0 = W.random_batch(100, 5, 3000, seed=11, err=0.05)
    b1 = W.random_batch(75, 5, 3000, seed=12, err=0.05)
    want = [R.oracle_align(b0, nthreads=4), R.oracle_align(b1, nthreads=4)]
    got = [None, None]

    def work(i, b):
        for _ in range(5):
            got[i] = S.align_host(b, lane=i)

    th = [threading.Thread(target=work, args=(i, b)) for i, b in enumerate((b0, b1))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for b, w, g in zip((b0, b1), want, got):
        check_equal(b, w[0], w[1], w[2], g)


def test_device_entry_matches_host_entry(saru_lib):
    import torch
    b = W.random_batch(100, 5, 5000, seed=21, err=0.05)
    host = S.align_host(b)
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(genome=b.genome, reads=b.reads, goff=b.genome_offsets, roff=b.read_offsets,
              dirs=b.dirs).items()}
    scores = torch.zeros(b.n, dtype=torch.int32, device=dev)
    ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nbytes = S.scratch_bytes(b.n, b.m, b.k)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    sb = S.SaruBatch(t["genome"].data_ptr(), t["reads"].data_ptr(), t["goff"].data_ptr(),
                     t["roff"].data_ptr(), t["dirs"].data_ptr(), b.n, b.k, 0, 1, 1, b.m,
                     len(b.genome), b.total_genome)
    sr = S.SaruResult(scores.data_ptr(), ra.data_ptr(), ga.data_ptr(), status.data_ptr())
    stream = torch.cuda.current_stream()
    S.align_device(sb, sr, scratch.data_ptr(), nbytes, stream.cuda_stream)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    np.testing.assert_array_equal(scores.cpu().numpy(), host.scores)
    tot = b.total_genome
    assert np.array_equal(ra[:tot].cpu().numpy(), host.read_aln)
    assert np.array_equal(ga[:tot].cpu().numpy(), host.genome_aln)


def test_misaligned_scratch_is_refused(saru_lib):
    """The kernel copies 16-byte plane units through the scratch: a scratch
    pointer off a 16-byte boundary is refused before anything is enqueued."""
    import torch
    b = W.random_batch(100, 5, 64, seed=22, err=0.05)
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(genome=b.genome, reads=b.reads, goff=b.genome_offsets, roff=b.read_offsets,
              dirs=b.dirs).items()}
    scores = torch.zeros(b.n, dtype=torch.int32, device=dev)
    ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nbytes = S.scratch_bytes(b.n, b.m, b.k)
    scratch = torch.empty(nbytes + 64, dtype=torch.uint8, device=dev)
    sb = S.SaruBatch(t["genome"].data_ptr(), t["reads"].data_ptr(), t["goff"].data_ptr(),
                     t["roff"].data_ptr(), t["dirs"].data_ptr(), b.n, b.k, 0, 1, 1, b.m,
                     len(b.genome), b.total_genome)
    sr = S.SaruResult(scores.data_ptr(), ra.data_ptr(), ga.data_ptr(), status.data_ptr())
    with pytest.raises(S.SaruError, match="16-byte aligned"):
        S.align_device(sb, sr, scratch.data_ptr() + 8, nbytes, 0)
    torch.cuda.synchronize()
    S.align_device(sb, sr, scratch.data_ptr(), nbytes, 0)  # the aligned pointer runs
    torch.cuda.synchronize()
    assert int(status.item()) == 0


@pytest.mark.parametrize("shape", [("c2", 100, 5, 0.03), ("c4", 250, 15, 0.04)])
def test_full_size_batch_sampled_against_oracle(saru_lib, shape):
    """A batch of the benchmark's shape and size; every candidate is
    checked by the oracle on a sample, and all by size-independent
    properties (slot bytes outside the printed strings are zero; aligned
    read strings spell the read)."""
    name, m, k, rate = shape
    g = W.repeat_genome(2_000_000, seed=5) if name == "c2" else W.uniform_genome(2_000_000, 6)
    n_reads = 200_000 if m == 100 else 40_000
    rd = W.sample_reads(g, n_reads, m, rate, seed=7)
    b = W.synthetic_candidates(g, rd, m, k, seed=8, extra_hits=0.3)
    r = S.align_host(b)
    rng = np.random.default_rng(0)
    idx = np.unique(rng.integers(1, b.n, size=400))
    ss = b.slot_starts()
    for i in idx:
        pair, _ = sub_batch(b, [b""] * b.n, int(i) - 1, 2)  # keep candidate i non-first
        s1, ra1, ga1, _ = R.oracle_align(pair)
        assert int(r.scores[i]) == min(int(s1[1]), k + 1)
        lo = int(ss[i])
        hi = lo + int(b.lengths[i]) + k
        o = int(pair.slot_starts()[1])
        assert np.array_equal(r.read_aln[lo:hi], ra1[o:o + hi - lo])
        assert np.array_equal(r.genome_aln[lo:hi], ga1[o:o + hi - lo])
    ok = r.scores <= k
    assert ok.mean() > 0.3
    # read strings without gaps are substrings of the read ending at its end
    reads = b.reads.reshape(-1, m)
    for i in np.nonzero(ok)[0][:2000]:
        lo = int(ss[i])
        s = r.read_aln[lo:lo + int(b.lengths[i]) + k]
        s = s[:np.argmax(s == 0)] if (s == 0).any() else s
        letters = s[s != ord("_")].tobytes()
        assert reads[i].tobytes().endswith(letters)


def _multi_call_setup():
    """Device buffers and expected bytes of seven calls of different read
    lengths, k and band widths, one of them continuing an earlier call."""
    import torch
    dev = torch.device("cuda:0")
    specs = [(36, 3, 3000, True), (75, 5, 2000, True), (100, 6, 2500, True), (150, 9, 1200, True),
             (250, 15, 400, True), (100, 6, 700, False), (40, 2, 33, True)]
    keep, sbs, srs, want = [], [], [], []
    for i, (m, k, n, first) in enumerate(specs):
        b = W.random_batch(m, k, n, seed=100 + i, err=0.05, alphabet=b"ACGT" if i % 3 else b"ACGTN")
        if first:
            s1, ra1, ga1, _ = R.oracle_align(b, nthreads=8)
            want.append((b, s1, ra1, ga1, 0))
        else:
            # candidate 0 continues a call: compare with the oracle's view of
            # the same candidates behind one extra leading candidate
            lead = W.random_batch(m, k, 1, seed=999, err=0.05)
            both = W.make_batch(m, k, [lead.genome] + [b.genome[b.genome_offsets[t] - b.lengths[t]:
                                                                  b.genome_offsets[t]]
                                                       for t in range(b.n)],
                                np.concatenate([lead.reads, b.reads]).reshape(-1, m),
                                np.concatenate([lead.dirs, b.dirs]))
            s1, ra1, ga1, _ = R.oracle_align(both, nthreads=8)
            off = int(both.slot_starts()[1])
            want.append((b, s1[1:], ra1[off:], ga1[off:], 0))
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        bufs = dict(g=T(b.genome), r=T(b.reads), go=T(b.genome_offsets), ro=T(b.read_offsets),
                    d=T(b.dirs), s=torch.zeros(b.n, dtype=torch.int32, device=dev),
                    ra=torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev),
                    ga=torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev))
        keep.append(bufs)
        sbs.append(S.SaruBatch(bufs["g"].data_ptr(), bufs["r"].data_ptr(), bufs["go"].data_ptr(),
                               bufs["ro"].data_ptr(), bufs["d"].data_ptr(), b.n, b.k, 0, 1,
                               1 if first else 0, m, len(b.genome), b.total_genome))
        srs.append(S.SaruResult(bufs["s"].data_ptr(), bufs["ra"].data_ptr(), bufs["ga"].data_ptr(),
                                None))
    return sbs, srs, keep, want


def _check_multi(keep, want):
    for (b, s1, ra1, ga1, _), bufs in zip(want, keep):
        tot = b.total_genome
        r = S.AlignResult(bufs["s"].cpu().numpy(), bufs["ra"][:tot].cpu().numpy(),
                          bufs["ga"][:tot].cpu().numpy())
        check_equal(b, s1, ra1, ga1, r)


def test_multi_call_launch_matches_each_call(saru_lib):
    """Calls of different read lengths, k and band widths (and a call that
    continues an earlier one) aligned in one launch give each call's own
    reference bytes."""
    import torch
    sbs, srs, keep, want = _multi_call_setup()
    status = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    nscr = S.multi_scratch_bytes(sbs)
    scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda:0")
    S.align_multi_device(sbs, srs, status.data_ptr(), scratch.data_ptr(), nscr,
                         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    _check_multi(keep, want)


def test_multi_call_launch_with_compact_records(saru_lib):
    """saru_align_multi_device_compact: the same mixed calls in one launch,
    each call's compact records expanded on the host give its reference
    bytes; every record is fully written (the same bytes on a second run
    over records filled with other bytes)."""
    import torch
    sbs, srs, keep, want = _multi_call_setup()
    status = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    nscr = S.multi_scratch_bytes(sbs)
    scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda:0")
    recs, crs = [], []
    for (b, *_), sr in zip(want, srs):
        rb = S.compact_record_bytes(b.m, b.k)
        rec = torch.full((b.n * rb,), 0x5A, dtype=torch.uint8, device="cuda:0")
        recs.append((rec, rb))
        crs.append(S.SaruResult(sr.scores, rec.data_ptr(), None, None))
    outs = []
    for fill in (0x5A, 0xC3):
        for rec, _ in recs:
            rec.fill_(fill)
        S.align_multi_device_compact(sbs, crs, status.data_ptr(), scratch.data_ptr(), nscr,
                                     torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        outs.append([rec.cpu().numpy() for rec, _ in recs])
    for (b, s1, ra1, ga1, _), sb, bufs, (rec, rb), r0, r1 in zip(want, sbs, keep, recs, *outs):
        assert np.array_equal(r0, r1)
        sc = bufs["s"].cpu().numpy()
        ex = S.expand_compact(b, sc, r0, rb, first_of_call=bool(sb.first_of_call))
        check_equal(b, s1, ra1, ga1, ex)


def test_multi_call_request_replays_from_a_cuda_graph(saru_lib):
    """saru_align_multi_device captured once in a CUDA graph (its class
    launches forked onto side streams and joined back inside the capture)
    and replayed: every replay rewrites each call's reference bytes."""
    import torch
    sbs, srs, keep, want = _multi_call_setup()
    status = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    nscr = S.multi_scratch_bytes(sbs)
    scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda:0")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):  # first call outside capture: one-time setup
        S.align_multi_device(sbs, srs, status.data_ptr(), scratch.data_ptr(), nscr,
                             side.cuda_stream)
    side.synchronize()
    g = torch.cuda.CUDAGraph()
    n0 = S.kernel_launches()
    with torch.cuda.graph(g):
        S.align_multi_device(sbs, srs, status.data_ptr(), scratch.data_ptr(), nscr,
                             torch.cuda.current_stream().cuda_stream)
    assert S.kernel_launches() - n0 >= 1
    for _ in range(2):
        for bufs in keep:
            for key in ("s", "ra", "ga"):
                bufs[key].zero_()
        g.replay()
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        _check_multi(keep, want)
    del g


def _compact_roundtrip(b):
    """saru_align_device_compact on the GPU, records expanded on the host."""
    import torch
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    g, r, go, ro, d = T(b.genome), T(b.reads), T(b.genome_offsets), T(b.read_offsets), T(b.dirs)
    R_ = S.compact_record_bytes(b.m, b.k)
    sc = torch.zeros(max(b.n, 1), dtype=torch.int32, device=dev)
    rec = torch.zeros(max(b.n, 1) * R_, dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    sb = S.SaruBatch(g.data_ptr(), r.data_ptr(), go.data_ptr(), ro.data_ptr(), d.data_ptr(), b.n,
                     b.k, 0, 1, 1, b.m, len(b.genome), b.total_genome)
    nscr = S.scratch_bytes(b.n, b.m, b.k)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    S.align_device_compact(sb, sc.data_ptr(), rec.data_ptr(), R_, st.data_ptr(), scr.data_ptr(),
                           nscr)
    torch.cuda.synchronize()
    _compact_roundtrip.last = (sc.cpu().numpy()[:b.n], rec.cpu().numpy(), R_)
    return int(st.item()), S.expand_compact(b, sc.cpu().numpy()[:b.n], rec.cpu().numpy(), R_)


@pytest.mark.parametrize("name", G.fixture_names())
def test_compact_records_rebuild_the_golden_slots(saru_lib, name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    if not (b.m > 3 * b.k and b.k <= 15 and b.match == 0 and b.mismatch == 1):
        pytest.skip("outside the banded kernel's domain")
    st, r = _compact_roundtrip(b)
    if st & (S.SARU_S_IRREGULAR | S.SARU_S_ALPHABET):
        pytest.skip("fixture takes the exact path")
    assert st == 0
    check_equal(b, exp["scores"], exp["read_aln"], exp["genome_aln"], r)
    # the reference's TSV straight from the device's records
    sc, rec, rb = _compact_roundtrip.last
    text, _, _ = S.format_tsv_compact(b, sc, rec, rb, S.name_table(G.names_by_id(b, names)),
                                      read_length=m, nthreads=4)
    assert text == exp["tsv"]


@pytest.mark.parametrize("m,k", [(36, 3), (100, 5), (150, 9), (250, 15)])
def test_compact_records_match_slot_mode(saru_lib, m, k):
    b = W.random_batch(m, k, 1500, seed=m * 7 + k, err=0.05, alphabet=b"ACGTN")
    st, r = _compact_roundtrip(b)
    assert st == 0
    want = S.align_host(b)
    assert np.array_equal(r.scores, want.scores)
    assert np.array_equal(r.read_aln, want.read_aln)
    assert np.array_equal(r.genome_aln, want.genome_aln)
