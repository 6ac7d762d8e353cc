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


def gather_case(m: int, k: int, nreads: int, seed: int, n_alpha: bool = False):
    """A genome, its sequenced reads and the candidate batch the filter's
    host loop would build from them (windows + reverse-complemented reads)."""
    g = W.uniform_genome(300_000, seed=seed)
    if n_alpha:  # a few N runs in the genome
        g = g.copy()
        g[1000:1010] = ord("N")
        g[50_000:50_003] = ord("N")
    rd = W.sample_reads(g, nreads, m, 0.03, seed=seed + 1, unmapped=0.05)
    b = W.synthetic_candidates(g, rd, m, k, seed=seed + 2, extra_hits=1.5)
    return g, rd.seqs, b


def test_gather_device_builds_the_reference_layout(saru_lib):
    """saru_gather_device writes exactly the windows, reads and read offsets
    of the host-built call, and aligning them gives saru_align_host's bytes."""
    import torch
    dev = torch.device("cuda:0")
    g, table, b = gather_case(100, 5, 3000, seed=21, n_alpha=True)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dg, dt, di, dp, dd, dgo = (T(g), T(table.reshape(-1)), T(b.ids), T(b.pos), T(b.dirs),
                               T(b.genome_offsets))
    win = torch.zeros(len(b.genome) + 64, dtype=torch.uint8, device=dev)
    rds = torch.zeros(b.n * b.m + 64, dtype=torch.uint8, device=dev)
    ro = torch.zeros(b.n, dtype=torch.int32, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    call = S.SaruGatherCall(dt.data_ptr(), di.data_ptr(), dp.data_ptr(), dd.data_ptr(),
                            dgo.data_ptr(), b.n, table.shape[0], b.k, 0, 1, 1, b.m,
                            len(b.genome), b.total_genome)
    sb = S.gather_device(call, dg.data_ptr(), len(g), win.data_ptr(), rds.data_ptr(),
                         ro.data_ptr(), st.data_ptr())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    np.testing.assert_array_equal(win[:len(b.genome)].cpu().numpy(), b.genome)
    np.testing.assert_array_equal(rds[:b.n * b.m].cpu().numpy(), b.reads)
    np.testing.assert_array_equal(ro.cpu().numpy(), b.read_offsets)
    sc = torch.zeros(b.n, dtype=torch.int32, device=dev)
    ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    res = S.SaruResult(sc.data_ptr(), ra.data_ptr(), ga.data_ptr(), st.data_ptr())
    nscr = S.scratch_bytes(b.n, b.m, b.k)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    S.align_device(sb, res, scr.data_ptr(), nscr)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    want = S.align_host(b)
    assert_same(S.AlignResult(sc.cpu().numpy(), ra[:b.total_genome].cpu().numpy(),
                              ga[:b.total_genome].cpu().numpy()), want)


def test_gather_flags_candidates_outside_the_genome(saru_lib):
    import torch
    dev = torch.device("cuda:0")
    g, table, b = gather_case(36, 2, 200, seed=3)
    pos = b.pos.copy()
    pos[7] = len(g) - 10  # window runs past the genome end
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dg, dt, di, dp, dd, dgo = (T(g), T(table.reshape(-1)), T(b.ids), T(pos), T(b.dirs),
                               T(b.genome_offsets))
    win = torch.zeros(len(b.genome) + 64, dtype=torch.uint8, device=dev)
    rds = torch.zeros(b.n * b.m + 64, dtype=torch.uint8, device=dev)
    ro = torch.zeros(b.n, dtype=torch.int32, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    call = S.SaruGatherCall(dt.data_ptr(), di.data_ptr(), dp.data_ptr(), dd.data_ptr(),
                            dgo.data_ptr(), b.n, table.shape[0], b.k, 0, 1, 1, b.m,
                            len(b.genome), b.total_genome)
    S.gather_device(call, dg.data_ptr(), len(g), win.data_ptr(), rds.data_ptr(), ro.data_ptr(),
                    st.data_ptr())
    torch.cuda.synchronize()
    assert int(st.item()) & S.SARU_S_GATHER


def gather_case_on(g, m: int, k: int, nreads: int, seed: int):
    rd = W.sample_reads(g, nreads, m, 0.03, seed=seed + 1, unmapped=0.05)
    b = W.synthetic_candidates(g, rd, m, k, seed=seed + 2, extra_hits=1.5)
    return rd.seqs, b


def test_server_resident_genome_requests(saru_lib):
    """Gather requests against the resident genome (kept 2 bits a base on
    the device, its N runs and other non-ACGT bytes as exceptions) give
    saru_align_host's bytes for the host-built calls, mixed with window
    requests; a call with m <= 3k is redone on the exact path from its
    gathered windows."""
    g = W.uniform_genome(300_000, seed=40).copy()
    g[1000:1010] = ord("N")
    g[50_000:50_003] = ord("N")
    g[120_000] = ord("R")
    g[7919::7919] = ord("Y")
    g[-3:] = ord("N")
    shapes = [(36, 3, 2000), (75, 5, 1500), (100, 6, 1200), (150, 9, 800), (12, 5, 300)]
    cases = [gather_case_on(g, m, k, n, seed=40 + 7 * i) for i, (m, k, n) in enumerate(shapes)]
    with S.Server(pipeline=True, max_requests_per_launch=8, budget_bytes=1 << 30) as srv:
        srv.set_genome(g)
        reqs = []
        for table, b in cases:
            reqs.append(S.GatherRequest([b], [table]))
            reqs.append(S.HostRequest([b]))
        reqs.append(S.GatherRequest([b for _, b in cases], [t for t, _ in cases]))
        tickets = [srv.submit(r) for r in reqs]
        with pytest.raises(S.SaruError):  # requests are unfinished until waited for
            srv.set_genome(g)
        redone = 0
        for t in tickets:
            rc, st = srv.wait(t)
            assert rc == S.SARU_OK, S.last_error()
            redone += st.redone_calls
        assert redone >= 3  # the m <= 3k call, alone twice and inside the last request
        srv.set_genome(g)
    for i, (table, b) in enumerate(cases):
        want = S.align_host(b)
        assert_same(reqs[2 * i].result(0), want)
        assert_same(reqs[2 * i + 1].result(0), want)
        assert_same(reqs[-1].result(i), want)


def test_gather_request_needs_a_genome(saru_lib):
    g, table, b = gather_case(36, 2, 100, seed=5)
    with S.Server(budget_bytes=1 << 24) as srv:
        with pytest.raises(S.SaruError) as e:
            srv.submit(S.GatherRequest([b], [table]))
        assert e.value.code == S.SARU_E_INVALID


def test_compact_requests_expand_to_the_same_bytes(saru_lib):
    """Requests asking for compact records (window and gather calls, an
    m <= 3k call redone on the exact path) expand on the host to exactly
    saru_align_host's slots, mixed with slot-string requests."""
    g = W.uniform_genome(300_000, seed=60)
    shapes = [(36, 3, 1500), (100, 6, 1200), (150, 9, 700), (12, 5, 200)]
    cases = [gather_case_on(g, m, k, n, seed=60 + 5 * i) for i, (m, k, n) in enumerate(shapes)]
    for pipeline in (True, False):
        with S.Server(pipeline=pipeline, max_requests_per_launch=8, budget_bytes=1 << 30) as srv:
            srv.set_genome(g)
            reqs = []
            for table, b in cases:
                reqs.append(S.GatherRequest([b], [table], compact=True))
                reqs.append(S.HostRequest([b], compact=True))
                reqs.append(S.HostRequest([b]))
            tickets = [srv.submit(r) for r in reqs]
            for t in tickets:
                rc, _ = srv.wait(t)
                assert rc == S.SARU_OK, S.last_error()
        for i, (table, b) in enumerate(cases):
            want = S.align_host(b)
            for r in reqs[3 * i:3 * i + 3]:
                assert_same(r.result(0), want)


def test_a_bad_request_fails_alone(saru_lib):
    """A gather request with a candidate outside the genome ends with
    SARU_E_INVALID; the requests around it, in the same launch groups,
    still get saru_align_host's bytes."""
    g = W.uniform_genome(200_000, seed=70)
    good = [gather_case_on(g, 100, 5, 600, seed=71 + i) for i in range(4)]
    table, bad = gather_case_on(g, 100, 5, 300, seed=90)
    bad.pos = bad.pos.copy()
    bad.pos[10] = len(g) - 20  # its window runs past the genome end
    with S.Server(pipeline=True, max_requests_per_launch=8, budget_bytes=1 << 28) as srv:
        srv.set_genome(g)
        reqs = [S.GatherRequest([b], [t]) for t, b in good[:2]]
        reqs.append(S.GatherRequest([bad], [table]))
        reqs += [S.GatherRequest([b], [t]) for t, b in good[2:]]
        tickets = [srv.submit(r) for r in reqs]
        rcs = [srv.wait(t)[0] for t in tickets]
    assert rcs == [S.SARU_OK, S.SARU_OK, S.SARU_E_INVALID, S.SARU_OK, S.SARU_OK]
    for r, (t, b) in zip(reqs[:2] + reqs[3:], good):
        assert_same(r.result(0), S.align_host(b))


def test_concurrent_clients(saru_lib):
    """Four client threads submit and wait on their own requests at once;
    every request's bytes equal saru_align_host's."""
    import threading
    reqs = make_requests(32, seed=11)
    want = [alone(calls) for calls in reqs]
    hrs = [S.HostRequest(calls) for calls in reqs]
    errors = []
    with S.Server(pipeline=True, max_requests_per_launch=16, budget_bytes=1 << 29) as srv:
        def client(c):
            try:
                mine = list(range(c, len(hrs), 4))
                tickets = [srv.submit(hrs[q]) for q in mine]
                for t in tickets:
                    rc, _ = srv.wait(t)
                    assert rc == S.SARU_OK
            except Exception as e:  # surfaced in the main thread
                errors.append(e)
        th = [threading.Thread(target=client, args=(c,)) for c in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join(300)
    assert not errors, errors
    for h, w in zip(hrs, want):
        for i in range(len(w)):
            assert_same(h.result(i), w[i])


# ---- reads-only requests: the filter inside the request path -------------

def read_lines(res: dict, g: np.ndarray, reads: np.ndarray, m: int, k: int,
               names: list[bytes]) -> list[bytes]:
    """Every line the reference program prints for a reads-only request's
    set: the writer's lines of each call, and the filter's perfect hits."""
    cs = W.callset(g, reads, m, k, res["ids"], res["pos"], res["dirs"], res["call_begin"],
                   res["call_strand"])
    tab = S.name_table(names)
    lines = []
    for c in range(cs.ncalls):
        b = cs.call(c)
        a0, a1 = int(res["call_begin"][c]), int(res["call_begin"][c + 1])
        s0, s1 = int(res["slot_begin"][c]), int(res["slot_begin"][c + 1])
        if "records" in res:
            rb = res["record_bytes"]
            r = S.expand_compact(b, res["scores"][a0:a1], res["records"][a0 * rb:a1 * rb], rb)
        else:
            r = S.AlignResult(res["scores"][a0:a1], res["read_aln"][s0:s1],
                              res["genome_aln"][s0:s1])
        text, _, _ = S.format_tsv(b, r, tab, read_length=m)
        lines += text.splitlines(keepends=True)
    for rid, g1, st in zip(res["perfect_ids"], res["perfect_pos"], res["perfect_strand"]):
        rd = reads[rid]
        if st == 4:
            rd = W.reverse_complement(rd[None])[0]
        lines.append(b"%s\t%d\t%d\t%s\t%s\t%s\t0\n" % (
            names[rid], g1, g1 - 1 + m, b"<<" if st == 4 else b">>", g[g1:g1 + m].tobytes(),
            rd.tobytes()))
    return lines


def host_pipeline(g, reads, m, k, cv):
    """The same reads through the device filter and saru_align_host call by
    call (the pipeline the reference's strand daemons run)."""
    with S.Filter(g, m, k) as f:
        outs = [(dr, f.run(reads, dr, cv)) for dr in (0, 4)]
    ids = np.concatenate([o.ids for _, o in outs])
    pos = np.concatenate([o.pos for _, o in outs])
    dirs = np.concatenate([o.dirs for _, o in outs])
    cb, strand, off = [0], [], 0
    for dr, o in outs:
        cb.extend((o.call_begin[1:] + off).tolist())
        strand += [dr] * (len(o.call_begin) - 1)
        off += len(o.ids)
    cs = W.callset(g, reads, m, k, ids, pos, dirs, np.asarray(cb), np.asarray(strand))
    res = [S.align_host(cs.call(c)) for c in range(cs.ncalls)]
    return cs, res


def test_reads_only_requests_print_the_reference_output(saru_lib):
    """A request of reads only (the drop-in dataset's reads) through the
    server -- filter on both strands, calls, gather, alignment -- prints
    exactly the reference program's output (SHA-256 of the sorted lines),
    alone and in the middle of a mix of other reads-only requests of other
    read lengths; every request's calls equal the device filter followed by
    saru_align_host call by call."""
    import hashlib
    import json
    from pathlib import Path
    spec = json.loads((Path(__file__).resolve().parent / "golden" /
                       "dropin_c1small.json").read_text())
    g = W.uniform_genome(spec["genome_len"], seed=spec["genome_seed"])
    m = spec["m"]
    k = int(np.floor(m * spec["e"]))
    reads = W.sample_reads(g, spec["reads"], m, spec["rate"], seed=spec["read_seed"]).seqs
    cv = int(spec["args"][spec["args"].index("-s") + 1])
    names = [b"r%d" % i for i in range(reads.shape[0])]
    others = []
    for i, (mo, ko, nr) in enumerate([(75, 5, 900), (100, 6, 1500), (36, 3, 3000),
                                      (150, 9, 700)]):
        rd = W.sample_reads(g, nr, mo, 0.03, seed=300 + i).seqs
        others.append((rd, ko, 0))
    for compact in (False, True):
        with S.Server(pipeline=True, max_requests_per_launch=8, max_inflight=2,
                      budget_bytes=2 << 30) as srv:
            srv.set_genome(g)
            t_alone = srv.submit_reads([(reads, k, cv)], compact=compact)
            rc, _ = srv.wait(t_alone)
            assert rc == S.SARU_OK, S.last_error()
            alone_res = srv.read_results(t_alone, 0)
            srv.release(t_alone)
            # the same request in the middle of a mix (submitted at once)
            ts = [srv.submit_reads([others[0], others[1]], compact=compact),
                  srv.submit_reads([(reads, k, cv)], compact=compact),
                  srv.submit_reads([others[2], others[3]], compact=compact)]
            for t in ts:
                rc, _ = srv.wait(t)
                assert rc == S.SARU_OK, S.last_error()
            mix_res = srv.read_results(ts[1], 0)
            other_res = [srv.read_results(ts[0], 0), srv.read_results(ts[0], 1),
                         srv.read_results(ts[2], 0), srv.read_results(ts[2], 1)]
            for t in ts:
                srv.release(t)
        for key in alone_res:
            np.testing.assert_array_equal(alone_res[key], mix_res[key], err_msg=key)
        lines = sorted(read_lines(mix_res, g, reads, m, k, names))
        assert len(lines) == spec["lines"]
        assert hashlib.sha256(b"".join(lines)).hexdigest() == spec["sha256_sorted_stdout"]
        for (rd, ko, _), res in zip(others, other_res):
            mo = rd.shape[1]
            cs, want = host_pipeline(g, rd, mo, ko, W.chunk_value_for(mo, ko))
            np.testing.assert_array_equal(res["ids"], cs.ids)
            np.testing.assert_array_equal(res["call_begin"], cs.call_begin)
            for c in range(cs.ncalls):
                a0, a1 = int(cs.call_begin[c]), int(cs.call_begin[c + 1])
                s0, s1 = int(cs.sbase[c]), int(cs.sbase[c + 1])
                np.testing.assert_array_equal(res["scores"][a0:a1], want[c].scores)
                if compact:
                    rb = res["record_bytes"]
                    got = S.expand_compact(cs.call(c), res["scores"][a0:a1],
                                           res["records"][a0 * rb:a1 * rb], rb)
                    assert_same(got, want[c])
                else:
                    np.testing.assert_array_equal(res["read_aln"][s0:s1], want[c].read_aln)
                    np.testing.assert_array_equal(res["genome_aln"][s0:s1], want[c].genome_aln)


def test_reads_only_request_needs_a_genome_and_valid_sets(saru_lib):
    with S.Server(pipeline=True, budget_bytes=1 << 28) as srv:
        rd = np.frombuffer(b"ACGT" * 25, np.uint8).reshape(1, 100)
        with pytest.raises(S.SaruError):
            srv.submit_reads([(rd, 5, 0)])
        srv.set_genome(W.uniform_genome(50_000, seed=2))
        with pytest.raises(S.SaruError):
            srv.submit_reads([(rd, 16, 0)])  # k > 15
        t = srv.submit_reads([(np.zeros((0, 100), np.uint8), 5, 0)])  # nothing to align
        rc, _ = srv.wait(t)
        assert rc == S.SARU_OK
        assert srv.read_results(t, 0)["ids"].size == 0
        srv.release(t)
