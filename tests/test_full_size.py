"""Benchmarked configurations at their full size, every candidate checked
against the oracle.

Each configuration's workload is built exactly as bench.py builds it: the
reads of every length bin, the calls the reference's q-gram filter makes
for them on both strands (the library's device filter), cut at the
reference's queue threshold.  Every call goes through the host entry point
(saru_align_host) and every candidate of every call is compared with the
oracle (oracle/saru_oracle.c through saru_oracle_check, on all host
threads): min(score, k + 1) and both L + k byte slots.  The TSV lines the
library's writer prints for each call are compared with the oracle's
writer.  Each configuration prints its candidate count and a SHA-256 of its
outputs."""
from __future__ import annotations

import hashlib
import importlib.util
import os
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

import refkit as R
import saruman_b200 as S

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_mod"] = mod
    spec.loader.exec_module(mod)
    return mod


def align_and_check(cs, tag: str, report, outputs=None) -> None:
    """Aligns every call of CallSet `cs` on the GPU (or takes `outputs` =
    (scores, read strings, window strings) made elsewhere) and checks every
    candidate and every call's TSV against the oracle."""
    k, m = cs.k, cs.m
    cb, sb = cs.call_begin, cs.sbase
    spans = [(int(cb[c]), int(cb[c + 1]), int(sb[c]), int(sb[c + 1])) for c in range(cs.ncalls)]
    if outputs is None:
        sc = np.zeros(cs.n, np.int32)
        ra = np.zeros(cs.total_slots + 64, np.uint8)
        ga = np.zeros(cs.total_slots + 64, np.uint8)
        for c, (a0, a1, s0, s1) in enumerate(spans):
            S.align_host(cs.call(c), lane=0, out=S.AlignResult(sc[a0:a1], ra[s0:s1], ga[s0:s1]))
    else:
        sc, ra, ga = outputs
    bad_total = 0
    for c, (a0, a1, s0, s1) in enumerate(spans):
        bad, first, st = R.oracle_check(cs.call(c), sc[a0:a1], ra[s0:s1], ga[s0:s1])
        assert st == 0, (tag, c, st)
        assert bad == 0, f"{tag}: call {c}: {bad} candidates differ, first {first}"
        bad_total += bad
    # the writer's lines, call by call, against the oracle's writer
    n_ids = int(cs.ids.max()) + 1
    names_l = [b"read%d" % i for i in range(n_ids)]
    lib_names, ora_names = S.name_table(names_l), R.name_table(names_l)

    def tsv(c):
        a0, a1, s0, s1 = spans[c]
        b = cs.call(c)
        res = S.AlignResult(sc[a0:a1], ra[s0:s1], ga[s0:s1])
        ours, _, _ = S.format_tsv(b, res, lib_names, read_length=m)
        theirs, st, _ = R.oracle_tsv(b, sc[a0:a1], ra[s0:s1], ga[s0:s1], ora_names,
                                     read_length=m)
        return ours == theirs and st == 0, len(ours)

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        res = list(ex.map(tsv, range(cs.ncalls)))
    assert all(ok for ok, _ in res), [c for c, (ok, _) in enumerate(res) if not ok][:5]
    h = hashlib.sha256()
    for a in (sc, ra[:cs.total_slots], ga[:cs.total_slots]):
        h.update(memoryview(a))
    report(f"FULLSIZE {tag} m={m} k={k} candidates={cs.n} calls={cs.ncalls} "
           f"aligned={int((sc <= k).sum())} tsv_bytes={sum(n for _, n in res)} "
           f"sha256={h.hexdigest()[:16]} oracle: every candidate equal")


@pytest.mark.parametrize("name", ["c1", "c2", "c4", "c3"])
def test_full_size_config_matches_the_oracle(saru_lib, report, name):
    import torch
    torch.cuda.set_device(0)
    bench = load_bench()
    cfg = dict(bench.CONFIGS[name])
    css = bench.build_callsets(cfg, 0)
    assert sum(cs.n for cs in css) > 0
    for cs in css:
        align_and_check(cs, name, report)


def test_full_size_serving_request_matches_the_oracle(saru_lib, report):
    """The serving workload's largest request (500k reads, a quarter of
    them in each length bin) as a reads-only request through the server:
    every candidate of every call the server's filter made matches the
    oracle, and the calls equal the device filter's own."""
    import torch
    from saruman_b200 import workloads as W
    torch.cuda.set_device(0)
    bench = load_bench()
    cfg = dict(bench.CONFIGS["c5"])
    g, _ = bench.build_genome(cfg)
    sets = []
    for i, m in enumerate(cfg["lengths"]):
        rd = W.sample_reads(g, 125_000, m, cfg["rate"], seed=1000 + i, mix=cfg["mix"]).seqs
        sets.append((rd, W.k_for(m), 0))
    with S.Server(pipeline=True, budget_bytes=40 << 30) as srv:
        srv.set_genome(g)
        t = srv.submit_reads(sets)
        rc, _ = srv.wait(t, 1_800_000)
        assert rc == S.SARU_OK, S.last_error()
        res = [srv.read_results(t, i) for i in range(len(sets))]
        srv.release(t)
    for (rd, k, _), r in zip(sets, res):
        m = rd.shape[1]
        cs = W.callset(g, rd, m, k, r["ids"], r["pos"], r["dirs"], r["call_begin"],
                       r["call_strand"])
        np.testing.assert_array_equal(cs.sbase, r["slot_begin"])
        pad = np.zeros(64, np.uint8)
        align_and_check(cs, f"c5-request-m{m}", report,
                        outputs=(r["scores"], np.concatenate([r["read_aln"], pad]),
                                 np.concatenate([r["genome_aln"], pad])))
