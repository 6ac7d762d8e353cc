"""Host side of the compact result format, on the CPU: records built from
the reference's own slots (golden fixtures) expand back to those slots, and
the TSV writer that reads records directly prints the reference's lines,
for several thread counts (so the chunk edges fall in different places)."""
from __future__ import annotations

import numpy as np
import pytest

import golden_io as G
import saruman_b200 as S


def records_from_slots(b, scores, ra, ga):
    """Compact records of a call from its slot strings: the string's columns
    in reverse order, '_' in the read an UP step, '_' in the window a LEFT
    step, otherwise DIAG."""
    rb = S.compact_record_bytes(b.m, b.k)
    rec = np.zeros((b.n, rb // 4), np.uint32)
    ss = b.slot_starts()
    cap = b.lengths.astype(np.int64) + b.k
    for t in range(b.n):
        if scores[t] > b.k:
            continue
        s = ra[ss[t]:ss[t] + cap[t]]
        g = ga[ss[t]:ss[t] + cap[t]]
        nz = np.flatnonzero(s == 0)
        n = int(nz[0]) if nz.size else int(cap[t])
        ops = np.where(s[:n] == ord("_"), 2, np.where(g[:n] == ord("_"), 3, 1))[::-1]
        for st, op in enumerate(ops):
            rec[t, 1 + st // 16] |= np.uint32(int(op) << (2 * (st % 16)))
        rec[t, 0] = n
    return rec.view(np.uint8).reshape(-1), rb


@pytest.mark.parametrize("name", G.fixture_names())
def test_compact_host_writer_prints_the_reference_tsv(saru_lib, name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    if b.m > 512 or b.k > 15:
        pytest.skip("records are sized for the banded kernel's domain")
    sc = np.asarray(exp["scores"], np.int32)
    rec, rb = records_from_slots(b, sc, exp["read_aln"], exp["genome_aln"])
    out = S.expand_compact(b, sc, rec, rb, nthreads=3)
    assert np.array_equal(out.read_aln, exp["read_aln"])
    assert np.array_equal(out.genome_aln, exp["genome_aln"])
    tab = S.name_table(G.names_by_id(b, names))
    for nt in (1, 3, 16):
        text, df, dr = S.format_tsv_compact(b, sc, rec, rb, tab, read_length=m, nthreads=nt)
        assert text == exp["tsv"], nt
        assert df + dr == int((sc <= b.k).sum())


def random_walk_records(b, rng, p_full=0.2, p_noletter=0.1):
    """Records of random valid walks from (L, m): some fill their slot
    exactly (no NUL: the writer's scans run into the next slot), some are
    all gaps in the read (no read byte: its backward scan runs into the
    previous slots); scores mark every third candidate unreported."""
    rb = S.compact_record_bytes(b.m, b.k)
    rec = np.zeros((b.n, rb // 4), np.uint32)
    sc = np.zeros(b.n, np.int32)
    for t in range(b.n):
        L, m, k = int(b.lengths[t]), b.m, b.k
        cap = L + k
        if t % 3 == 2:
            sc[t] = k + 1
            continue
        u = rng.random()
        ops = []
        row, col = L, m
        if u < p_noletter:
            n = int(rng.integers(1, L + 1))
            ops = [2] * n
        else:
            # a full slot: a walk of cap steps, mostly gaps so it cannot run out
            n = cap if u < p_noletter + p_full else int(rng.integers(1, cap + 1))
            while len(ops) < n:
                choices = [op for op, ok in ((1, row > 0 and col > 0), (2, row > 0), (3, col > 0))
                           if ok]
                if not choices:  # the walk reached (0, 0)
                    break
                op = choices[int(rng.integers(len(choices)))]
                if len(ops) < n - 1 and rng.random() < 0.7 and row > 0 and col > 0:
                    op = 1
                ops.append(op)
                row -= op in (1, 2)
                col -= op in (1, 3)
        for st, op in enumerate(ops):
            rec[t, 1 + st // 16] |= np.uint32(op << (2 * (st % 16)))
        rec[t, 0] = len(ops)
        sc[t] = int(rng.integers(0, k + 1))
    return rec.view(np.uint8).reshape(-1), rb, sc


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_compact_writer_chunk_edges(saru_lib, seed):
    """For any valid records the direct writer equals the slot writer run on
    the expanded slots, whatever the chunking."""
    from saruman_b200 import workloads as W
    rng = np.random.default_rng(seed)
    b = W.random_batch(40, 3, 1200, seed=seed + 30, err=0.05, alphabet=b"ACGTN")
    rec, rb, sc = random_walk_records(b, rng)
    slots = S.expand_compact(b, sc, rec, rb, nthreads=1)
    tab = S.name_table([b"r%d" % i for i in range(int(b.ids.max()) + 1)])
    want, f0, r0 = S.format_tsv(b, slots, tab)
    for nt in (1, 2, 5, 17):
        text, f1, r1 = S.format_tsv_compact(b, sc, rec, rb, tab, nthreads=nt)
        assert text == want and (f1, r1) == (f0, r0), nt
