"""The benchmark's full C2 step (2M reads x 100 bp, 18.95M candidates),
checked at that size by properties that do not need the oracle on every
candidate: the slot strings of the host entry point (slot mode) equal, byte
for byte over all candidates, the compact records of the device entry point
expanded on the host (two independent output paths); every slot is its
string followed by zeros; a read string without its gaps is a suffix of
the read; and a sample of candidates matches the oracle."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

import refkit as R
import saruman_b200 as S
from nwbio import sub_batch

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_mod"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_full_c2_step(saru_lib):
    import torch
    bench = load_bench()
    b = bench.build_batches(dict(bench.CONFIGS["c2"]), 0)[0]
    assert b.n > 18_000_000
    slot = S.align_host(b)
    # the compact path on the device, expanded on the host
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    g, r, go, ro, d = T(b.genome), T(b.reads), T(b.genome_offsets), T(b.read_offsets), T(b.dirs)
    rb = S.compact_record_bytes(b.m, b.k)
    sc = torch.zeros(b.n, dtype=torch.int32, device=dev)
    rec = torch.empty(b.n * rb, dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    sb = S.SaruBatch(g.data_ptr(), r.data_ptr(), go.data_ptr(), ro.data_ptr(), d.data_ptr(), b.n,
                     b.k, 0, 1, 1, b.m, len(b.genome), b.total_genome)
    nscr = S.scratch_bytes(b.n, b.m, b.k)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    S.align_device_compact(sb, sc.data_ptr(), rec.data_ptr(), rb, st.data_ptr(), scr.data_ptr(),
                           nscr)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    del g, r, go, ro, d, scr
    comp = S.expand_compact(b, sc.cpu().numpy(), rec.cpu().numpy(), rb)
    del rec
    assert np.array_equal(comp.scores, slot.scores)
    assert np.array_equal(comp.read_aln, slot.read_aln)
    assert np.array_equal(comp.genome_aln, slot.genome_aln)
    k = b.k
    ok = slot.scores <= k
    assert 0.3 < ok.mean() < 1.0
    # every slot: its string, then zeros; unreported candidates all zeros
    ss = b.slot_starts()
    cap = b.lengths.astype(np.int64) + k
    rng = np.random.default_rng(1)
    reads = b.reads.reshape(-1, b.m)
    for i in rng.choice(b.n, 20_000, replace=False):
        lo, hi = int(ss[i]), int(ss[i] + cap[i])
        s = slot.read_aln[lo:hi]
        gsl = slot.genome_aln[lo:hi]
        nz = np.flatnonzero(s == 0)
        n = int(nz[0]) if nz.size else hi - lo
        assert not s[n:].any() and not gsl[n:].any()
        if not ok[i]:
            assert n == 0
        if ok[i]:
            letters = s[:n][s[:n] != ord("_")].tobytes()
            assert reads[i].tobytes().endswith(letters)
    # a sample against the oracle (each candidate behind its predecessor)
    for i in rng.choice(np.arange(1, b.n), 300, replace=False):
        pair, _ = sub_batch(b, [b""] * b.n, int(i) - 1, 2)
        s1, ra1, ga1, _ = R.oracle_align(pair)
        assert int(slot.scores[i]) == min(int(s1[1]), k + 1)
        lo, hi = int(ss[i]), int(ss[i] + cap[i])
        o = int(pair.slot_starts()[1])
        assert np.array_equal(slot.read_aln[lo:hi], ra1[o:o + hi - lo])
        assert np.array_equal(slot.genome_aln[lo:hi], ga1[o:o + hi - lo])
