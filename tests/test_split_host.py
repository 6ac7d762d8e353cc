"""The host entry point splits a large banded call into slices of whole
32-candidate tiles whose copies in, kernels and copies out overlap on three
streams.  Its output must be the bytes one launch over the whole call gives:
here a 660k-candidate C2-shaped call (three slices, the last one partial)
through saru_align_host against the same call through saru_align_device in
a single launch."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

import saruman_b200 as S

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_split", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_split"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_split_host_call_equals_one_launch(saru_lib):
    import torch
    bench = load_bench()
    cfg = dict(bench.CONFIGS["c2"])
    cfg["reads"] = 70_000
    b = bench.build_batches(cfg, 0)[0]
    assert 2 * (1 << 18) <= b.n < 3 * (1 << 18) and b.n % 32 != 0
    host = S.align_host(b)
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    g, r, go, ro, d = T(b.genome), T(b.reads), T(b.genome_offsets), T(b.read_offsets), T(b.dirs)
    sc = torch.zeros(b.n, dtype=torch.int32, device=dev)
    ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    sb = S.SaruBatch(g.data_ptr(), r.data_ptr(), go.data_ptr(), ro.data_ptr(), d.data_ptr(), b.n,
                     b.k, 0, 1, 1, b.m, len(b.genome), b.total_genome)
    sr = S.SaruResult(sc.data_ptr(), ra.data_ptr(), ga.data_ptr(), st.data_ptr())
    nscr = S.scratch_bytes(b.n, b.m, b.k)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    S.align_device(sb, sr, scr.data_ptr(), nscr)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert np.array_equal(host.scores, sc.cpu().numpy())
    assert np.array_equal(host.read_aln, ra.cpu().numpy()[:b.total_genome])
    assert np.array_equal(host.genome_aln, ga.cpu().numpy()[:b.total_genome])
    assert (host.scores <= b.k).sum() > b.n // 4



def test_compact_host_call_expands_to_the_slot_strings(saru_lib):
    """saru_align_host_compact over the same sliced call: its records,
    expanded on the host, are the slot strings saru_align_host returns."""
    bench = load_bench()
    cfg = dict(bench.CONFIGS["c2"])
    cfg["reads"] = 70_000
    b = bench.build_batches(cfg, 0)[0]
    slots = S.align_host(b)
    sc, rec, rb = S.align_host_compact(b)
    comp = S.expand_compact(b, sc, rec, rb)
    assert np.array_equal(comp.scores, slots.scores)
    assert np.array_equal(comp.read_aln, slots.read_aln)
    assert np.array_equal(comp.genome_aln, slots.genome_aln)


def test_compact_host_call_on_the_exact_path(saru_lib):
    """A call the banded kernel hands to the exact path (a read with five
    distinct non-ACGT bytes) still comes back as records."""
    from saruman_b200 import workloads as W
    b = W.random_batch(100, 5, 3000, seed=21, err=0.03)
    b.reads[100 * 7:100 * 7 + 5] = np.frombuffer(b"NRYKM", np.uint8)
    slots = S.align_host(b)
    sc, rec, rb = S.align_host_compact(b)
    comp = S.expand_compact(b, sc, rec, rb)
    assert np.array_equal(comp.scores, slots.scores)
    assert np.array_equal(comp.read_aln, slots.read_aln)
    assert np.array_equal(comp.genome_aln, slots.genome_aln)
    assert (slots.scores <= 5).sum() > 100


def test_split_host_call_with_64_bit_bands(saru_lib):
    """A sliced call at k = 9 (150 bp): each slice chooses its own band word
    (64 bits where it has start gaps); slot strings and compact records
    equal one launch over the whole call."""
    import torch
    bench = load_bench()
    cfg = dict(bench.CONFIGS["c2"], m=150, k=9, reads=60_000)
    b = bench.build_batches(cfg, 0)[0]
    assert b.n >= 2 * (1 << 18) and b.k == 9
    host = S.align_host(b)
    sc, rec, rb = S.align_host_compact(b)
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    g, r, go, ro, d = T(b.genome), T(b.reads), T(b.genome_offsets), T(b.read_offsets), T(b.dirs)
    dsc = torch.zeros(b.n, dtype=torch.int32, device=dev)
    ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    sb = S.SaruBatch(g.data_ptr(), r.data_ptr(), go.data_ptr(), ro.data_ptr(), d.data_ptr(), b.n,
                     b.k, 0, 1, 1, b.m, len(b.genome), b.total_genome)
    sr = S.SaruResult(dsc.data_ptr(), ra.data_ptr(), ga.data_ptr(), st.data_ptr())
    nscr = S.scratch_bytes(b.n, b.m, b.k)
    scr = torch.empty(nscr, dtype=torch.uint8, device=dev)
    S.align_device(sb, sr, scr.data_ptr(), nscr)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert np.array_equal(host.scores, dsc.cpu().numpy())
    assert np.array_equal(host.read_aln, ra.cpu().numpy()[:b.total_genome])
    assert np.array_equal(host.genome_aln, ga.cpu().numpy()[:b.total_genome])
    comp = S.expand_compact(b, sc, rec, rb)
    assert np.array_equal(comp.read_aln, host.read_aln)
    assert np.array_equal(comp.genome_aln, host.genome_aln)
