"""CPU checks of the C ABI library: it loads, exports every symbol
include/saruman_b200.h declares, and its host TSV writer reproduces the
reference writer on the golden fixtures (host code only, no GPU call)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import golden_io as G
import saruman_b200 as S

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "saruman_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    funcs = set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text))
    funcs -= {"sizeof", "defined"}
    data = set(re.findall(r"extern\s+[a-z ]+\s+\**([a-z_][a-z0-9_]*)\s*\[", text))
    return funcs, data


def test_header_symbols_listed():
    funcs, data = declared_symbols()
    assert funcs == set(S.ABI_FUNCTIONS)
    assert data == set(S.ABI_DATA)


def test_library_exports_every_declared_symbol(saru_lib):
    funcs, data = declared_symbols()
    out = subprocess.run(["nm", "-D", "--defined-only", str(S.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = (funcs | data) - exported
    assert not missing, missing
    for name in funcs | data:
        assert hasattr(saru_lib, name)


def test_reference_globals_exported(saru_lib):
    """The reference's host program reads and writes these through the
    library (src/cuda-functions.h:15-28, src/saruman.h:55-66)."""
    for name in ("read_names", "read_length_value", "be_verbose_value", "use_gpu_value",
                 "cuda_memory_per_thread", "forward_alignments_done", "reverse_alignments_done",
                 "forward_alignment_candidates", "reverse_alignment_candidates",
                 "forward_output_control", "reverse_output_control", "main_alloc_ptr_for",
                 "main_alloc_ptr_rev"):
        C.c_int.in_dll(saru_lib, name)


@pytest.mark.parametrize("name", G.fixture_names())
def test_writer_matches_reference_writer(saru_lib, name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    r = S.AlignResult(exp["scores"].astype(np.int32), exp["read_aln"], exp["genome_aln"])
    tab = S.name_table(G.names_by_id(b, names))
    tsv, df, dr = S.format_tsv(b, r, tab, read_length=m)
    assert tsv == exp["tsv"]
    assert df + dr == int((exp["scores"] <= b.k).sum())


@pytest.mark.parametrize("seed,n", [(0, 3000), (1, 3000), (2, 3000), (3, 70000)])
def test_writer_matches_oracle_writer_on_irregular_slots(saru_lib, seed, n):
    """The writer's scans (leading gaps, the trailing gap/NUL run read
    backwards across slots, the forward gap count with its growing bound,
    the NUL-cut strings) against the oracle's byte-by-byte restatement of
    src/cuda-functions.cu:827-1006, on slots the aligner would not write:
    gap runs anywhere, NULs inside slots, all-gap and all-NUL slots.  70k
    candidates take several host threads (ordered ranges)."""
    import refkit as R
    from saruman_b200.workloads import Batch

    rng = np.random.default_rng(seed)
    m, k = 40, 4
    L = rng.integers(m - k, m + 2 * k + 1, n)
    go = np.cumsum(L).astype(np.int32)
    total = int(go[-1]) + k * n
    alphabet = np.frombuffer(b"ACGT_", np.uint8)
    ra = alphabet[rng.choice(5, total, p=[0.22, 0.22, 0.22, 0.22, 0.12])].copy()
    ga = alphabet[rng.choice(5, total, p=[0.22, 0.22, 0.22, 0.22, 0.12])].copy()
    for v in range(n):
        s0 = int(go[v - 1]) + k * v if v else 0
        s1 = s0 + int(L[v]) + k
        kind = rng.integers(0, 8)
        if kind == 0:
            ra[s0:s1] = ord("_")
        elif kind == 1:
            ra[s0:s1] = 0
        elif kind == 2:
            ra[s0 + rng.integers(0, s1 - s0):s1] = 0
            ga[s0 + rng.integers(0, s1 - s0):s1] = 0
        elif kind == 3:
            ra[s0:s0 + rng.integers(0, 12)] = ord("_")
            ra[s1 - rng.integers(0, 12):s1] = ord("_")
        elif kind == 4:
            ra[s1 - k:s1] = 0
            ga[s1 - k:s1] = 0
        elif kind == 5:
            ra[s0 + rng.integers(0, s1 - s0)] = 0
    b = Batch(m=m, k=k, genome=np.zeros(int(go[-1]), np.uint8), reads=np.zeros(n * m, np.uint8),
              genome_offsets=go, read_offsets=(np.arange(1, n + 1) * m).astype(np.int32),
              edit_offsets=np.zeros(n, np.int32),
              dirs=rng.choice(np.array([1, 2, 3, 5, 6, 7], np.int8), n),
              ids=rng.integers(0, 50, n).astype(np.int32),
              pos=rng.integers(0, 1 << 20, n).astype(np.int32))
    scores = rng.integers(0, k + 2, n).astype(np.int32)
    names = {i: f"read_{seed}_{i}".encode() for i in range(50)}
    tsv, df, dr = S.format_tsv(b, S.AlignResult(scores, ra, ga), S.name_table(names),
                               read_length=m)
    want, _, (wf, wr) = R.oracle_tsv(b, scores, ra, ga, R.name_table(names), read_length=m)
    assert tsv == want
    assert (df, dr) == (wf, wr)


def test_load_fails_loudly_without_library(tmp_path):
    with pytest.raises(RuntimeError, match="not built"):
        S.load(tmp_path / "missing.so")


def test_large_call_offsets_checked_before_any_copy(saru_lib):
    """A call large enough to be streamed in slices has the offsets at its
    slice edges checked before any copy is issued: each copy reads the
    caller's arrays between two edges.  Host code only: the check comes
    before the library looks for a device."""
    n, m, k = 600_000, 36, 2
    L = np.full(n, m + k, np.int64)
    go = np.cumsum(L).astype(np.int32)
    ro = (np.arange(1, n + 1) * m).astype(np.int32)
    dirs = np.ones(n, np.int8)
    genome = np.zeros(int(go[-1]), np.uint8)
    reads = np.zeros(int(ro[-1]), np.uint8)
    bad_go = go.copy()
    bad_go[(2 << 18) - 1] = go[(1 << 18) - 1] - 7  # the second slice edge before the first
    for offs, total, what in ((bad_go, int(go[-1]), "decrease"),
                              (go, int(go[-1]) - 1, "genome_bytes")):
        sb = S.SaruBatch(genome.ctypes.data, reads.ctypes.data, offs.ctypes.data, ro.ctypes.data,
                         dirs.ctypes.data, n, k, 0, 1, 1, m, total, int(go[-1]) + k * n)
        res = S.SaruResult(None, None, None, None)
        rc = saru_lib.saru_align_host(C.byref(sb), C.byref(res), 0)
        assert rc == S.SARU_E_INVALID
        assert what in S.last_error()


def test_compact_host_call_refuses_bad_record_sizes(saru_lib):
    """saru_align_host_compact checks its record size before any device work."""
    from saruman_b200 import workloads as W
    b = W.random_batch(36, 2, 10, seed=1)
    sb, keep = S.host_batch(b)
    sc = np.zeros(b.n, np.int32)
    rec = np.zeros(b.n * 64, np.uint8)
    for rb in (0, 8, 40):  # not a multiple of 16, or too small
        rc = saru_lib.saru_align_host_compact(C.byref(sb), sc.ctypes.data, rec.ctypes.data, rb, 0)
        assert rc == S.SARU_E_INVALID
