"""The input readers (saru_reads_*, saru_genome_*): the reference's read
batches and genome chunks.

* against the plain-Python restatement (oracle/input_oracle.py) on files
  made to hit the readers' edges: lines longer than the fgets buffers,
  CRLF line ends, lower case, Ns, short reads, empty names, a missing final
  newline, later header lines in the genome, chunks that end inside the
  read buffer or exactly at the end of the file;
* end to end against the reference program itself (oracle/_ref/
  saruman_emul): its sorted output on a genome read in three chunks, with
  FASTA and FASTQ reads that the reader must filter, equals what the
  readers, the host restatement of the filter (chunk offsets and window
  limit), the oracle aligner and the library's writer print.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import refkit as R
import saruman_b200 as S
from saruman_b200 import workloads as W
from test_filter_host import EMUL, harness

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import input_oracle as O  # noqa: E402


def reads_both(path: Path, m: int, max_n: int, batch: int, fastq: bool):
    ours = [(list(map(bytes, rb.reads)), rb.names, rb.records)
            for rb in S.read_batches(path, m, max_n, batch, fastq)]
    return ours, O.read_batches(path.read_bytes(), m, max_n, batch, fastq)


def genome_both(path: Path, chunk: int, m: int):
    ours = [(c.seq.tobytes(), c.bases, c.total) for c in S.genome_chunks(path, chunk, m)]
    return ours, O.genome_chunks(path.read_bytes(), chunk, m)


READ_FILES = {
    "plain": b">r0\nACGTACGTAC\n>r1\nacgtNNacgt\n>r2\nACGTNNNACG\n>r3\nACG\n>r4\nTTTTTTTTTT\n",
    "long_line": b">a\nACGTACGTACGTAC\n>b\nCCCCCCCCCC\n>c\nGGGGGGGGGG\n",
    "crlf": b">a\r\nACGTACGTAC\r\n>b\r\nCCCCCCCCCC\r\n>c\r\nGGGGGGGGGG\r\n",
    "long_name": b">" + b"n" * 70 + b"\nACGTACGTAC\n>b\nCCCCCCCCCC\n",
    "empty_name": b">\nACGTACGTAC\n\nCCCCCCCCCC\n>c\nGGGGGGGGGG",
    "no_final_newline": b">a\nACGTACGTAC\n>b\nCCCCCCCCCC",
    "name_without_read": b">a\nACGTACGTAC\n>b\n",
}


@pytest.mark.parametrize("name", sorted(READ_FILES))
@pytest.mark.parametrize("batch", [1, 2, 3, 100])
def test_read_batches_match_the_restatement(saru_lib, tmp_path, name, batch):
    p = tmp_path / "r.fa"
    p.write_bytes(READ_FILES[name])
    ours, want = reads_both(p, 10, 2, batch, False)
    assert ours == want


def test_fastq_batches_match_the_restatement(saru_lib, tmp_path):
    recs = []
    for i, s in enumerate([b"ACGTACGTAC", b"acgtnacgtn", b"ACG", b"NNNACGTACG", b"TTTTTTTTTT"]):
        recs.append(b"@q%d\n%s\n+q%d\n%s\n" % (i, s, i, b"I" * len(s)))
    p = tmp_path / "r.fq"
    p.write_bytes(b"".join(recs))
    for batch in (1, 2, 5, 10):
        ours, want = reads_both(p, 10, 2, batch, True)
        assert ours == want
    ours, _ = reads_both(p, 10, 2, 10, True)
    assert [r for b in ours for r in b[0]] == [b"ACGTACGTAC", b"ACGTNACGTN", b"TTTTTTTTTT"]
    assert [n for b in ours for n in b[1]] == [b"q0", b"q1", b"q4"]


def genome_text(seq: bytes, width: int, header: bytes = b">chr test", final_nl: bool = True):
    lines = [seq[i:i + width] for i in range(0, len(seq), width)]
    return header + b"\n" + b"\n".join(lines) + (b"\n" if final_nl else b"")


GENOME_CASES = {
    "lines70": (genome_text(b"ACGT" * 2000, 70), 1000, 36),
    "lines70_no_final_newline": (genome_text(b"ACGT" * 2000, 70, final_nl=False), 1000, 36),
    "one_line": (genome_text(b"ACGTTGCA" * 1000, 10_000), 1000, 36),  # chunks end inside the buffer
    "lower_and_n": (genome_text(b"acgtNNNNacgt" * 700, 60), 999, 20),
    "second_header": (genome_text(b"ACGT" * 500, 60) + b">second\n" +
                      genome_text(b"TTGG" * 500, 60, header=b"")[1:], 700, 30),
    "crlf": (b">g\r\n" + b"\r\n".join([b"ACGTACGTAC" * 6] * 60) + b"\r\n", 1000, 36),
    "exact_multiple": (genome_text(b"ACGT" * 750, 60), 1000, 36),
    "short": (genome_text(b"ACGT" * 10, 60), 1000, 36),
}


@pytest.mark.parametrize("name", sorted(GENOME_CASES))
def test_genome_chunks_match_the_restatement(saru_lib, tmp_path, name):
    data, chunk, m = GENOME_CASES[name]
    p = tmp_path / "g.fa"
    p.write_bytes(data)
    ours, want = genome_both(p, chunk, m)
    assert ours == want
    assert len(ours) >= 1


def test_genome_chunks_of_a_plain_file(saru_lib, tmp_path):
    """On an ordinary file (short lines, final newline) each chunk is the
    next chunk_value bases plus the following read_length bases."""
    g = W.uniform_genome(10_000, seed=3)
    p = tmp_path / "g.fa"
    p.write_bytes(genome_text(g.tobytes(), 60))
    chunks = list(S.genome_chunks(p, 3000, 36))
    assert [c.offset for c in chunks] == [0, 3000, 6000, 9000]
    for c in chunks:
        want = g[c.offset:c.offset + 3000 + 36].tobytes()
        assert c.seq.tobytes() == want
        assert c.total == min(c.offset + 3000, 10_000)


# ---------------------------------------------------------------------------
# end to end against the reference program


def write_reads(path: Path, seqs: np.ndarray, fastq: bool, rng) -> None:
    """Reads with what the reader has to deal with: lower case, Ns (some
    reads with more than the error count), short reads."""
    out = []
    for i, s in enumerate(seqs):
        b = bytearray(s.tobytes())
        r = rng.random()
        if r < 0.05:
            b = b.lower()
        elif r < 0.10:
            b[int(rng.integers(len(b)))] = ord("N")
        elif r < 0.13:
            for j in rng.choice(len(b), 3, replace=False):
                b[int(j)] = ord("N")
        elif r < 0.15:
            b = b[:len(b) - 5]
        name = b"read_%d" % i
        if fastq:
            out.append(b"@%s\n%s\n+\n%s\n" % (name, bytes(b), b"I" * len(b)))
        else:
            out.append(b">%s\n%s\n" % (name, bytes(b)))
    path.write_bytes(b"".join(out))


def map_on_cpu(genome_path: Path, reads_path: Path, m: int, k: int, fastq: bool, nread: int,
               chunk_value: int, gchunk: int) -> list[bytes]:
    """The reference program's output lines, made from the readers, the
    host restatement of the filter, the oracle aligner and the writer."""
    lib = harness()
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    lines = []
    for ch in S.genome_chunks(genome_path, gchunk, m):
        g = ch.seq
        for rb in S.read_batches(reads_path, m, k, nread, fastq):
            reads = rb.reads
            n = reads.shape[0]
            tab = S.name_table(rb.names)
            flat = np.ascontiguousarray(reads.reshape(-1))
            for dr, arrow in ((0, b">>"), (4, b"<<")):
                cb = np.zeros(1 << 12, np.int64)
                ids = np.zeros(1 << 20, np.int32)
                pos = np.zeros_like(ids)
                dirs = np.zeros(1 << 20, np.int8)
                pids = np.zeros(1 << 18, np.int32)
                ppos = np.zeros_like(pids)
                cnt = np.zeros(3, np.int64)
                rc = lib.filter_host_calls_chunk(
                    P(g), C.c_long(len(g)), C.c_long(ch.offset), C.c_long(ch.total), P(flat), n,
                    m, k, dr, chunk_value, C.c_uint(chunk_value), 4096, P(cb), C.c_int64(len(cb)),
                    P(ids), P(pos), P(dirs), C.c_int64(len(ids)), P(pids), P(ppos),
                    C.c_int64(len(pids)), P(cnt))
                assert rc == 0
                nc, na, npf = (int(x) for x in cnt)
                calls = S.FilterCalls(cb[:nc + 1], ids[:na], pos[:na], dirs[:na], pids[:npf],
                                      ppos[:npf], 0.0)
                for c in range(nc):
                    b = calls.call(g, reads, m, k, c, offset=ch.offset)
                    sc, ra, ga, _ = R.oracle_align(b)
                    text, _, _ = S.format_tsv(b, S.AlignResult(sc, ra, ga), tab, read_length=m)
                    lines += text.splitlines(keepends=True)
                for rid, g1 in zip(calls.perfect_ids, calls.perfect_pos):
                    rd = reads[rid]
                    if dr == 4:
                        rd = W.reverse_complement(rd[None])[0]
                    at = int(g1) - ch.offset
                    lines.append(b"%s\t%d\t%d\t%s\t%s\t%s\t0\n" % (
                        rb.names[rid], g1, g1 - 1 + m, arrow, g[at:at + m].tobytes(),
                        rd.tobytes()))
    return lines


@pytest.mark.skipif(not EMUL.exists(), reason="the reference's host build is not here")
@pytest.mark.parametrize("fastq,m,k", [(False, 36, 2), (True, 36, 2), (False, 75, 4), (True, 100, 5)])
def test_chunked_mapping_prints_the_reference_output(saru_lib, tmp_path, fastq, m, k):
    rng = np.random.default_rng(11 + fastq + m)
    g = W.uniform_genome(60_000, seed=12)
    text = bytearray(g.tobytes())
    text[5000:5400] = bytes(text[5000:5400]).lower()
    text[20000:20030] = b"N" * 30
    (tmp_path / "genome.fa").write_bytes(genome_text(bytes(text), 70, final_nl=False))
    rd = W.sample_reads(g, 1300, m, 0.02 if m < 50 else 0.03, seed=13).seqs
    write_reads(tmp_path / "reads.fa", rd, fastq, rng)
    nread, chunk_value, gchunk = 700, 900, 25_000  # 2 read batches, 3 genome chunks
    args = [str(EMUL), "-m", "0", "-i", "1", "-l", str(m), "-e", repr((k + 0.5) / m),
            "-c", str(nread), "-s", str(chunk_value), "-g", str(tmp_path / "genome.fa"),
            "-r", str(tmp_path / "reads.fa"), "-G", str(gchunk)] + (["-q"] if fastq else [])
    env = dict(os.environ, SARU_EMUL_FREE_MB="4096")
    ref = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env,
                         check=True, timeout=600).stdout
    want = sorted(ref.splitlines(keepends=True))
    got = sorted(map_on_cpu(tmp_path / "genome.fa", tmp_path / "reads.fa", m, k, fastq, nread,
                            chunk_value, gchunk))
    assert len(want) > 1000
    assert len(got) == len(want)
    assert hashlib.sha256(b"".join(got)).hexdigest() == hashlib.sha256(b"".join(want)).hexdigest()


def test_readers_refuse_bad_arguments(saru_lib, tmp_path):
    with pytest.raises(S.SaruError):
        list(S.read_batches(tmp_path / "missing.fa", 36, 2, 100))
    with pytest.raises(S.SaruError):
        list(S.genome_chunks(tmp_path / "missing.fa", 1000, 36))
    p = tmp_path / "g.fa"
    p.write_bytes(genome_text(b"ACGT" * 100, 60))
    with pytest.raises(S.SaruError):
        list(S.genome_chunks(p, 0, 36))
    with pytest.raises(S.SaruError):
        list(S.read_batches(p, 0, 2, 100))
