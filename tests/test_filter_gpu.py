"""The q-gram pair filter on the device (saru_filter_*): the calls it
assembles equal the reference program's own calls (committed golden calls,
read batches and data-array chunks included), and the whole mapping on the
GPU -- device filter, windows, banded alignment, the writer, and the
filter's perfect-hit lines -- prints exactly the reference program's
output on the drop-in dataset (SHA-256 of the sorted lines)."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import saruman_b200 as S
from saruman_b200 import workloads as W
from test_filter_host import golden_inputs, load_golden

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("name", ["f36k2", "f100k5", "f150k9", "f36k3"])
def test_device_filter_matches_the_golden_calls(saru_lib, name):
    z, specs = load_golden()
    spec = specs[name]
    _, _, nreads, m, k, _, chunk, rchunk = spec
    g, reads = golden_inputs(spec)
    with S.Filter(g, m, k) as f:
        for dr, strand in ((0, "fwd"), (4, "rev")):
            cbs, ids, pos, dirs = [np.zeros(1, np.int64)], [], [], []
            for b0 in range(0, nreads, rchunk):
                out = f.run(reads[b0:b0 + rchunk], dr, chunk)
                cbs.append(out.call_begin[1:] + cbs[-1][-1])
                ids.append(out.ids)
                pos.append(out.pos)
                dirs.append(out.dirs)
            assert np.array_equal(np.concatenate(cbs), z[f"{name}_{strand}_call_begin"])
            assert np.array_equal(np.concatenate(ids), z[f"{name}_{strand}_ids"])
            assert np.array_equal(np.concatenate(pos), z[f"{name}_{strand}_pos"])
            assert np.array_equal(np.concatenate(dirs), z[f"{name}_{strand}_dirs"])


def map_on_gpu(g, reads, m, k, chunk_value):
    """Every line the reference program would print for one read batch."""
    names = [b"r%d" % i for i in range(reads.shape[0])]
    tab = S.name_table(names)
    lines = []
    with S.Filter(g, m, k) as f:
        for dr, arrow in ((0, b">>"), (4, b"<<")):
            out = f.run(reads, dr, chunk_value)
            for c in range(len(out.call_begin) - 1):
                b = out.call(g, reads, m, k, c)
                r = S.align_host(b)
                text, _, _ = S.format_tsv(b, r, tab, read_length=m)
                lines += text.splitlines(keepends=True)
            for rid, g1 in zip(out.perfect_ids, out.perfect_pos):
                rd = reads[rid]
                if dr == 4:
                    rd = W.reverse_complement(rd[None])[0]
                lines.append(b"%s\t%d\t%d\t%s\t%s\t%s\t0\n" % (
                    names[rid], g1, g1 - 1 + m, arrow, g[g1:g1 + m].tobytes(), rd.tobytes()))
    return lines


def test_mapping_on_the_gpu_prints_the_reference_output(saru_lib):
    spec = json.loads((ROOT / "tests" / "golden" / "dropin_c1small.json").read_text())
    g = W.uniform_genome(spec["genome_len"], seed=spec["genome_seed"])
    reads = W.sample_reads(g, spec["reads"], spec["m"], spec["rate"], seed=spec["read_seed"]).seqs
    k = int(np.floor(spec["m"] * spec["e"]))
    chunk_value = int(spec["args"][spec["args"].index("-s") + 1])
    lines = sorted(map_on_gpu(g, reads, spec["m"], k, chunk_value))
    assert len(lines) == spec["lines"]
    assert hashlib.sha256(b"".join(lines)).hexdigest() == spec["sha256_sorted_stdout"]


def test_filter_rejects_bad_arguments(saru_lib):
    g = W.uniform_genome(10_000, seed=1)
    with pytest.raises(S.SaruError):
        S.Filter(g, 1, 2)
    with S.Filter(g, 36, 2) as f:
        with pytest.raises(S.SaruError):
            f.run(np.zeros((4, 36), np.uint8) + ord("A"), 1, 100)


def map_chunked_on_gpu(genome_path, reads_path, m, k, fastq, nread, chunk_value, gchunk):
    """map_on_gpu over the reference's genome chunks and read batches (the
    input readers), each chunk's filter told its offset and window limit."""
    lines = []
    for ch in S.genome_chunks(genome_path, gchunk, m):
        g = ch.seq
        with S.Filter(g, m, k) as f:
            f.set_chunk(ch.offset, ch.total)
            for rb in S.read_batches(reads_path, m, k, nread, fastq):
                reads = rb.reads
                tab = S.name_table(rb.names)
                for dr, arrow in ((0, b">>"), (4, b"<<")):
                    out = f.run(reads, dr, chunk_value)
                    for c in range(len(out.call_begin) - 1):
                        b = out.call(g, reads, m, k, c, offset=ch.offset)
                        r = S.align_host(b)
                        text, _, _ = S.format_tsv(b, r, tab, read_length=m)
                        lines += text.splitlines(keepends=True)
                    for rid, g1 in zip(out.perfect_ids, out.perfect_pos):
                        rd = reads[rid]
                        if dr == 4:
                            rd = W.reverse_complement(rd[None])[0]
                        at = int(g1) - ch.offset
                        lines.append(b"%s\t%d\t%d\t%s\t%s\t%s\t0\n" % (
                            rb.names[rid], g1, g1 - 1 + m, arrow, g[at:at + m].tobytes(),
                            rd.tobytes()))
    return lines


@pytest.mark.parametrize("fastq", [False, True])
def test_chunked_mapping_on_the_gpu_equals_the_host_pipeline(saru_lib, tmp_path, fastq):
    """The genome in three chunks and the reads in two batches through the
    input readers, the device filter and the banded kernel print what the
    host pipeline prints (the host pipeline equals the reference program's
    output: tests/test_input.py)."""
    import test_input as T
    m, k = 36, 2
    rng = np.random.default_rng(11 + fastq)
    g = W.uniform_genome(60_000, seed=12)
    text = bytearray(g.tobytes())
    text[5000:5400] = bytes(text[5000:5400]).lower()
    text[20000:20030] = b"N" * 30
    (tmp_path / "genome.fa").write_bytes(T.genome_text(bytes(text), 70, final_nl=False))
    rd = W.sample_reads(g, 1300, m, 0.02, seed=13).seqs
    T.write_reads(tmp_path / "reads.fa", rd, fastq, rng)
    args = (tmp_path / "genome.fa", tmp_path / "reads.fa", m, k, fastq, 700, 900, 25_000)
    got = sorted(map_chunked_on_gpu(*args))
    want = sorted(T.map_on_cpu(*args))
    assert len(got) > 1000
    assert got == want
