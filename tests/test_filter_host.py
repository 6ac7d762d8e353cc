"""The q-gram pair filter restated for the GPU (saruman_b200/csrc/
filter_core.cuh, with the call assembly of filter_calls.h), run on the CPU
with the reference's own data layout, against the calls the reference
program itself submits on the same genome and reads (its host build with
call capture, oracle/_ref/saruman_emul): every call's read ids, positions
and flags and the call boundaries, both strands, several read lengths, k,
repeat-rich genomes and queue thresholds small enough to split the work
into hundreds of calls."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import nwbio
from saruman_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "harness" / "filter_host.cpp"
SO = ROOT / "tests" / "_build" / "libfilter_host.so"
EMUL = ROOT / "oracle" / "_ref" / "saruman_emul"


def harness():
    SO.parent.mkdir(exist_ok=True)
    deps = [SRC, ROOT / "saruman_b200" / "csrc" / "filter_core.cuh",
            ROOT / "saruman_b200" / "csrc" / "filter_calls.h"]
    if not SO.exists() or SO.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(SO), str(SRC)],
                       check=True)
    return C.CDLL(str(SO))


def reference_calls(tmp: Path, g, reads, m, k, chunk_value):
    """The reference program's calls per strand, as captured batches."""
    W.write_fasta_genome(str(tmp / "genome.fa"), g)
    W.write_fasta_reads(str(tmp / "reads.fa"), reads)
    cap = tmp / "cap"
    cap.mkdir()
    env = dict(os.environ, SARU_CAPTURE_DIR=str(cap), SARU_EMUL_FREE_MB="4096")
    n = reads.shape[0]
    subprocess.run([str(EMUL), "-m", "0", "-i", "1", "-l", str(m), "-e", repr((k + 0.5) / m),
                    "-c", str(n + 1), "-s", str(chunk_value), "-g", str(tmp / "genome.fa"),
                    "-r", str(tmp / "reads.fa"), "-G", "100000000"],
                   stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env, check=True)
    return {s: [nwbio.read_nwb(f)[0] for f in sorted(cap.glob(f"batch_{s}_*.nwb"))]
            for s in ("fwd", "rev")}


def host_calls(lib, g, reads, m, k, dr, chunk_value):
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    n = reads.shape[0]
    cb = np.zeros(1 << 16, np.int64)
    ids = np.zeros(1 << 22, np.int32)
    pos = np.zeros_like(ids)
    dirs = np.zeros(1 << 22, np.int8)
    pids = np.zeros(1 << 20, np.int32)
    ppos = np.zeros_like(pids)
    cnt = np.zeros(3, np.int64)
    flat = np.ascontiguousarray(reads.reshape(-1))
    rc = lib.filter_host_calls(P(g), C.c_long(len(g)), P(flat), n, m, k, dr, chunk_value,
                               C.c_uint(chunk_value), 4096, P(cb), C.c_int64(len(cb)), P(ids),
                               P(pos), P(dirs), C.c_int64(len(ids)), P(pids), P(ppos),
                               C.c_int64(len(pids)), P(cnt))
    assert rc == 0
    nc, na = int(cnt[0]), int(cnt[1])
    return cb[:nc + 1], ids[:na], pos[:na], dirs[:na]


@pytest.mark.skipif(not EMUL.exists(), reason="the reference's host build is not here")
@pytest.mark.parametrize("m,k,nreads,glen,kind,chunk", [
    (36, 2, 1500, 100_000, "uniform", 6_000),
    (100, 5, 150, 200_000, "repeat", 300),
    (75, 5, 200, 200_000, "repeat", 150),
    (150, 9, 120, 200_000, "repeat", 250),
    (250, 15, 200, 150_000, "uniform", 40),
    (36, 3, 400, 200_000, "repeat", 97)])
def test_filter_calls_match_the_reference_program(tmp_path, m, k, nreads, glen, kind, chunk):
    seed = m * 31 + k
    g = (W.uniform_genome(glen, seed=seed) if kind == "uniform"
         else W.repeat_genome(glen, seed=seed, copies="zipf"))
    rd = W.sample_reads(g, nreads, m, 0.03, seed=seed + 1)
    ref = reference_calls(tmp_path, g, rd.seqs, m, k, chunk)
    lib = harness()
    for dr, strand in ((0, "fwd"), (4, "rev")):
        cb, ids, pos, dirs = host_calls(lib, g, rd.seqs, m, k, dr, chunk)
        assert len(cb) - 1 == len(ref[strand])
        for c, b in enumerate(ref[strand]):
            lo, hi = int(cb[c]), int(cb[c + 1])
            assert hi - lo == b.n
            assert np.array_equal(ids[lo:hi], b.ids)
            assert np.array_equal(pos[lo:hi], b.pos)
            assert np.array_equal(dirs[lo:hi], b.dirs)


def load_golden():
    import json
    z = np.load(ROOT / "tests" / "golden" / "filter_calls.npz")
    specs = json.loads(bytes(z["specs"]).decode())
    return z, specs


def golden_inputs(spec):
    name, (kind, glen, gseed), nreads, m, k, rseed, chunk, rchunk = spec
    g = (W.uniform_genome(glen, seed=gseed) if kind == "uniform"
         else W.repeat_genome(glen, seed=gseed, copies="zipf"))
    return g, W.sample_reads(g, nreads, m, 0.03, seed=rseed).seqs


@pytest.mark.parametrize("name", ["f36k2", "f100k5", "f150k9", "f36k3"])
def test_filter_calls_match_the_golden_calls(name):
    """Against the committed calls of the reference program (read batches of
    64 in f150k9, hundreds of calls in f36k3), no reference build needed.
    The reference maps its reads one batch (-c) at a time, read ids from 0
    in each batch, and chunks its data array by the queue threshold (-s)."""
    z, specs = load_golden()
    spec = specs[name]
    _, _, nreads, m, k, _, chunk, rchunk = spec
    g, reads = golden_inputs(spec)
    lib = harness()
    for dr, strand in ((0, "fwd"), (4, "rev")):
        cbs, idss, poss, dirss = [np.zeros(1, np.int64)], [], [], []
        for b0 in range(0, nreads, rchunk):
            cb, ids, pos, dirs = host_calls(lib, g, reads[b0:b0 + rchunk], m, k, dr, chunk)
            cbs.append(cb[1:] + cbs[-1][-1])
            idss.append(ids)
            poss.append(pos)
            dirss.append(dirs)
        assert np.array_equal(np.concatenate(cbs), z[f"{name}_{strand}_call_begin"])
        assert np.array_equal(np.concatenate(idss), z[f"{name}_{strand}_ids"])
        assert np.array_equal(np.concatenate(poss), z[f"{name}_{strand}_pos"])
        assert np.array_equal(np.concatenate(dirss), z[f"{name}_{strand}_dirs"])
