"""Drop-in: the reference's own host program (src/saruman.c, src/hash.c,
src/util.c: FASTA input, q-gram index, SEASHORE filter, candidate
collection) linked against libsaruman_b200.so instead of its CUDA module
prints, sorted, exactly the lines of the reference program with its own
module (golden hash recorded by tests/golden/make_golden.py)."""
from __future__ import annotations

import gzip
import hashlib
import json
import subprocess
from pathlib import Path

import pytest

from saruman_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "oracle" / "_ref" / "saruman_dropin"
SPEC = ROOT / "tests" / "golden" / "dropin_c1small.json"


@pytest.mark.gpu
def test_reference_program_on_library(saru_lib, tmp_path):
    if not DROPIN.exists():
        objs = ROOT / "oracle" / "_ref" / "ref_hash.o"
        if not objs.exists():
            pytest.skip("reference host objects were not built (no reference sources)")
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "dropin"], check=True)
    spec = json.loads(SPEC.read_text())
    g = W.uniform_genome(spec["genome_len"], seed=spec["genome_seed"])
    rd = W.sample_reads(g, spec["reads"], spec["m"], spec["rate"], seed=spec["read_seed"])
    W.write_fasta_genome(str(tmp_path / "genome.fa"), g)
    W.write_fasta_reads(str(tmp_path / "reads.fa"), rd.seqs)
    cmd = [str(DROPIN), *spec["args"], "-g", str(tmp_path / "genome.fa"), "-r",
           str(tmp_path / "reads.fa")]
    r = subprocess.run(cmd, capture_output=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = sorted(r.stdout.splitlines(keepends=True))
    blob = b"".join(lines)
    if hashlib.sha256(blob).hexdigest() != spec["sha256_sorted_stdout"]:
        want = gzip.open(ROOT / "tests" / "golden" / "dropin_c1small.tsv.gz").read()
        wl = want.splitlines(keepends=True)
        diff = [x for x in lines if x not in set(wl)][:5]
        pytest.fail(f"{len(lines)} lines vs {len(wl)} expected; first unexpected: {diff}")
    assert b"starting CUDA kernel" in r.stderr
