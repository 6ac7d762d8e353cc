"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run here, where the reference sources are available (it needs the oracle
build of the reference, `make -C oracle`):

    python tests/golden/make_golden.py

For each configuration shape it writes seeded synthetic FASTA files, runs
the reference program (src/saruman.c with its own q-gram filter and
candidate collection, GPU module emulated on the host) with batch capture
on, and keeps the first candidates of the forward and reverse batches as a
new call (<name>_<strand>.nwb.gz) together with what the reference kernel
and writer produce for it (<name>_<strand>.out.npz: scores, both slot
arrays, TSV bytes).  It also records the SHA-256 of the reference program's
sorted stdout on a small end-to-end dataset (dropin_c1small.json) for the
drop-in test.  No reference source is copied; only its outputs are kept.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from saruman_b200 import workloads as W  # noqa: E402
import nwbio  # noqa: E402
import refkit  # noqa: E402

EMUL = ROOT / "oracle" / "_ref" / "saruman_emul"

# name, genome spec, reads, m, error rate, mix, unmapped, -e value, keep
CONFIGS = [
    ("c1_m36k2", ("uniform", 1_000_000, 101), 40_000, 36, 0.02, (0.70, 0.15, 0.15), 0.0, 0.06, 1500),
    ("c2_m100k5", ("repeat", 5_000_000, 201, "uniform"), 20_000, 100, 0.03, (0.70, 0.15, 0.15), 0.0,
     0.055, 1500),
    ("c3_m36k3", ("repeat", 5_000_000, 301, "zipf"), 20_000, 36, 0.03, (0.70, 0.15, 0.15), 0.0,
     3.5 / 36, 1500),
    ("c3_m75k5", ("repeat", 5_000_000, 301, "zipf"), 15_000, 75, 0.03, (0.70, 0.15, 0.15), 0.0,
     5.5 / 75, 1200),
    ("c3_m100k6", ("repeat", 5_000_000, 301, "zipf"), 12_000, 100, 0.03, (0.70, 0.15, 0.15), 0.0,
     6.5 / 100, 1000),
    ("c3_m150k9", ("repeat", 5_000_000, 301, "zipf"), 8_000, 150, 0.03, (0.70, 0.15, 0.15), 0.0,
     9.5 / 150, 700),
    ("c4_m250k15", ("uniform", 2_000_000, 401), 4_000, 250, 0.04, (0.60, 0.20, 0.20), 0.05,
     15.5 / 250, 500),
]


def genome_for(spec):
    if spec[0] == "uniform":
        return W.uniform_genome(spec[1], seed=spec[2])
    return W.repeat_genome(spec[1], seed=spec[2], copies=spec[3])


def run_reference(workdir: Path, m: int, e: float, nreads: int, capture: bool = True,
                  extra_env=None) -> bytes:
    cap = workdir / "cap"
    if cap.exists():
        shutil.rmtree(cap)
    cap.mkdir()
    env = dict(os.environ)
    if capture:
        env["SARU_CAPTURE_DIR"] = str(cap)
    env["SARU_EMUL_FREE_MB"] = "4096"
    if extra_env:
        env.update(extra_env)
    cmd = [str(EMUL), "-m", "0", "-i", "1", "-l", str(m), "-e", repr(e), "-c", str(nreads + 1),
           "-s", str(4 * nreads + 1000), "-g", str(workdir / "genome.fa"),
           "-r", str(workdir / "reads.fa"), "-G", "100000000"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env, check=True)
    return r.stdout


def main() -> None:
    refkit.build_oracle()
    if not EMUL.exists():
        raise SystemExit("oracle/_ref/saruman_emul missing: the reference sources are needed")
    stats = {}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        genomes = {}
        for name, gspec, nreads, m, rate, mix, unm, e, keep in CONFIGS:
            wd = td / name
            wd.mkdir()
            key = gspec
            if key not in genomes:
                genomes[key] = genome_for(gspec)
            g = genomes[key]
            rd = W.sample_reads(g, nreads, m, rate, seed=zlib.crc32(name.encode()), mix=mix,
                                unmapped=unm)
            W.write_fasta_genome(str(wd / "genome.fa"), g)
            W.write_fasta_reads(str(wd / "reads.fa"), rd.seqs)
            run_reference(wd, m, e, nreads)
            flags = {}
            for strand in ("fwd", "rev"):
                files = sorted((wd / "cap").glob(f"batch_{strand}_*.nwb"))
                b, names, do_rev, rl = nwbio.read_nwb(files[0])
                for f in files:
                    bb, _, _, _ = nwbio.read_nwb(f)
                    for fl, c in zip(*np.unique(bb.dirs, return_counts=True)):
                        flags[int(fl)] = flags.get(int(fl), 0) + int(c)
                sb, sn = nwbio.sub_batch(b, names, 0, keep)
                out = HERE / f"{name}_{strand}.nwb.gz"
                nwbio.write_nwb(out, sb, sn, do_rev)
                scores, ra, ga = refkit.ref_align(sb, strict=True)
                tmp = refkit.write_temp_nwb(sb, sn, do_rev)
                try:
                    tsv = refkit.ref_module_tsv(tmp)
                finally:
                    os.unlink(tmp)
                np.savez_compressed(HERE / f"{name}_{strand}.out.npz", scores=scores,
                                    read_aln=ra, genome_aln=ga,
                                    tsv=np.frombuffer(tsv, np.uint8))
                print(name, strand, sb.n, "candidates, k", sb.k, "aligned",
                      int((scores <= sb.k).sum()), "tsv bytes", len(tsv))
            stats[name] = {"flags": flags}
        # end-to-end drop-in golden (small C1-shaped dataset)
        wd = td / "dropin"
        wd.mkdir()
        spec = dict(genome_len=300_000, genome_seed=501, reads=20_000, m=36, rate=0.02,
                    read_seed=502, e=0.06)
        g = W.uniform_genome(spec["genome_len"], seed=spec["genome_seed"])
        rd = W.sample_reads(g, spec["reads"], spec["m"], spec["rate"], seed=spec["read_seed"])
        W.write_fasta_genome(str(wd / "genome.fa"), g)
        W.write_fasta_reads(str(wd / "reads.fa"), rd.seqs)
        out = run_reference(wd, spec["m"], spec["e"], spec["reads"], capture=False)
        lines = sorted(out.splitlines(keepends=True))
        blob = b"".join(lines)
        spec["sha256_sorted_stdout"] = hashlib.sha256(blob).hexdigest()
        spec["lines"] = len(lines)
        spec["args"] = ["-m", "0", "-i", "1", "-l", "36", "-e", "0.06", "-c",
                        str(spec["reads"] + 1), "-s", str(4 * spec["reads"] + 1000), "-G",
                        "100000000"]
        (HERE / "dropin_c1small.json").write_text(json.dumps(spec, indent=1) + "\n")
        with gzip.open(HERE / "dropin_c1small.tsv.gz", "wb", compresslevel=9) as f:
            f.write(blob)
        print("dropin lines", len(lines))
    (HERE / "flag_stats.json").write_text(json.dumps(stats, indent=1) + "\n")


if __name__ == "__main__":
    main()
