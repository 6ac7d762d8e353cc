"""Golden calls of the reference's own q-gram filter for the device filter's
tests (filter_calls.npz).  Run here, where the reference's host build exists
(`make -C oracle`):

    python tests/golden/make_filter_golden.py

For each seeded dataset it runs the reference program with call capture and
keeps, per strand, every submitted call's read ids, positions and flags and
the call boundaries.  The inputs are regenerated from their seeds by the
tests (saruman_b200.workloads), so only the reference's outputs are stored.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from saruman_b200 import workloads as W  # noqa: E402
import nwbio  # noqa: E402

EMUL = ROOT / "oracle" / "_ref" / "saruman_emul"

# name, genome (kind, length, seed), reads, m, k, read seed, queue threshold (-s), read chunk (-c)
DATASETS = [
    ("f36k2", ("uniform", 200_000, 601), 3000, 36, 2, 602, 12_000, 3001),
    ("f100k5", ("repeat", 400_000, 611), 300, 100, 5, 612, 300, 301),
    ("f150k9", ("repeat", 400_000, 621), 200, 150, 9, 622, 250, 64),
    ("f36k3", ("repeat", 300_000, 631), 800, 36, 3, 632, 97, 801),
]


def inputs(spec):
    name, (kind, glen, gseed), nreads, m, k, rseed, chunk, rchunk = spec
    g = (W.uniform_genome(glen, seed=gseed) if kind == "uniform"
         else W.repeat_genome(glen, seed=gseed, copies="zipf"))
    rd = W.sample_reads(g, nreads, m, 0.03, seed=rseed)
    return g, rd.seqs


def main() -> None:
    out = {}
    specs = {}
    for spec in DATASETS:
        name, _, nreads, m, k, _, chunk, rchunk = spec
        g, reads = inputs(spec)
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            W.write_fasta_genome(str(td / "genome.fa"), g)
            W.write_fasta_reads(str(td / "reads.fa"), reads)
            cap = td / "cap"
            cap.mkdir()
            env = dict(os.environ, SARU_CAPTURE_DIR=str(cap), SARU_EMUL_FREE_MB="4096")
            subprocess.run([str(EMUL), "-m", "0", "-i", "1", "-l", str(m), "-e",
                            repr((k + 0.5) / m), "-c", str(rchunk), "-s", str(chunk), "-g",
                            str(td / "genome.fa"), "-r", str(td / "reads.fa"), "-G", "100000000"],
                           stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env, check=True)
            for strand in ("fwd", "rev"):
                calls = [nwbio.read_nwb(f)[0] for f in sorted(cap.glob(f"batch_{strand}_*.nwb"))]
                cb = np.cumsum([0] + [b.n for b in calls]).astype(np.int64)
                cat = lambda a: np.concatenate(a) if a else np.zeros(0)  # noqa: E731
                out[f"{name}_{strand}_call_begin"] = cb
                out[f"{name}_{strand}_ids"] = cat([b.ids for b in calls]).astype(np.int32)
                out[f"{name}_{strand}_pos"] = cat([b.pos for b in calls]).astype(np.int32)
                out[f"{name}_{strand}_dirs"] = cat([b.dirs for b in calls]).astype(np.int8)
                print(name, strand, len(calls), "calls", int(cb[-1]), "candidates")
        specs[name] = list(spec)
    out["specs"] = np.frombuffer(json.dumps(specs).encode(), np.uint8)
    np.savez_compressed(HERE / "filter_calls.npz", **out)


if __name__ == "__main__":
    main()
