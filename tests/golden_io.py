"""Access to the committed golden fixtures (tests/golden/)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

import nwbio

GOLDEN = Path(__file__).resolve().parent / "golden"


def fixture_names() -> list[str]:
    return sorted(p.name[:-len(".nwb.gz")] for p in GOLDEN.glob("*.nwb.gz"))


def load_fixture(name: str):
    """(batch, names, do_reverse, read_length, expected) where expected has
    the reference's scores, read_aln, genome_aln and tsv bytes."""
    b, names, do_rev, m = nwbio.read_nwb(GOLDEN / f"{name}.nwb.gz")
    z = np.load(GOLDEN / f"{name}.out.npz")
    exp = {"scores": z["scores"], "read_aln": z["read_aln"], "genome_aln": z["genome_aln"],
           "tsv": z["tsv"].tobytes()}
    return b, names, do_rev, m, exp


def names_by_id(b, names) -> dict[int, bytes]:
    return dict(zip(b.ids.tolist(), names))
