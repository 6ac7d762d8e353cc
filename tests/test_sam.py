"""SAM conversion of the reference writer's TSV (golden fixtures): every
record's CIGAR spans stop - start + 1 genome bases and its SEQ length,
SEQ is the read string without gaps, strand maps to FLAG 16."""
from __future__ import annotations

import pytest

import golden_io as G
from saruman_b200 import sam


def cigar_lengths(c: str) -> tuple[int, int]:
    ref = qry = 0
    num = ""
    for ch in c:
        if ch.isdigit():
            num += ch
            continue
        n = int(num)
        num = ""
        if ch in "MD":
            ref += n
        if ch in "MI":
            qry += n
    return ref, qry


@pytest.mark.parametrize("name", G.fixture_names())
def test_sam_records_agree_with_the_tsv(name):
    b, names, do_rev, m, exp = G.load_fixture(name)
    lines = exp["tsv"].decode().splitlines()
    text = sam.tsv_to_sam(lines, "genome", 5_000_000)
    recs = [r for r in text.splitlines() if not r.startswith("@")]
    assert len(recs) == len(lines)
    for line, rec in zip(lines, recs):
        f = line.split("\t")
        s = rec.split("\t")
        assert s[1] == ("16" if f[3] == "<<" else "0")
        assert s[3] == f[1]
        assert s[9] == f[4].replace("_", "")
        ref, qry = cigar_lengths(s[5])
        assert qry == len(s[9])
        assert ref == int(f[2]) - int(f[1]) + 1
        assert s[11] == f"NM:i:{f[6]}"


def test_unmapped_line():
    rec = sam.line_to_sam("r1 extra\t*\t*\t>>\tACGT\t*\t4\n", "g")
    assert rec.split("\t")[:4] == ["r1", "4", "*", "0"]
