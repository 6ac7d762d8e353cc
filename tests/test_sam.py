"""SAM conversion of the reference writer's TSV (golden fixtures): every
record's CIGAR spans stop - start + 1 genome bases and its SEQ length,
SEQ is the read string without gaps, strand maps to FLAG 16."""
from __future__ import annotations

import pytest

import golden_io as G
from saruman_b200 import sam


# The checker: a plain-Python statement of the conversion rules.
def cigar(read_aln: str, genome_aln: str) -> str:
    ops = []
    for r, g in zip(read_aln, genome_aln):
        op = "D" if r == "_" else ("I" if g == "_" else "M")
        if ops and ops[-1][0] == op:
            ops[-1][1] += 1
        else:
            ops.append([op, 1])
    return "".join(f"{n}{op}" for op, n in ops)


def line_to_sam(line: str, rname: str) -> str:
    f = line.rstrip("\n").split("\t")
    name, start, stop, strand, read_aln, genome_aln, score = f[:7]
    qname = name.split()[0] if name.split() else "*"
    if start == "*":
        return "\t".join([qname, "4", "*", "0", "0", "*", "*", "0", "0", read_aln, "*"])
    flag = "16" if strand == "<<" else "0"
    seq = read_aln.replace("_", "")
    return "\t".join([qname, flag, rname, start, "255", cigar(read_aln, genome_aln), "*", "0",
                      "0", seq or "*", "*", f"NM:i:{score}"])


def python_sam(text: str, rname: str, rlen: int) -> str:
    head = (f"@HD\tVN:1.6\tSO:unsorted\n@SQ\tSN:{rname}\tLN:{rlen}\n"
            "@PG\tID:saruman_b200\tPN:saruman_b200\n")
    return head + "".join(line_to_sam(x, rname) + "\n" for x in text.split("\n") if x.strip())


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


def test_unmapped_line(saru_lib):
    text = sam.tsv_bytes_to_sam(b"r1 extra\t*\t*\t>>\tACGT\t*\t4\n", "g", 10).decode()
    rec = [x for x in text.splitlines() if not x.startswith("@")][0]
    assert rec.split("\t")[:4] == ["r1", "4", "*", "0"]


@pytest.mark.parametrize("name", G.fixture_names())
def test_library_converter_equals_the_rules(saru_lib, name):
    """saru_tsv_to_sam (the library, callable from C) writes exactly what
    the conversion rules give, on every golden TSV."""
    b, names, do_rev, m, exp = G.load_fixture(name)
    text = exp["tsv"].decode()
    assert sam.tsv_bytes_to_sam(exp["tsv"], "chr_x", 1234567).decode() == \
        python_sam(text, "chr_x", 1234567)


def test_library_converter_edge_lines(saru_lib):
    lines = ["  lead blank name\t10\t20\t>>\tAC_GT\tACTGT\t1\n",
             "\t5\t9\t<<\tACGT\tA_GT\t2\r\n",  # empty name, CR kept in the score
             "unm\t*\t*\t>>\tACGTACGT\t*\t8\n",
             "   \n",
             "gapsonly\t1\t1\t>>\t___\tAAA\t3\n",
             "short\t1\t2\t>>\tAA\tAAAA\t0"]
    text = "".join(lines)
    assert sam.tsv_bytes_to_sam(text.encode(), "g", 99).decode() == python_sam(text, "g", 99)
    import saruman_b200 as S
    with pytest.raises(S.SaruError):
        sam.tsv_bytes_to_sam(b"too\tfew\tfields\n", "g", 1)
