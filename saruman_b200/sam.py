"""SAM records from the reference writer's TSV lines.

The reference prints one line per alignment (src/cuda-functions.cu:987):
name, start, stop, strand (">>" forward, "<<" reverse), the aligned read
string, the aligned genome string (gaps as '_'), the edit distance; perfect
hits come from the filter in the same layout, with genome and read strings
equal (src/hash.c:580), and unmapped reads, when printed, as name, '*', '*',
strand, read, '*', length (src/hash.c:821).  Its README points to an
external script for SAM; this is a native converter:

    QNAME  the name up to the first blank
    FLAG   16 for '<<', 0 for '>>', 4 for an unmapped line
    RNAME  the reference name given to the converter
    POS    start (1-based, as printed)
    MAPQ   255 (not computed)
    CIGAR  run-length of the columns: M (bytes in both strings), I ('_' in
           the genome string), D ('_' in the read string)
    SEQ    the read string without gaps (reverse-complemented reads are
           already in genome orientation, as SAM wants for FLAG 16)
    QUAL   '*'
    NM:i   the printed edit distance
"""
from __future__ import annotations

import io
from typing import Iterable


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
    if len(f) < 7:
        raise ValueError(f"not a TSV alignment line: {line!r}")
    name, start, stop, strand, read_aln, genome_aln, score = f[:7]
    qname = name.split()[0] if name.split() else "*"
    if start == "*":  # unmapped read
        return "\t".join([qname, "4", "*", "0", "0", "*", "*", "0", "0", read_aln, "*"])
    flag = "16" if strand == "<<" else "0"
    seq = read_aln.replace("_", "")
    return "\t".join([qname, flag, rname, start, "255", cigar(read_aln, genome_aln), "*", "0",
                      "0", seq or "*", "*", f"NM:i:{score}"])


def tsv_to_sam(lines: Iterable[str], rname: str, rlen: int, out: io.TextIOBase | None = None):
    """Writes the SAM header and one record per TSV line; returns the text
    when `out` is None."""
    buf = out or io.StringIO()
    buf.write("@HD\tVN:1.6\tSO:unsorted\n")
    buf.write(f"@SQ\tSN:{rname}\tLN:{rlen}\n")
    buf.write("@PG\tID:saruman_b200\tPN:saruman_b200\n")
    for line in lines:
        if line.strip():
            buf.write(line_to_sam(line, rname) + "\n")
    return buf.getvalue() if out is None else None


if __name__ == "__main__":
    import sys
    if len(sys.argv) != 3:
        sys.exit("usage: python -m saruman_b200.sam REFERENCE_NAME REFERENCE_LENGTH < tsv > sam")
    tsv_to_sam(sys.stdin, sys.argv[1], int(sys.argv[2]), sys.stdout)
