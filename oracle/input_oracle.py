"""Plain-Python restatement of the reference's input readers, for tests only.

Test infrastructure: the product's readers are saruman_b200/csrc/input.cpp
(saru_reads_*, saru_genome_*); tests compare them with this restatement on
crafted files, and the end-to-end test in tests/test_input.py pins both
against the reference program's own output.

* reads: src/util.c:294-452 (read_multiple_fasta_file) -- records of two or
  four lines read with fgets into fixed buffers (name 60 bytes, sequence
  and quality read_length + 2), the sequence cut at read_length and
  upper-cased, short reads and reads with more than max_n Ns dropped, the
  name the name line minus its first and last byte.
* genome: src/saruman.c:139-271 -- chunks of chunk_value bases plus a
  read_length overhang through a buffer of chunk_value + read_length bytes,
  newlines dropped, the first line skipped, the rest read a byte at a time
  (a failed one-byte read at the end of the file keeps the byte left at
  the buffer's start), the next chunk resuming where the chunk's own bases
  ended, first with what is left of the buffer.
"""
from __future__ import annotations


class _File:
    def __init__(self, data: bytes):
        self.data = data
        self.pos = 0

    def fgets(self, size: int):
        """bytes of one fgets into a buffer of `size`, or None at the end."""
        if self.pos >= len(self.data):
            return None
        end = self.pos
        while end < len(self.data) and end - self.pos < size - 1:
            end += 1
            if self.data[end - 1] == 0x0A:
                break
        out = self.data[self.pos:end]
        self.pos = end
        return out

    def fread(self, n: int) -> bytes:
        out = self.data[self.pos:self.pos + n]
        self.pos += len(out)
        return out


def _c_string(buf: bytearray) -> bytes:
    i = buf.find(0)
    return bytes(buf if i < 0 else buf[:i])


def read_batches(data: bytes, m: int, max_n: int, batch: int, fastq: bool = False):
    """[(reads, names, records)] of the reference's batches (see
    saruman_b200.read_batches for the batching)."""
    f = _File(data)
    name = bytearray(60)
    seq = bytearray(m + 2)
    qname = bytearray(60)
    qual = bytearray(m + 2)

    def load(buf: bytearray, line):
        if line is None:  # fgets leaves the buffer as it was
            return
        buf[:len(line)] = line
        buf[len(line)] = 0

    out = []
    while True:
        reads, names, records = [], [], 0
        while records < batch:
            line = f.fgets(60)
            if line is None:
                break
            load(name, line)
            load(seq, f.fgets(m + 2))
            if fastq:
                load(qname, f.fgets(60))
                load(qual, f.fgets(m + 2))
            records += 1
            seq[m] = 0
            nm = _c_string(name)
            if nm:
                nm = nm[:-1]
            s = bytes(seq[:m]).upper()
            seq[:m] = s
            text = _c_string(seq)
            if len(text) < m or s.count(b"N") > max_n:
                continue
            reads.append(text[:m])
            names.append(nm[1:])
        if records == 0:
            return out
        if reads:
            out.append((reads, names, records))
        if records < batch:
            return out


def genome_chunks(data: bytes, chunk: int, m: int):
    """[(bytes, bases, total)] of the reference's genome chunks."""
    f = _File(data)
    cap = chunk + m
    buf = bytearray(cap)
    buf_read = 0
    buf_pos = 0
    file_pos = 0
    first = True
    total = 0
    chunks = []
    while True:
        out = bytearray()

        def keep(c: int) -> bool:
            if c != 0x0A:
                out.append(ord(chr(c).upper()) if 0x61 <= c <= 0x7A else c)
                return True
            return False

        if not first:
            f.pos = file_pos
            if buf_pos < cap:
                p = buf_pos
                while len(out) < chunk and p < buf_read:
                    keep(buf[p])
                    p += 1
        got = f.fread(cap)
        buf[:len(got)] = got
        buf_read = len(got)
        p = 0
        if first:
            while p < buf_read and buf[p] not in (0x0A, 0x00):
                p += 1
        while len(out) < chunk and p < buf_read:
            keep(buf[p])
            p += 1
        buf_pos = p
        first = False
        more = True
        while len(out) < chunk and more:
            b = f.fread(1)
            more = len(b) == 1
            if more:
                buf[0] = b[0]
            keep(buf[0])
        own = len(out)
        total += own
        file_pos = f.pos
        over = 0
        while over < m and more:
            b = f.fread(1)
            more = len(b) == 1
            if more:
                buf[0] = b[0]
            if keep(buf[0]):
                over += 1
        chunks.append((bytes(out), own, total))
        if own < chunk:
            return chunks
