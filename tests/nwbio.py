"""Reader/writer for captured alignment batches (.nwb).

A capture is the exact argument list of one reference call of
cuda_needleman_wunsch (src/cuda-functions.h:55-63), written by the oracle
build's capture wrapper (oracle/ref_shim/emul_glue.c), plus the read name of
each candidate.  Test infrastructure only.
"""
from __future__ import annotations

import gzip
import io
import struct
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from saruman_b200.workloads import Batch  # noqa: E402

MAGIC = b"SARUNWB1"
NAME_LEN = 60


def _open(path):
    path = str(path)
    return gzip.open(path, "rb") if path.endswith(".gz") else open(path, "rb")


def read_nwb(path) -> tuple[Batch, list[bytes], int, int]:
    """Returns (batch, names, do_reverse, read_length)."""
    with _open(path) as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError(f"{path}: not an .nwb capture")
    match, mismatch, n, k, do_rev, m = struct.unpack_from("<6i", data, 8)
    tg, tr, te = struct.unpack_from("<3q", data, 32)
    o = 56
    glen = tg - n * k

    def take(nbytes, dtype):
        nonlocal o
        a = np.frombuffer(data, dtype=dtype, count=nbytes // np.dtype(dtype).itemsize, offset=o)
        o += nbytes
        return a.copy()

    genome = take(glen, np.uint8)
    reads = take(tr, np.uint8)
    go = take(4 * n, np.int32)
    ro = take(4 * n, np.int32)
    eo = take(4 * n, np.int32)
    ids = take(4 * n, np.int32)
    pos = take(4 * n, np.int32)
    dirs = take(n, np.int8)
    names = []
    for i in range(n):
        raw = data[o:o + NAME_LEN]
        o += NAME_LEN
        names.append(raw.split(b"\0", 1)[0])
    b = Batch(m=m, k=k, genome=genome, reads=reads, genome_offsets=go, read_offsets=ro,
              edit_offsets=eo, dirs=dirs, ids=ids, pos=pos, match=match, mismatch=mismatch)
    assert b.total_genome == tg and b.total_edit == te, (b.total_genome, tg, b.total_edit, te)
    return b, names, do_rev, m


def write_nwb(path, b: Batch, names: list[bytes], do_reverse: int) -> None:
    n = b.n
    buf = io.BytesIO()
    buf.write(MAGIC)
    buf.write(struct.pack("<6i", b.match, b.mismatch, n, b.k, do_reverse, b.m))
    buf.write(struct.pack("<3q", b.total_genome, n * b.m, b.total_edit))
    for a in (b.genome, b.reads, b.genome_offsets, b.read_offsets, b.edit_offsets, b.ids,
              b.pos, b.dirs):
        buf.write(np.ascontiguousarray(a).tobytes())
    for nm in names:
        buf.write(nm[:NAME_LEN - 1].ljust(NAME_LEN, b"\0"))
    raw = buf.getvalue()
    path = str(path)
    if path.endswith(".gz"):
        with gzip.open(path, "wb", compresslevel=9) as f:
            f.write(raw)
    else:
        Path(path).write_bytes(raw)


def sub_batch(b: Batch, names: list[bytes], start: int, count: int) -> tuple[Batch, list[bytes]]:
    """Candidates [start, start+count) re-based into a batch of their own (a
    new call: its first candidate is the first of the call)."""
    s, e = start, min(b.n, start + count)
    L = b.lengths
    gs = int(np.concatenate([[0], np.cumsum(L)])[s])
    ge = int(np.cumsum(L)[e - 1])
    Ls = L[s:e]
    go = np.cumsum(Ls).astype(np.int32)
    ro = ((np.arange(e - s) + 1) * b.m).astype(np.int32)
    esz = (b.m + 1) * (Ls + 1)
    eo = (np.cumsum(esz) - esz).astype(np.int32)
    nb = Batch(m=b.m, k=b.k, genome=b.genome[gs:ge].copy(),
               reads=b.reads[s * b.m:e * b.m].copy(), genome_offsets=go, read_offsets=ro,
               edit_offsets=eo, dirs=b.dirs[s:e].copy(), ids=b.ids[s:e].copy(),
               pos=b.pos[s:e].copy(), match=b.match, mismatch=b.mismatch)
    return nb, names[s:e]
