"""Child-process driver of the reference-compatible entry point
cuda_needleman_wunsch (include/saruman_b200.h) for the tests.

    python tests/legacy_call.py <fixture.nwb.gz> [lib]

Sets the caller-owned globals the reference's host program would own
(read_length_value, the read_names uthash table, output-control arrays),
makes the call and lets the library print its TSV lines to stdout.  The
read_names table is built as a uthash list linked in application order
(struct read_name_hash, src/util.h:350-354): int read_number; char
name[60]; UT_hash_handle hh, whose third pointer links the elements.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import nwbio  # noqa: E402


class UTHandle(C.Structure):
    _fields_ = [("tbl", C.c_void_p), ("prev", C.c_void_p), ("next", C.c_void_p),
                ("hh_prev", C.c_void_p), ("hh_next", C.c_void_p), ("key", C.c_void_p),
                ("keylen", C.c_uint), ("hashv", C.c_uint)]


class ReadName(C.Structure):
    _fields_ = [("read_number", C.c_int), ("name", C.c_char * 60), ("hh", UTHandle)]


def build_names(names_by_id: dict[int, bytes]):
    ids = sorted(names_by_id)
    arr = (ReadName * max(len(ids), 1))()
    for i, rid in enumerate(ids):
        arr[i].read_number = rid
        arr[i].name = names_by_id[rid][:59]
    base = C.addressof(arr)
    for i in range(len(ids)):
        arr[i].hh.next = base + (i + 1) * C.sizeof(ReadName) if i + 1 < len(ids) else None
    return arr


def main():
    path = sys.argv[1]
    lib_path = sys.argv[2] if len(sys.argv) > 2 else str(
        Path(__file__).resolve().parents[1] / "saruman_b200" / "libsaruman_b200.so")
    b, names, do_rev, m = nwbio.read_nwb(path)
    lib = C.CDLL(lib_path)
    table = build_names(dict(zip(b.ids.tolist(), names)))
    C.c_void_p.in_dll(lib, "read_names").value = C.addressof(table)
    C.c_ushort.in_dll(lib, "read_length_value").value = m
    n_ids = int(b.ids.max()) + 1 if b.n else 1
    fwd = (C.c_char * n_ids)()
    rev = (C.c_char * n_ids)()
    C.c_void_p.in_dll(lib, "forward_output_control").value = C.addressof(fwd)
    C.c_void_p.in_dll(lib, "reverse_output_control").value = C.addressof(rev)
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    lib.cuda_allocate_memory(C.c_int(4 if do_rev else 0))
    lib.cuda_needleman_wunsch(C.c_int(b.match), C.c_int(b.mismatch), P(b.genome), P(b.reads),
                              P(b.genome_offsets), P(b.read_offsets), P(b.edit_offsets),
                              C.c_int(b.n), P(b.ids), P(b.pos), P(b.dirs), C.c_int(b.k),
                              C.c_size_t(b.total_genome), C.c_size_t(b.n * b.m),
                              C.c_size_t(b.total_edit), C.c_int(do_rev))
    C.CDLL(None).fflush(None)
    done = C.c_uint.in_dll(lib, "reverse_alignments_done" if do_rev else
                           "forward_alignments_done").value
    marked = int(np.frombuffer(rev if do_rev else fwd, np.uint8).sum())
    lib.cuda_free_memory(C.c_int(4 if do_rev else 0))
    sys.stderr.write(f"DONE {done} MARKED {marked}\n")


if __name__ == "__main__":
    main()
