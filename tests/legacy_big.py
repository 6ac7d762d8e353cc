"""Child-process driver for the drop-in entry on a large call: one seeded
random call of N candidates (large enough that the writer splits it over
threads), made twice through cuda_needleman_wunsch -- first against name
table A, then against table B (other names, another list) -- so the
caller's table is read again when it changes.  Writes the two calls' TSV to
stdout, separated by a marker line.

    python tests/legacy_big.py <m> <k> <n> <seed>
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from legacy_call import build_names  # noqa: E402
from saruman_b200 import workloads as W  # noqa: E402

MARK = b"==== second call ====\n"


def main():
    m, k, n, seed = (int(x) for x in sys.argv[1:5])
    b = W.random_batch(m, k, n, seed=seed, err=0.05, alphabet=b"ACGTN")
    lib = C.CDLL(str(Path(__file__).resolve().parents[1] / "saruman_b200" / "libsaruman_b200.so"))
    C.c_ushort.in_dll(lib, "read_length_value").value = m
    n_ids = int(b.ids.max()) + 1
    fwd, rev = (C.c_char * n_ids)(), (C.c_char * n_ids)()
    C.c_void_p.in_dll(lib, "forward_output_control").value = C.addressof(fwd)
    C.c_void_p.in_dll(lib, "reverse_output_control").value = C.addressof(rev)
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    libc = C.CDLL(None)
    keep = []
    for tag in (b"A", b"B"):
        table = build_names({i: b"%s_read%d" % (tag, i) for i in range(n_ids)})
        keep.append(table)
        C.c_void_p.in_dll(lib, "read_names").value = C.addressof(table)
        lib.cuda_needleman_wunsch(C.c_int(0), C.c_int(1), P(b.genome), P(b.reads),
                                  P(b.genome_offsets), P(b.read_offsets), P(b.edit_offsets),
                                  C.c_int(b.n), P(b.ids), P(b.pos), P(b.dirs), C.c_int(k),
                                  C.c_size_t(b.total_genome), C.c_size_t(b.n * m),
                                  C.c_size_t(b.total_edit), C.c_int(0))
        libc.fflush(None)
        if tag == b"A":
            sys.stdout.flush()
            sys.stdout.buffer.write(MARK)
            sys.stdout.flush()


if __name__ == "__main__":
    main()
