"""SAM records from the reference writer's TSV lines (saru_tsv_to_sam in
the library; include/saruman_b200.h says what each SAM column holds).

The reference prints one line per alignment (src/cuda-functions.cu:987),
perfect hits (src/hash.c:580) and unmapped reads (src/hash.c:821) in the
same layout, and leaves SAM to an external script (README.md:32).

    python -m saruman_b200.sam REFERENCE_NAME REFERENCE_LENGTH < tsv > sam
"""
from __future__ import annotations

import ctypes as C
import io
from typing import Iterable

import numpy as np


def tsv_bytes_to_sam(tsv: bytes, rname: str, rlen: int) -> bytes:
    """SAM text (header and one record per non-blank line) for TSV bytes."""
    from . import SARU_E_INVALID, SaruError, last_error, load
    lib = load()
    lib.saru_tsv_to_sam.restype = C.c_int64
    lib.saru_tsv_to_sam.argtypes = [C.c_char_p, C.c_int64, C.c_char_p, C.c_int64, C.c_void_p,
                                    C.c_int64]
    name = rname.encode()
    need = lib.saru_tsv_to_sam(tsv, len(tsv), name, rlen, None, 0)
    if need < 0:
        raise SaruError(SARU_E_INVALID, last_error())
    out = np.zeros(need, np.uint8)
    lib.saru_tsv_to_sam(tsv, len(tsv), name, rlen, out.ctypes.data, need)
    return out.tobytes()


def tsv_to_sam(lines: Iterable[str], rname: str, rlen: int, out: io.TextIOBase | None = None):
    """Writes the SAM header and one record per TSV line; returns the text
    when `out` is None."""
    text = "".join(line if line.endswith("\n") else line + "\n" for line in lines)
    sam = tsv_bytes_to_sam(text.encode(), rname, rlen).decode()
    if out is None:
        return sam
    out.write(sam)
    return None


if __name__ == "__main__":
    import sys
    if len(sys.argv) != 3:
        sys.exit("usage: python -m saruman_b200.sam REFERENCE_NAME REFERENCE_LENGTH < tsv > sam")
    sys.stdout.buffer.write(tsv_bytes_to_sam(sys.stdin.buffer.read(), sys.argv[1],
                                             int(sys.argv[2])))
