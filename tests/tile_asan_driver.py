"""Runs the host emulation of the banded kernel's warp loop under
AddressSanitizer (child process of tests/test_tile_host.py).

Every array is allocated at exactly its size and placed at a chosen
misalignment, so any out-of-range shared-slice, plane, input or output
access aborts the run; the outputs are compared with the oracle.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import refkit as R  # noqa: E402
from saruman_b200 import workloads as W  # noqa: E402


def exact(a: np.ndarray, off: int) -> np.ndarray:
    """Copy of `a` whose data ends exactly at the end of its allocation and
    starts `off` bytes past a 16-byte boundary (when the allocator aligns)."""
    raw = np.empty(a.nbytes + off, np.uint8)
    v = raw[off:].view(a.dtype)
    v[...] = a.reshape(-1)
    return v


def compact_case(lib, b, g, r, go, ro, d, wide, s1, ra1, ga1) -> int:
    import saruman_b200 as S
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    R_ = S.compact_record_bytes(b.m, b.k)
    rec = exact(np.zeros(b.n * R_, np.uint8), 0)
    sc = np.zeros(b.n, np.int32)
    st = lib.tile_align_compact(P(g), P(r), P(go), P(ro), P(d), C.c_long(b.n), C.c_int(b.k),
                                C.c_int(b.m), C.c_int(wide), C.c_int(1), C.c_int(3), P(sc),
                                P(rec), C.c_long(R_))
    out = S.expand_compact(b, sc, rec, R_, nthreads=2)
    ok = (st == 0 and np.array_equal(np.minimum(s1, b.k + 1), sc)
          and np.array_equal(ra1, out.read_aln) and np.array_equal(ga1, out.genome_aln))
    if not ok:
        print("COMPACT MISMATCH", b.m, b.k, st, flush=True)
    return 0 if ok else 1


def main():
    lib = C.CDLL(sys.argv[1])
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    cases = [(36, 2, 0.05), (100, 5, 0.04), (75, 5, 0.2), (150, 9, 0.05), (250, 15, 0.05),
             (20, 1, 0.1), (40, 7, 0.1), (64, 15, 0.3), (512, 15, 0.03), (2, 0, 0.1),
             (8, 1, 0.1)]
    bad = 0
    for ci, (m, k, err) in enumerate(cases):
        for seed in range(2):
            n = 97 + 31 * seed  # ragged last tile
            b = W.random_batch(m, k, n, seed=seed + 5 * ci, err=err,
                               alphabet=b"ACGT" if seed == 0 else b"ACGTN")
            s1, ra1, ga1, _ = R.oracle_align(b)
            # 64-bit bands for k > 7; a launch shape may also ask for them at
            # any k (the second seed)
            wide = 1 if (k > 7 or seed == 1) else 0
            for off in (0, 3, 9):
                g = exact(b.genome, off)
                r = exact(b.reads, (off + 5) % 16)
                go = exact(b.genome_offsets, 0)
                ro = exact(b.read_offsets, 0)
                d = exact(b.dirs, 1)
                sc = np.zeros(n, np.int32)
                ra = exact(np.zeros(b.total_genome, np.uint8), (off + 7) % 16)
                ga = exact(np.zeros(b.total_genome, np.uint8), (off + 11) % 16)
                st = lib.tile_align_batch(P(g), P(r), P(go), P(ro), P(d), C.c_long(n), C.c_int(k),
                                          C.c_int(m), C.c_int(wide), C.c_int(1), C.c_int(3),
                                          P(sc), P(ra), P(ga))
                ok = (st == 0 and np.array_equal(np.minimum(s1, k + 1), sc)
                      and np.array_equal(ra1, ra) and np.array_equal(ga1, ga))
                if not ok:
                    bad += 1
                    print("MISMATCH", m, k, seed, off, st, flush=True)
                if off == 3:  # compact records, expanded on the host by the library
                    bad += compact_case(lib, b, g, r, go, ro, d, wide, s1, ra1, ga1)
                if off == 9:  # the call in slices of whole tiles
                    sc2 = np.zeros(n, np.int32)
                    ra2 = exact(np.zeros(b.total_genome, np.uint8), 2)
                    ga2 = exact(np.zeros(b.total_genome, np.uint8), 13)
                    st2 = lib.tile_align_slices(P(g), P(r), P(go), P(ro), P(d), C.c_long(n),
                                                C.c_int(k), C.c_int(m), C.c_int(wide), C.c_int(1),
                                                C.c_int(3), C.c_long(32 * (1 + seed)), P(sc2),
                                                P(ra2), P(ga2))
                    if not (st2 == 0 and np.array_equal(np.minimum(s1, k + 1), sc2)
                            and np.array_equal(ra1, ra2) and np.array_equal(ga1, ga2)):
                        bad += 1
                        print("SLICE MISMATCH", m, k, seed, st2, flush=True)
    # an irregular tile (window far too long) must be rejected, not staged
    b = W.random_batch(36, 2, 40, seed=1)
    go = b.genome_offsets.copy()
    go[5:] += 100000
    g = np.zeros(int(go[-1]), np.uint8)
    sc = np.zeros(b.n, np.int32)
    ra = np.zeros(int(go[-1]) + 2 * b.n, np.uint8)
    ga = np.zeros_like(ra)
    st = lib.tile_align_batch(P(g), P(b.reads), P(go), P(b.read_offsets), P(b.dirs),
                              C.c_long(b.n), C.c_int(2), C.c_int(36), C.c_int(0), C.c_int(1),
                              C.c_int(3), P(sc), P(ra), P(ga))
    if not (st & 1):
        bad += 1
        print("irregular tile not reported", st)
    bad += multi_launch(lib)
    print("BAD", bad)
    sys.exit(1 if bad else 0)


class HostSeg(C.Structure):
    _fields_ = [("genome", C.c_void_p), ("reads", C.c_void_p), ("goff", C.c_void_p),
                ("roff", C.c_void_p), ("dirs", C.c_void_p), ("scores", C.c_void_p),
                ("ra", C.c_void_p), ("ga", C.c_void_p), ("n", C.c_long), ("k", C.c_int),
                ("max_m", C.c_int), ("first_of_call", C.c_int), ("wide", C.c_int)]


def multi_launch(lib) -> int:
    """Calls of mixed read lengths and band widths in one emulated launch,
    every warp's fill before any traceback (the interleaving in which lanes
    could clobber each other's decision planes)."""
    specs = [(36, 3, 300), (75, 5, 200), (100, 6, 250), (150, 9, 120), (250, 15, 40), (40, 2, 33)]
    keep, segs = [], []
    for i, (m, k, n) in enumerate(specs):
        b = W.random_batch(m, k, n, seed=100 + i, err=0.05, alphabet=b"ACGT" if i % 3 else b"ACGTN")
        sc = np.zeros(n, np.int32)
        ra = exact(np.zeros(b.total_genome, np.uint8), i % 16)
        ga = exact(np.zeros(b.total_genome, np.uint8), (i + 5) % 16)
        g = exact(b.genome, (i + 3) % 16)
        r = exact(b.reads, (i + 7) % 16)
        keep.append((b, sc, ra, ga, g, r))
        segs.append(HostSeg(g.ctypes.data, r.ctypes.data, b.genome_offsets.ctypes.data,
                            b.read_offsets.ctypes.data, b.dirs.ctypes.data, sc.ctypes.data,
                            ra.ctypes.data, ga.ctypes.data, n, k, m, 1, 1 if k > 7 else 0))
    order = sorted(range(len(specs)), key=lambda i: -(specs[i][0] * (specs[i][1] + 1)))
    arr = (HostSeg * len(segs))(*[segs[i] for i in order])
    st = lib.tile_align_multi(arr, len(segs), 5)
    bad = 1 if st else 0
    for (b, sc, ra, ga, _, _), spec in zip(keep, specs):
        s1, ra1, ga1, _ = R.oracle_align(b, nthreads=4)
        if not (np.array_equal(np.minimum(s1, b.k + 1), sc) and np.array_equal(ra1, ra)
                and np.array_equal(ga1, ga)):
            print("MULTI MISMATCH", spec, flush=True)
            bad += 1
    return bad


if __name__ == "__main__":
    main()
