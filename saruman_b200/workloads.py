"""Seeded synthetic workloads for the alignment stage.

No public dataset is used: the reference points to sample data on an FTP
server that is not available here.  These generators produce genomes, reads
and candidate batches with the shapes, sizes and error distributions of the
five benchmark configurations:

* C1  1 Mbp uniform-ACGT genome, 100k reads of 36 bp, 2 % errors (70/15/15
      substitution/insertion/deletion), k = 2.
* C2  5 Mbp genome at 50 % GC with 40 repeat families of 1.5 kbp (5-50 copies,
      99 % copy identity), 2M reads of 100 bp, 3 % errors, k = 5.
* C3  the C2 genome with Zipf(1.5, max 500) copy numbers, reads of mixed
      length {36, 75, 100, 150}, k = ceil(0.06 * length).
* C4  10 Mbp uniform genome, 1M reads of 250 bp, 4 % errors (60/20/20),
      k = 15, 5 % unmapped random reads.
* C5  serving: the C3 genome, Poisson-arriving requests.

Candidate batches follow the layout the reference's candidate collection
builds (src/hash.c:898-1111): windows of length L = m + so + eo packed back to
back, reads packed at stride m, `genome_offsets` the inclusive prefix sum of
L, `read_offsets[t] = (t+1)*m`, `edit_offsets` the exclusive prefix sum of
(m+1)(L+1), and a direction/flank flag per candidate (1/5: eo = k; 2/6:
so = k; 3/7: so = eo = k; flags > 3 mean the read was reverse complemented).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.arange(256, dtype=np.uint8)
for _a, _b in ((b"A", b"T"), (b"C", b"G"), (b"G", b"C"), (b"T", b"A")):
    _COMP[_a[0]] = _b[0]


def reverse_complement(seqs: np.ndarray) -> np.ndarray:
    """Reverse complement of rows of ASCII bytes; only A/C/G/T are swapped
    and other bytes (N) are kept, as in the reference (src/util.c:35-57)."""
    return _COMP[seqs[..., ::-1]]


def k_for(m: int, rate: float = 0.06) -> int:
    return int(math.ceil(rate * m))


def uniform_genome(n: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return BASES[rng.integers(0, 4, size=n, dtype=np.uint8)]


def repeat_genome(n: int, seed: int, families: int = 40, family_len: int = 1500,
                  copies: str = "uniform", identity: float = 0.99,
                  gc: float = 0.5) -> np.ndarray:
    """Background at the given GC content with inserted repeat families.

    copies="uniform": 5-50 copies per family (C2); copies="zipf": Zipf(1.5)
    capped at 500 (C3).  Each copy carries (1-identity) substitutions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    g = BASES[rng.choice(4, size=n, p=p).astype(np.uint8)]
    for _ in range(families):
        fam = BASES[rng.choice(4, size=family_len, p=p).astype(np.uint8)]
        if copies == "zipf":
            c = int(min(rng.zipf(1.5), 500))
        else:
            c = int(rng.integers(5, 51))
        for _ in range(c):
            cp = fam.copy()
            mut = rng.random(family_len) < (1.0 - identity)
            cp[mut] = BASES[(np.searchsorted(BASES, cp[mut]) + rng.integers(1, 4, mut.sum())) % 4]
            at = int(rng.integers(0, n - family_len))
            g[at:at + family_len] = cp
    return g


@dataclasses.dataclass
class Reads:
    seqs: np.ndarray      # (n, m) uint8 ASCII, as sequenced (maybe reverse complemented)
    origin: np.ndarray    # (n,) int64 genome start of the source fragment, -1 if random
    reverse: np.ndarray   # (n,) bool
    span: np.ndarray      # (n,) genome bases consumed by the read


def sample_reads(genome: np.ndarray, n: int, m: int, rate: float, seed: int,
                 mix=(0.70, 0.15, 0.15), unmapped: float = 0.0,
                 chunk: int = 262144) -> Reads:
    """Reads of fixed length m sampled uniformly from `genome`, with per-base
    error events (substitution, insertion, deletion) at `rate` split by `mix`,
    half of them reverse complemented, plus a fraction of random reads."""
    rng = np.random.Generator(np.random.PCG64(seed))
    G = len(genome)
    out = np.empty((n, m), dtype=np.uint8)
    origin = np.empty(n, dtype=np.int64)
    span = np.empty(n, dtype=np.int64)
    rev = rng.random(n) < 0.5
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        c = e - s
        ev = rng.random((c, m)) < rate
        kind = rng.choice(3, size=(c, m), p=np.asarray(mix))
        ins = ev & (kind == 1)
        dele = ev & (kind == 2)
        sub = ev & (kind == 0)
        step = np.where(ins, 0, np.where(dele, 2, 1)).astype(np.int64)
        # genome index consumed by read position t: origin + sum(step[:t]) + dele[t]
        before = np.cumsum(step, axis=1) - step
        span_c = step.sum(axis=1) + 1
        org = rng.integers(0, G - int(span_c.max()) - 1, size=c)
        idx = org[:, None] + before + dele.astype(np.int64)
        r = genome[idx]
        rnd = BASES[rng.integers(0, 4, size=(c, m), dtype=np.uint8)]
        r = np.where(ins, rnd, r)
        shift = rng.integers(1, 4, size=(c, m))
        code = np.searchsorted(BASES, r)
        r = np.where(sub, BASES[(code + shift) % 4], r)
        out[s:e] = r
        origin[s:e] = org
        span[s:e] = span_c
    if unmapped > 0:
        um = rng.random(n) < unmapped
        out[um] = BASES[rng.integers(0, 4, size=(int(um.sum()), m), dtype=np.uint8)]
        origin[um] = -1
    out[rev] = reverse_complement(out[rev])
    return Reads(out, origin, rev, span)


def write_fasta_genome(path: str, genome: np.ndarray, name: str = "synthetic_genome",
                       width: int = 80) -> None:
    with open(path, "wb") as f:
        f.write(b">" + name.encode() + b"\n")
        for i in range(0, len(genome), width):
            f.write(genome[i:i + width].tobytes() + b"\n")


def write_fasta_reads(path: str, reads: np.ndarray, prefix: str = "r") -> None:
    with open(path, "wb") as f:
        buf = []
        for i in range(reads.shape[0]):
            buf.append(b">%s%d\n%s\n" % (prefix.encode(), i, reads[i].tobytes()))
            if len(buf) >= 65536:
                f.write(b"".join(buf))
                buf = []
        f.write(b"".join(buf))


# ----------------------------------------------------------------------------
# candidate batches
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class Batch:
    """One alignment batch in the reference's call layout (one read length)."""
    m: int
    k: int
    genome: np.ndarray          # uint8, sum(L) window bytes back to back
    reads: np.ndarray           # uint8, n*m read bytes
    genome_offsets: np.ndarray  # int32 inclusive prefix sum of L
    read_offsets: np.ndarray    # int32 (t+1)*m
    edit_offsets: np.ndarray    # int32 exclusive prefix sum of (m+1)(L+1)
    dirs: np.ndarray            # int8 flags 1..3 / 5..7
    ids: np.ndarray             # int32 read ids
    pos: np.ndarray             # int32 genome positions
    match: int = 0
    mismatch: int = 1

    @property
    def n(self) -> int:
        return int(self.dirs.shape[0])

    @property
    def lengths(self) -> np.ndarray:
        go = self.genome_offsets.astype(np.int64)
        return np.diff(np.concatenate([[0], go]))

    @property
    def total_genome(self) -> int:
        """sum(L + k): the size the reference gives its alignment slot arrays."""
        return int(self.genome.shape[0]) + self.n * self.k

    @property
    def total_edit(self) -> int:
        L = self.lengths
        return int(((self.m + 1) * (L + 1)).sum())

    def slot_starts(self) -> np.ndarray:
        L = self.lengths
        return np.concatenate([[0], np.cumsum(L + self.k)[:-1]]).astype(np.int64)


def make_batch(m: int, k: int, windows: list[np.ndarray] | np.ndarray, reads: np.ndarray,
               dirs: np.ndarray, ids: np.ndarray | None = None,
               pos: np.ndarray | None = None, match: int = 0, mismatch: int = 1) -> Batch:
    n = len(dirs)
    if isinstance(windows, np.ndarray) and windows.ndim == 1:
        gbytes = windows
        L = None
    else:
        L = np.array([len(w) for w in windows], dtype=np.int64)
        gbytes = np.concatenate(windows) if n else np.zeros(0, np.uint8)
    if L is None:
        raise ValueError("pass a list of windows")
    go = np.cumsum(L).astype(np.int32)
    ro = ((np.arange(n, dtype=np.int64) + 1) * m).astype(np.int32)
    esz = (m + 1) * (L + 1)
    eo = np.concatenate([[0], np.cumsum(esz)[:-1]]).astype(np.int32) if n else np.zeros(0, np.int32)
    return Batch(m=m, k=k, genome=np.ascontiguousarray(gbytes, dtype=np.uint8),
                 reads=np.ascontiguousarray(reads.reshape(-1), dtype=np.uint8),
                 genome_offsets=go, read_offsets=ro, edit_offsets=eo,
                 dirs=np.asarray(dirs, dtype=np.int8),
                 ids=np.arange(n, dtype=np.int32) if ids is None else np.asarray(ids, np.int32),
                 pos=np.zeros(n, np.int32) if pos is None else np.asarray(pos, np.int32),
                 match=match, mismatch=mismatch)


def flank(flag: int, k: int) -> tuple[int, int]:
    """(start_offset, end_offset) of a direction/flank flag
    (src/hash.c:938-979, src/cuda-functions.cu:383-410)."""
    f = flag & 3
    so = k if f in (2, 3) else 0
    eo = k if f in (1, 3) else 0
    return so, eo


# flag mix of the reference filter, measured on its own output for C1/C2
# (fraction of candidates with flank class 1 = end free, 2 = start free,
# 3 = both free); see tests/golden/make_golden.py
DEFAULT_FLANK_MIX = (0.60, 0.0, 0.40)


def synthetic_candidates(genome: np.ndarray, rd: Reads, m: int, k: int, seed: int,
                         flank_mix=DEFAULT_FLANK_MIX, extra_hits: float = 0.0,
                         max_candidates: int | None = None) -> Batch:
    """Candidate windows placed as the q-gram filter places them: at the
    read's origin, with a flank class drawn from `flank_mix`, plus
    `extra_hits` decoy windows per read at random genome positions (the
    multi-hit candidates of repeats and the rejections of unmapped reads)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = rd.seqs.shape[0]
    G = len(genome)
    cls = rng.choice(3, size=n, p=np.asarray(flank_mix)) + 1
    so = np.where((cls == 2) | (cls == 3), k, 0)
    eo = np.where((cls == 1) | (cls == 3), k, 0)
    org = np.where(rd.origin >= 0, rd.origin, rng.integers(k, G - m - 3 * k, size=n))
    start = org - so
    nx = rng.poisson(extra_hits, size=n) if extra_hits > 0 else np.zeros(n, np.int64)
    rid = np.concatenate([np.arange(n), np.repeat(np.arange(n), nx)])
    st = np.concatenate([start, rng.integers(k, G - m - 3 * k, size=int(nx.sum()))])
    cl = np.concatenate([cls, np.repeat(cls, nx)])
    s_o = np.where((cl == 2) | (cl == 3), k, 0)
    e_o = np.where((cl == 1) | (cl == 3), k, 0)
    st = np.clip(st, 0, G - (m + s_o + e_o))
    order = rng.permutation(len(rid))
    if max_candidates is not None:
        order = order[:max_candidates]
    rid, st, cl, s_o, e_o = rid[order], st[order], cl[order], s_o[order], e_o[order]
    L = m + s_o + e_o
    go = np.cumsum(L)
    gstart = go - L
    total = int(go[-1]) if len(go) else 0
    gbytes = np.empty(total, dtype=np.uint8)
    # gather windows: index = st + (position within window)
    seg = np.repeat(np.arange(len(st)), L)
    within = np.arange(total) - np.repeat(gstart, L)
    gbytes[:] = genome[np.repeat(st, L) + within] if total else gbytes
    _ = seg
    dirs = (cl + np.where(rd.reverse[rid], 4, 0)).astype(np.int8)
    reads = rd.seqs[rid]
    # the reference aligns the reverse complement of reverse-strand reads
    # (src/hash.c:1027-1034); `rd.seqs` holds reads as sequenced, so undo it
    reads = np.where(rd.reverse[rid][:, None], reverse_complement(reads), reads)
    n_c = len(rid)
    ro = ((np.arange(n_c, dtype=np.int64) + 1) * m).astype(np.int32)
    esz = (m + 1) * (L + 1)
    eoff = (np.cumsum(esz) - esz).astype(np.int32) if n_c else np.zeros(0, np.int32)
    return Batch(m=m, k=k, genome=gbytes, reads=np.ascontiguousarray(reads.reshape(-1)),
                 genome_offsets=go.astype(np.int32), read_offsets=ro, edit_offsets=eoff,
                 dirs=dirs, ids=rid.astype(np.int32), pos=st.astype(np.int32))


def random_batch(m: int, k: int, n: int, seed: int, err: float = 0.05,
                 alphabet: bytes = b"ACGT", flags=(1, 2, 3, 5, 6, 7)) -> Batch:
    """Small random batch for parity tests: each window is the read placed at
    its flank offsets with random edits, so most pairs score <= k but many
    do not; `alphabet` may add other bytes (N) to reads and windows."""
    rng = np.random.Generator(np.random.PCG64(seed))
    alpha = np.frombuffer(alphabet, dtype=np.uint8)
    fl = rng.choice(np.asarray(flags), size=n)
    reads = alpha[rng.integers(0, len(alpha), size=(n, m))]
    windows = []
    for t in range(n):
        so, eo = flank(int(fl[t]), k)
        core = list(reads[t])
        i = 0
        out = []
        while i < len(core):
            u = rng.random()
            if u < err * 0.6:
                out.append(int(alpha[rng.integers(0, len(alpha))]))
                i += 1
            elif u < err * 0.8:
                out.append(int(alpha[rng.integers(0, len(alpha))]))
            elif u < err:
                i += 1
            else:
                out.append(int(core[i]))
                i += 1
        need = m
        out = (out + [int(a) for a in alpha[rng.integers(0, len(alpha), size=need)]])[:need]
        pre = alpha[rng.integers(0, len(alpha), size=so)]
        post = alpha[rng.integers(0, len(alpha), size=eo)]
        windows.append(np.concatenate([pre, np.asarray(out, np.uint8), post]).astype(np.uint8))
    return make_batch(m, k, windows, reads, fl.astype(np.int8))
