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


_CODE = np.zeros(256, dtype=np.uint8)
_CODE[BASES] = np.arange(4, dtype=np.uint8)


def reverse_complement(seqs: np.ndarray) -> np.ndarray:
    """Reverse complement of rows of ASCII bytes; only A/C/G/T are swapped
    and other bytes (N) are kept, as in the reference (src/util.c:35-57)."""
    return _COMP[seqs[..., ::-1]]


def k_for(m: int, rate: float = 0.06) -> int:
    return int(math.ceil(rate * m))


def uniform_genome(n: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return BASES[rng.integers(0, 4, size=n, dtype=np.uint8)]


@dataclasses.dataclass
class RepeatMap:
    """Where the inserted repeat copies are: copy i of family fam[i] starts
    at start[i] and is family_len bases long (later copies may overwrite
    parts of earlier ones)."""
    fam: np.ndarray
    start: np.ndarray
    family_len: int


def repeat_genome(n: int, seed: int, families: int = 40, family_len: int = 1500,
                  copies: str = "uniform", identity: float = 0.99,
                  gc: float = 0.5) -> np.ndarray:
    """Background at the given GC content with inserted repeat families.

    copies="uniform": 5-50 copies per family (C2); copies="zipf": Zipf(1.5)
    capped at 500 (C3).  Each copy carries (1-identity) substitutions."""
    return repeat_genome_with_map(n, seed, families, family_len, copies, identity, gc)[0]


def repeat_genome_with_map(n: int, seed: int, families: int = 40, family_len: int = 1500,
                           copies: str = "uniform", identity: float = 0.99,
                           gc: float = 0.5) -> tuple[np.ndarray, RepeatMap]:
    rng = np.random.Generator(np.random.PCG64(seed))
    cfam, cstart = [], []
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    g = BASES[rng.choice(4, size=n, p=p).astype(np.uint8)]
    for fi in range(families):
        fam = BASES[rng.choice(4, size=family_len, p=p).astype(np.uint8)]
        if copies == "zipf":
            c = int(min(rng.zipf(1.5), 500))
        else:
            c = int(rng.integers(5, 51))
        for _c in range(c):
            cp = fam.copy()
            mut = rng.random(family_len) < (1.0 - identity)
            cp[mut] = BASES[(np.searchsorted(BASES, cp[mut]) + rng.integers(1, 4, mut.sum())) % 4]
            at = int(rng.integers(0, n - family_len))
            g[at:at + family_len] = cp
            cfam.append(fi)
            cstart.append(at)
    return g, RepeatMap(np.asarray(cfam, np.int64), np.asarray(cstart, np.int64), family_len)


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
        u = rng.random((c, m))
        ev = u < rate
        # event type from the same uniform draw: [0, rate*mix0) substitution,
        # then insertion, then deletion
        sub = u < rate * mix[0]
        ins = ev & ~sub & (u < rate * (mix[0] + mix[1]))
        dele = ev & ~sub & ~ins
        step = np.where(ins, 0, np.where(dele, 2, 1)).astype(np.int64)
        # genome index consumed by read position t: origin + sum(step[:t]) + dele[t]
        before = np.cumsum(step, axis=1) - step
        span_c = step.sum(axis=1) + 1
        org = rng.integers(0, G - int(span_c.max()) - 1, size=c)
        idx = org[:, None] + before + dele.astype(np.int64)
        r = genome[idx]
        r[ins] = BASES[rng.integers(0, 4, size=int(ins.sum()), dtype=np.uint8)]
        r[sub] = BASES[(_CODE[r[sub]] + rng.integers(1, 4, size=int(sub.sum()),
                                                     dtype=np.uint8)) % 4]
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


# flank-class mix of the reference filter's candidates (1 = end gap free,
# 2 = start gap free, 3 = both): about 60/0/40 on the uniform 36 bp shape and
# 45/0/55 on the repeat-rich 100 bp shape, as counted from its own output
DEFAULT_FLANK_MIX = (0.45, 0.0, 0.55)


def repeat_hits(rd: Reads, rmap: RepeatMap, max_per_read: int = 1000):
    """For reads whose source lies inside a repeat copy, the same offset in
    every other copy of that family (where the q-gram filter finds exact
    q-gram pairs).  Returns (read index, genome position) arrays."""
    order = np.lexsort((rmap.start, rmap.fam))      # copies grouped by family
    fs, cs = rmap.fam[order], rmap.start[order]
    byst = np.argsort(cs)
    o = rd.origin
    i = np.searchsorted(cs[byst], o, side="right") - 1
    ii = byst[np.maximum(i, 0)]
    inside = (o >= 0) & (i >= 0) & (o + rd.span <= cs[ii] + rmap.family_len)
    r = np.nonzero(inside)[0]
    if r.size == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    c = ii[r]                                        # index of the source copy in (fs, cs)
    f = fs[c]
    first = np.searchsorted(fs, f, side="left")
    cnt = np.minimum(np.searchsorted(fs, f, side="right") - first, max_per_read)
    tot = int(cnt.sum())
    rid = np.repeat(r, cnt)
    within = np.arange(tot) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    src = np.repeat(first, cnt) + within
    keep = src != np.repeat(c, cnt)
    off = np.repeat(o[r] - cs[c], cnt)
    return rid[keep], (cs[src] + off)[keep]


def pack_windows(genome: np.ndarray, st: np.ndarray, L: np.ndarray,
                 chunk: int = 1 << 20) -> np.ndarray:
    """genome[st[t] : st[t] + L[t]] for all t, back to back."""
    lmax = int(L.max()) if len(L) else 0
    out = np.empty(int(L.sum()), dtype=np.uint8)
    if lmax == 0:
        return out
    view = np.lib.stride_tricks.sliding_window_view(genome, lmax)
    pos = 0
    for s0 in range(0, len(st), chunk):
        s1 = min(len(st), s0 + chunk)
        rows = view[np.minimum(st[s0:s1], len(genome) - lmax)]
        # rows too close to the end: fall back to exact slices
        lens = L[s0:s1]
        if (lmax == lens).all():
            part = rows.reshape(-1)
        else:
            mask = np.arange(lmax)[None, :] < lens[:, None]
            part = rows[mask]
        near_end = st[s0:s1] > len(genome) - lmax
        out[pos:pos + len(part)] = part
        if near_end.any():
            starts = pos + np.concatenate([[0], np.cumsum(lens)[:-1]])
            for j in np.nonzero(near_end)[0]:
                a = int(st[s0 + j])
                out[starts[j]:starts[j] + lens[j]] = genome[a:a + lens[j]]
        pos += len(part)
    return out


def synthetic_candidates(genome: np.ndarray, rd: Reads, m: int, k: int, seed: int,
                         flank_mix=DEFAULT_FLANK_MIX, extra_hits: float = 0.0,
                         repeats: RepeatMap | None = None,
                         max_candidates: int | None = None, max_hits: int = 1000) -> Batch:
    """Candidate windows placed as the q-gram filter places them: at the
    read's origin, with a flank class drawn from `flank_mix`; with a repeat
    map, also at the same offset of every other copy of the read's repeat
    family; plus `extra_hits` decoy windows per read at random positions
    (the rejections of reads without a true origin)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = rd.seqs.shape[0]
    G = len(genome)
    cls = rng.choice(3, size=n, p=np.asarray(flank_mix)) + 1
    so = np.where((cls == 2) | (cls == 3), k, 0)
    org = np.where(rd.origin >= 0, rd.origin, rng.integers(k, G - m - 3 * k, size=n))
    start = org - so
    nx = rng.poisson(extra_hits, size=n) if extra_hits > 0 else np.zeros(n, np.int64)
    rid = np.concatenate([np.arange(n), np.repeat(np.arange(n), nx)])
    st = np.concatenate([start, rng.integers(k, G - m - 3 * k, size=int(nx.sum()))])
    cl = np.concatenate([cls, np.repeat(cls, nx)])
    if repeats is not None:
        hr, hp = repeat_hits(rd, repeats, max_per_read=max_hits)
        hc = rng.choice(3, size=len(hr), p=np.asarray(flank_mix)) + 1
        hso = np.where((hc == 2) | (hc == 3), k, 0)
        rid = np.concatenate([rid, hr])
        st = np.concatenate([st, hp - hso])
        cl = np.concatenate([cl, hc])
    s_o = np.where((cl == 2) | (cl == 3), k, 0)
    e_o = np.where((cl == 1) | (cl == 3), k, 0)
    st = np.clip(st, 0, G - (m + s_o + e_o))
    # candidates grouped by read, as the reference's collection loop emits
    # them (src/hash.c:926-1082)
    order = np.argsort(rid, kind="stable")
    if max_candidates is not None:
        order = order[:max_candidates]
    rid, st, cl, s_o, e_o = rid[order], st[order], cl[order], s_o[order], e_o[order]
    L = m + s_o + e_o
    go = np.cumsum(L)
    gbytes = pack_windows(genome, st, L)
    dirs = (cl + np.where(rd.reverse[rid], 4, 0)).astype(np.int8)
    # the reference aligns the reverse complement of reverse-strand reads
    # (src/hash.c:1027-1034); `rd.seqs` holds reads as sequenced, so undo it
    fwd = rd.seqs.copy()
    fwd[rd.reverse] = reverse_complement(fwd[rd.reverse])
    reads = fwd[rid]
    n_c = len(rid)
    ro = ((np.arange(n_c, dtype=np.int64) + 1) * m).astype(np.int32)
    esz = (m + 1) * (L.astype(np.int64) + 1)
    ecum = np.cumsum(esz) - esz
    # the reference's int edit offsets; batches past 2^31 cells cannot be one
    # reference call and carry -1 (the banded path does not read them)
    eoff = ecum.astype(np.int32) if n_c and ecum[-1] + esz[-1] < 2**31 else np.full(n_c, -1, np.int32)
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


def chunk_value_for(m: int, k: int) -> int:
    """The reference's queue threshold (-s, candidates per call) for read
    length m: calls stay under 2^31 matrix cells and a 4 GiB arena, as a
    run of the reference must (about 1.2M candidates at 36 bp, 180k at
    100 bp, 28k at 250 bp)."""
    return int(0.92 * 2**31 / ((m + 1) * (m + 2 * k + 1))) // 1000 * 1000


@dataclasses.dataclass
class CallSet:
    """Calls of one read length as the reference's q-gram filter submits
    them (src/hash.c:840-850, 1094-1098), stored back to back: call c holds
    candidates call_begin[c] .. call_begin[c + 1]; its offsets restart at 0
    (each call is a reference call of its own, candidate 0 opening it), its
    windows start at byte gbase[c], its reads at rbase[c] and its slots at
    sbase[c] of the set's slot arrays."""
    m: int
    k: int
    genome: np.ndarray          # uint8 windows of all calls
    reads: np.ndarray           # uint8 reads of all calls, as aligned
    genome_offsets: np.ndarray  # int32, per call inclusive prefix sums of L
    read_offsets: np.ndarray    # int32, per call (t - begin + 1) * m
    edit_offsets: np.ndarray    # int32, per call exclusive prefix sums of (m+1)(L+1)
    dirs: np.ndarray
    ids: np.ndarray
    pos: np.ndarray
    call_begin: np.ndarray      # int64, ncalls + 1
    strand: np.ndarray          # int8 per call: 0 forward, 4 reverse (do_reverse)
    gbase: np.ndarray           # int64, ncalls + 1
    sbase: np.ndarray           # int64, ncalls + 1
    perfect: int = 0            # perfect hits the filter printed (never aligned)
    filter_ms: float = 0.0      # device time of the filter runs that made the calls

    @property
    def n(self) -> int:
        return int(self.dirs.shape[0])

    @property
    def ncalls(self) -> int:
        return int(self.call_begin.shape[0]) - 1

    @property
    def total_slots(self) -> int:
        return int(self.sbase[-1])

    @property
    def total_genome(self) -> int:
        """sum(L + k) over all calls (the Batch name of the slot bytes)."""
        return self.total_slots

    @property
    def lengths(self) -> np.ndarray:
        so = np.where(np.isin(self.dirs & 3, (2, 3)), self.k, 0)
        eo = np.where(np.isin(self.dirs & 3, (1, 3)), self.k, 0)
        return (self.m + so + eo).astype(np.int64)

    def call(self, c: int) -> Batch:
        """Call c as a Batch (views into the set's arrays)."""
        a, b = int(self.call_begin[c]), int(self.call_begin[c + 1])
        m = self.m
        return Batch(m=m, k=self.k, genome=self.genome[self.gbase[c]:self.gbase[c + 1]],
                     reads=self.reads[a * m:b * m], genome_offsets=self.genome_offsets[a:b],
                     read_offsets=self.read_offsets[a:b], edit_offsets=self.edit_offsets[a:b],
                     dirs=self.dirs[a:b], ids=self.ids[a:b], pos=self.pos[a:b])


def callset(genome: np.ndarray, seqs: np.ndarray, m: int, k: int, ids: np.ndarray,
            pos: np.ndarray, dirs: np.ndarray, call_begin: np.ndarray,
            strand: np.ndarray, perfect: int = 0) -> CallSet:
    """A CallSet from per-candidate (read id, window start, flag) in call
    order: windows cut from `genome` (m + so + eo bytes from the start,
    src/hash.c:986-1024), reads taken from `seqs` (as sequenced) and
    reverse-complemented for flags 4-7 (src/hash.c:1027-1034)."""
    dirs = np.asarray(dirs, np.int8)
    n = len(dirs)
    so = np.where(np.isin(dirs & 3, (2, 3)), k, 0)
    eo = np.where(np.isin(dirs & 3, (1, 3)), k, 0)
    L = (m + so + eo).astype(np.int64)
    cb = np.asarray(call_begin, np.int64)
    call_of = np.repeat(np.arange(len(cb) - 1), np.diff(cb))
    gcum = np.cumsum(L)
    gbase = np.concatenate([[0], gcum[cb[1:] - 1]]) if n else np.zeros(len(cb), np.int64)
    goff = (gcum - gbase[call_of]).astype(np.int32)
    t_in = np.arange(n, dtype=np.int64) - cb[call_of]
    roff = ((t_in + 1) * m).astype(np.int32)
    esz = (m + 1) * (L + 1)
    ecum = np.cumsum(esz)
    ebase = np.concatenate([[0], ecum[cb[1:] - 1]]) if n else np.zeros(len(cb), np.int64)
    eoff64 = ecum - esz - ebase[call_of]
    eoff = np.where(eoff64 + esz < 2**31, eoff64, -1).astype(np.int32)
    rd = np.ascontiguousarray(seqs[np.asarray(ids)])
    rev = dirs > 3
    if rev.any():
        rd[rev] = reverse_complement(rd[rev])
    sbase = gbase + k * cb
    return CallSet(m=m, k=k, genome=pack_windows(genome, np.asarray(pos, np.int64), L),
                   reads=rd.reshape(-1), genome_offsets=goff, read_offsets=roff,
                   edit_offsets=eoff, dirs=dirs, ids=np.asarray(ids, np.int32),
                   pos=np.asarray(pos, np.int32), call_begin=cb,
                   strand=np.asarray(strand, np.int8), gbase=gbase.astype(np.int64),
                   sbase=sbase.astype(np.int64), perfect=perfect)


def filter_callset(genome: np.ndarray, seqs: np.ndarray, m: int, k: int,
                   chunk_value: int | None = None, device: int = -1) -> CallSet:
    """The calls the reference's q-gram filter makes for reads `seqs` (one
    read batch, ids from 0) on both strands, from the library's device
    filter (saru_filter_*, the reference's filter on the GPU): forward
    strand calls first, then the reverse strand's, as the two strand
    threads submit them."""
    from . import Filter
    cv = chunk_value or chunk_value_for(m, k)
    parts = []
    with Filter(genome, m, k, device) as f:
        for dr in (0, 4):
            parts.append((dr, f.run(seqs, dr, cv)))
    ms = sum(p.ms for _, p in parts)
    ids = np.concatenate([p.ids for _, p in parts])
    pos = np.concatenate([p.pos for _, p in parts])
    dirs = np.concatenate([p.dirs for _, p in parts])
    cb, strand, off = [0], [], 0
    for dr, p in parts:
        cb.extend((p.call_begin[1:] + off).tolist())
        strand.extend([dr] * (len(p.call_begin) - 1))
        off += len(p.ids)
    perfect = sum(len(p.perfect_ids) for _, p in parts)
    cs = callset(genome, seqs, m, k, ids, pos, dirs, np.asarray(cb, np.int64),
                 np.asarray(strand, np.int8), perfect)
    cs.filter_ms = ms
    return cs
