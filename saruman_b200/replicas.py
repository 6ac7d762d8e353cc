"""Replicas across GPUs: one reference-style call split into contiguous
candidate ranges, one range per rank, with no collective on the data path.

Candidates are independent except for one rule of the reference's
traceback: only candidate 0 of a call stops on row 0, every later candidate
walks along it (its loop bound is the absolute cell index,
src/cuda-functions.cu:129).  So the range of rank r > 0 is aligned as a
continuation (first_of_call = 0), and the ranks' outputs, concatenated in
rank order, are the whole call's scores and slot arrays byte for byte.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .workloads import Batch


@dataclasses.dataclass
class Shard:
    batch: Batch          # the rank's candidates, offsets re-based
    first_of_call: bool   # True only for the range that starts the call
    cand: tuple[int, int]   # candidate range in the call
    slots: tuple[int, int]  # byte range of its slots in the call's slot arrays


def shard(b: Batch, rank: int, world: int) -> Shard:
    """Rank `rank`'s contiguous share of the call (sizes differ by at most one)."""
    lo = b.n * rank // world
    hi = b.n * (rank + 1) // world
    L = b.lengths.astype(np.int64)
    gend = np.concatenate([[0], np.cumsum(L)])
    g0, g1 = int(gend[lo]), int(gend[hi])
    go = (gend[lo + 1:hi + 1] - g0).astype(np.int32)
    ro = ((np.arange(hi - lo, dtype=np.int64) + 1) * b.m).astype(np.int32)
    esz = (b.m + 1) * (L[lo:hi] + 1)
    eo = (np.cumsum(esz) - esz).astype(np.int32)
    part = Batch(m=b.m, k=b.k, genome=b.genome[g0:g1], reads=b.reads[lo * b.m:hi * b.m],
                 genome_offsets=go, read_offsets=ro, edit_offsets=eo, dirs=b.dirs[lo:hi],
                 ids=b.ids[lo:hi], pos=b.pos[lo:hi], match=b.match, mismatch=b.mismatch)
    s0 = g0 + b.k * lo
    return Shard(part, rank == 0, (lo, hi), (s0, s0 + part.total_genome))


def concat(parts: list[tuple[np.ndarray, np.ndarray, np.ndarray]]):
    """Scores and both slot arrays of the ranks, in rank order -> the call's."""
    return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
            np.concatenate([p[2] for p in parts]))
