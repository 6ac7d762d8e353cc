"""The multi-GPU path is replicas: one call split into contiguous candidate
ranges, one per rank, no collective on the data path.  Two gloo ranks on the
CPU each align their range (here with the oracle, as a stand-in for their
GPU) and rank 0 gathers the outputs: the concatenation equals the whole
call's result byte for byte, because every range after the first is
aligned as a continuation of the call."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import refkit as R  # noqa: E402
from saruman_b200 import replicas as P  # noqa: E402
from saruman_b200 import workloads as W  # noqa: E402


def align_shard(sh: P.Shard, whole: W.Batch):
    """The rank's range as its GPU would align it: the first range as a call
    of its own; a later one behind its predecessor candidate, whose output
    is dropped (the oracle's way to start a call mid-stream)."""
    if sh.first_of_call:
        s, ra, ga, st = R.oracle_align(sh.batch)
        assert st == 0
        return s, ra, ga
    lo, hi = sh.cand
    gend = np.concatenate([[0], whole.genome_offsets.astype(np.int64)])
    part = W.make_batch(whole.m, whole.k,
                        [whole.genome[gend[t]:gend[t + 1]] for t in range(lo - 1, hi)],
                        whole.reads[(lo - 1) * whole.m:hi * whole.m].reshape(-1, whole.m),
                        whole.dirs[lo - 1:hi])
    s, ra, ga, st = R.oracle_align(part)
    assert st == 0
    off = int(part.lengths[0]) + whole.k
    return s[1:], ra[off:], ga[off:]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = W.random_batch(75, 5, 301, seed=11, err=0.06)
        sh = P.shard(b, rank, world)
        out = align_shard(sh, b)
        parts = [None] * world
        dist.all_gather_object(parts, (sh.cand, sh.slots, out))
        if rank == 0:
            assert [p[0] for p in parts] == sorted(p[0] for p in parts)
            s, ra, ga = P.concat([p[2] for p in parts])
            ws, wra, wga, st = R.oracle_align(b)
            ok = (st == 0 and np.array_equal(s, ws) and np.array_equal(ra, wra)
                  and np.array_equal(ga, wga) and parts[-1][1][1] == b.total_genome)
            q.put(bool(ok))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_equal_the_whole_call():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) is True


def test_shards_cover_the_call():
    b = W.random_batch(36, 2, 103, seed=3)
    cov, slots = [], []
    for r in range(4):
        sh = P.shard(b, r, 4)
        assert sh.first_of_call == (r == 0)
        cov.append(sh.cand)
        slots.append(sh.slots)
        assert sh.batch.total_genome == sh.slots[1] - sh.slots[0]
    assert cov[0][0] == 0 and cov[-1][1] == b.n
    assert all(a[1] == c[0] for a, c in zip(cov, cov[1:]))
    assert all(a[1] == c[0] for a, c in zip(slots, slots[1:]))
    assert slots[-1][1] == b.total_genome


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3, 5])
def test_gpu_shards_equal_the_whole_call(saru_lib, world):
    """The library aligning each range (continuations with first_of_call =
    0), as the ranks of `bench.py --gpus N` would, reproduces the whole
    call's bytes."""
    import saruman_b200 as S
    b = W.random_batch(100, 5, 997, seed=21, err=0.05, alphabet=b"ACGTN")
    whole = S.align_host(b)
    parts = []
    for r in range(world):
        sh = P.shard(b, r, world)
        res = S.align_host(sh.batch, first_of_call=sh.first_of_call)
        parts.append((res.scores, res.read_aln, res.genome_aln))
    s, ra, ga = P.concat(parts)
    assert np.array_equal(s, whole.scores)
    assert np.array_equal(ra, whole.read_aln) and np.array_equal(ga, whole.genome_aln)
