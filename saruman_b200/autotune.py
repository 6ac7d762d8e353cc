"""Autotuner of the banded kernel's launch shape per (read length, k).

A shape is (warps per CTA, CTAs per SM cap, band word bits); 0 keeps the
library's default for that field.  For one (m, k) bin the tuner aligns a
sample batch of that bin with every shape of the search space, timed with
CUDA events on the device, and installs the fastest through
saru_tuning_set.  Results are identical for every shape (the parity tests
run each one); only the time differs.  The cache maps a GPU name to the
chosen shapes and the measured times, so a later process installs them
without timing again.
"""
from __future__ import annotations

import dataclasses
import json
from pathlib import Path

import numpy as np

from . import workloads as W

CACHE = Path(__file__).resolve().parent / "tuning_cache.json"


def search_space(k: int) -> list[tuple[int, int, int]]:
    """Every shape the tuner may pick for a bin with threshold k."""
    words = (32, 64) if k <= 7 else (64,)
    return [(w, c, b) for w in (1, 2, 3, 4) for c in (0, 2, 3) for b in words]


def default_shape(k: int) -> tuple[int, int, int]:
    return (0, 0, 0)


@dataclasses.dataclass
class Sample:
    """A bin's sample batch resident on the device, with its C-ABI views."""
    batch: W.Batch
    keep: list

    @staticmethod
    def build(m: int, k: int, n_reads: int, seed: int = 7, genome_len: int = 2_000_000,
              device: str = "cuda:0") -> "Sample":
        import torch
        import saruman_b200 as S
        g = W.uniform_genome(genome_len, seed=seed)
        rd = W.sample_reads(g, n_reads, m, 0.03, seed=seed + 1, unmapped=0.05)
        b = W.synthetic_candidates(g, rd, m, k, seed=seed + 2, extra_hits=3.0)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        bufs = [T(b.genome), T(b.reads), T(b.genome_offsets), T(b.read_offsets), T(b.dirs),
                torch.zeros(b.n, dtype=torch.int32, device=device),
                torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=device),
                torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=device),
                torch.zeros(1, dtype=torch.int32, device=device)]
        s = Sample(b, bufs)
        s.sb = S.SaruBatch(*[x.data_ptr() for x in bufs[:5]], b.n, b.k, 0, 1, 1, b.m,
                           len(b.genome), b.total_genome)
        s.sr = S.SaruResult(*[x.data_ptr() for x in bufs[5:9]])
        return s

    @staticmethod
    def wrap(batch: W.Batch, sb, sr, status) -> "Sample":
        """A sample over buffers the caller already holds on the device
        (`status`: a device int32 tensor the launches OR their status into)."""
        s = Sample(batch, [None] * 8 + [status])
        s.sb, s.sr = sb, sr
        return s

    def prefix(self, n: int) -> "Sample":
        """The first n candidates (a valid call of their own), same buffers."""
        import saruman_b200 as S
        b = self.batch
        n = min(n, b.n)
        ge = int(b.genome_offsets[n - 1])
        pb = W.Batch(m=b.m, k=b.k, genome=b.genome[:ge], reads=b.reads[:n * b.m],
                     genome_offsets=b.genome_offsets[:n], read_offsets=b.read_offsets[:n],
                     edit_offsets=b.edit_offsets[:n], dirs=b.dirs[:n], ids=b.ids[:n],
                     pos=b.pos[:n])
        s = Sample(pb, self.keep)
        s.sb = S.SaruBatch(self.sb.genome, self.sb.reads, self.sb.genome_offsets,
                           self.sb.read_offsets, self.sb.dirs, n, b.k, 0, 1, 1, b.m, ge,
                           ge + b.k * n)
        s.sr = self.sr
        return s

    def start_gap_fraction(self) -> float:
        return float(np.isin(self.batch.dirs, (2, 3, 6, 7)).mean())


def time_shape(sample: Sample, shape: tuple[int, int, int], reps: int = 5,
               warmup: int = 2) -> float:
    """Median milliseconds of one banded launch of the sample with `shape`."""
    import torch
    import saruman_b200 as S
    b = sample.batch
    S.set_tuning(b.m, b.k, *shape)
    try:
        nscr = S.scratch_bytes(b.n, b.m, b.k)
        scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda:0")
        stream = torch.cuda.Stream()
        times = []
        for i in range(warmup + reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            S.align_device(sample.sb, sample.sr, scratch.data_ptr(), nscr, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            if i >= warmup:
                times.append(e0.elapsed_time(e1))
        if int(sample.keep[8].item()) & S.SARU_S_OVERFLOW:
            raise RuntimeError("banded traceback overflow while tuning")
        return float(np.median(times))
    finally:
        S.clear_tuning(b.m, b.k)


def tune_bin(sample: Sample, shapes: list[tuple[int, int, int]] | None = None,
             reps: int = 5, model=None, top: int = 3) -> dict:
    """Times `shapes` (the whole search space by default; with a trained
    cost model, only its `top` best-ranked shapes) and installs the fastest.
    Returns {"best": shape, "ms": {shape: ms}, "default_ms": ms}."""
    import saruman_b200 as S
    b = sample.batch
    space = shapes or search_space(b.k)
    if model is not None:
        space = model.rank(b.m, b.k, sample.start_gap_fraction(), b.n, space)[:top]
    ms = {sh: time_shape(sample, sh, reps) for sh in space}
    dflt = default_shape(b.k)
    if dflt not in ms:
        ms[dflt] = time_shape(sample, dflt, reps)
    best = min(ms, key=lambda sh: ms[sh])  # the default shape competes too
    S.set_tuning(b.m, b.k, *best)
    return {"m": b.m, "k": b.k, "n": b.n, "best": best, "ms": ms, "default_ms": ms[dflt]}


def gpu_name() -> str:
    import torch
    p = torch.cuda.get_device_properties(0)
    return f"{p.name}/{p.multi_processor_count}sm"


def save(results: list[dict], path: Path = CACHE) -> None:
    data = json.loads(path.read_text()) if path.exists() else {}
    entry = data.setdefault(gpu_name(), {})
    for r in results:
        entry[f"{r['m']},{r['k']}"] = {"shape": list(r["best"]), "n": r["n"],
                                       "best_ms": r["ms"][r["best"]],
                                       "default_ms": r["default_ms"]}
    path.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")


def install(path: Path = CACHE) -> int:
    """Installs the cached shapes of this GPU; returns how many."""
    import saruman_b200 as S
    if not path.exists():
        return 0
    entry = json.loads(path.read_text()).get(gpu_name(), {})
    for key, v in entry.items():
        m, k = (int(x) for x in key.split(","))
        S.set_tuning(m, k, *v["shape"])
    return len(entry)
