#!/usr/bin/env python
"""Benchmark of the B200 alignment stage (libsaruman_b200.so).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c1|c4]

Metric: candidate alignments per second (every candidate pair aligned,
including those that score above k), with GCUPS (rectangle cells m*L per
second) beside it.  Default workload: the microbial-scale configuration --
5 Mbp seeded genome at 50 % GC with 40 repeat families of 1.5 kbp (5-50
copies, 99 % identity), 2M reads of 100 bp from both strands with 3 % errors
(70/15/15), k = 5; candidate windows are placed where the reference's q-gram
filter places them (read origin, plus the same offset in every other copy of
a repeat family), ~9.5 candidates per read as the reference's filter gives
on this genome.  Synthetic data: there is no network for real data.

One step aligns one such batch.  `value` times saru_align_device on inputs
already resident in HBM (one kernel launch per step; inputs ~4 GB, larger
than L2, so no flush is needed).  `e2e` times the same batch through the
public host entry point (saru_align_host) with pinned host buffers: host
validation, H2D of the inputs, the kernels, D2H of the scores and both
alignment-slot arrays, every step (the library overlaps the copies and the
kernels in slices of the call).

With torchrun (N > 1) each rank aligns its own batch (replicas, weak
scaling); rank 0 prints the max-over-ranks timing.  `--impl reference` times
the reference's own alignment code (src/cuda-functions.cu compiled for the
host, oracle/_ref) on all host cores over a bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    "c2": dict(workload="microbial-scale plain kernel: 5 Mbp repeat-rich genome, 2M reads x 100 bp, "
               "3% errors, k=5", genome=("repeat", 5_000_000, 201, "uniform"), reads=2_000_000,
               m=100, k=5, rate=0.03, mix=(0.70, 0.15, 0.15), unmapped=0.0),
    "c1": dict(workload="small: 1 Mbp uniform genome, 100k reads x 36 bp, 2% errors, k=2",
               genome=("uniform", 1_000_000, 101), reads=100_000, m=36, k=2, rate=0.02,
               mix=(0.70, 0.15, 0.15), unmapped=0.0),
    "c4": dict(workload="long-read-end stress: 10 Mbp uniform genome, 1M reads x 250 bp, 4% errors "
               "(60/20/20), 5% unmapped, k=15", genome=("uniform", 10_000_000, 401),
               reads=1_000_000, m=250, k=15, rate=0.04, mix=(0.60, 0.20, 0.20), unmapped=0.05),
    "c3": dict(workload="batching: 5 Mbp genome with Zipf(1.5, max 500) repeat copies, 4M reads of "
               "lengths {36,75,100,150} (1M each), 3% errors, k=ceil(0.06 m); repeat hits capped at "
               "25 per read (~22M candidates of uneven count per read); all length bins in one launch",
               genome=("repeat", 5_000_000, 301, "zipf"), reads=4_000_000, lengths=(36, 75, 100, 150),
               rate=0.03, mix=(0.70, 0.15, 0.15), unmapped=0.0, max_hits=25),
    "c5": dict(workload="serving: 5 Mbp genome with Zipf(1.5, max 500) repeat copies; Poisson "
               "arrivals of requests of 1k-500k reads (log-uniform), read lengths {36,75,100,150} "
               "in equal parts, k=ceil(0.06 m), repeat hits capped at 25 per read; 60 GB device "
               "budget; continuous-batching server vs the plain per-request loop on one trace",
               genome=("repeat", 5_000_000, 301, "zipf"), reads=2_000_000,
               lengths=(36, 75, 100, 150), rate=0.03, mix=(0.70, 0.15, 0.15), unmapped=0.0,
               max_hits=25, requests=400, min_reads=1_000, max_reads=500_000, budget=60 << 30,
               load=0.8),
}


def build_batches(cfg: dict, rank: int, tables: list | None = None):
    """One batch per read-length bin (one for single-length configs); the
    sequenced reads of each bin go to `tables` when given."""
    from saruman_b200 import workloads as W
    gs = cfg["genome"]
    if gs[0] == "uniform":
        g, rmap = W.uniform_genome(gs[1], seed=gs[2]), None
    else:
        g, rmap = W.repeat_genome_with_map(gs[1], seed=gs[2], copies=gs[3])
    lengths = cfg.get("lengths", (cfg.get("m"),))
    per_bin = cfg["reads"] // len(lengths)
    out = []
    for i, m in enumerate(lengths):
        k = cfg.get("k", W.k_for(m))
        rd = W.sample_reads(g, per_bin, m, cfg["rate"], seed=1000 + 17 * rank + i, mix=cfg["mix"],
                            unmapped=cfg["unmapped"])
        out.append(W.synthetic_candidates(g, rd, m, k, seed=2000 + 17 * rank + i, repeats=rmap,
                                          max_hits=cfg.get("max_hits", 1000)))
        if tables is not None:
            tables.append(rd.seqs)
    if tables is not None:
        tables.append(g)  # the genome last
    return out


def build_batch(cfg: dict, rank: int):
    return build_batches(cfg, rank)[0]


def band_cells(b) -> int:
    """Cells of the band that must be evaluated per candidate: m*(2k+1)
    when only the end gap is free (so = 0), m*(4k+1) otherwise."""
    so_free = np.isin(b.dirs, (2, 3, 6, 7))
    per = np.where(so_free, b.m * (4 * b.k + 1), b.m * (2 * b.k + 1))
    return int(per.sum())


def rect_cells(b) -> int:
    return int((b.m * b.lengths).sum())


def algorithmic_bytes(b) -> int:
    """Bytes the stage must move per batch: read and window bytes, 9 bytes
    of offsets/flag per candidate in, 4-byte score and both alignment slots
    out."""
    return int(len(b.reads) + len(b.genome) + 9 * b.n + 4 * b.n + 2 * b.total_genome)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.3)
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""

    def summary(self) -> dict:
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


def profile_traffic() -> dict | None:
    """DRAM bytes per candidate of the banded kernel from the committed ncu
    summary (profiles/band_kernel_c2.json), if present."""
    p = ROOT / "profiles" / "band_kernel_c2.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return None
    return None


class Chunker:
    """Consecutive sub-batches of a batch, each re-based as a call of its
    own (the layout the reference's host code would build for it)."""

    def __init__(self, b):
        from saruman_b200 import workloads as W
        self.b = b
        self.W = W
        self.L = b.lengths.astype(np.int64)
        self.gend = np.cumsum(self.L)

    def take(self, start: int, count: int):
        b, W = self.b, self.W
        e = min(b.n, start + count)
        gs = int(self.gend[start - 1]) if start else 0
        ge = int(self.gend[e - 1])
        Ls = self.L[start:e]
        go = np.cumsum(Ls).astype(np.int32)
        ro = ((np.arange(e - start) + 1) * b.m).astype(np.int32)
        esz = (b.m + 1) * (Ls + 1)
        eo = (np.cumsum(esz) - esz).astype(np.int32)
        return W.Batch(m=b.m, k=b.k, genome=b.genome[gs:ge], reads=b.reads[start * b.m:e * b.m],
                       genome_offsets=go, read_offsets=ro, edit_offsets=eo, dirs=b.dirs[start:e],
                       ids=b.ids[start:e], pos=b.pos[start:e])


def cpu_reference_rate(b, seconds: float = 10.0, nthreads: int | None = None,
                       chunker: Chunker | None = None) -> dict:
    """The reference's own kernel code on the host (oracle/_ref), all host
    threads, over consecutive sub-batches of the workload until `seconds`."""
    import ctypes as C
    lib_path = ROOT / "oracle" / "_ref" / "libref_emul.so"
    if not lib_path.exists():
        return {"value": None, "unavailable": "oracle/_ref/libref_emul.so not built"}
    lib = C.CDLL(str(lib_path))
    lib.ref_align_batch.restype = C.c_int
    nthreads = nthreads or os.cpu_count() or 1
    ch = chunker or Chunker(b)
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    done = 0
    chunk = max(2000, 500 * nthreads)
    start = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds and start < b.n:
        sb = ch.take(start, chunk)
        sc = np.zeros(sb.n, np.int32)
        ra = np.zeros(sb.total_genome + 64, np.uint8)
        ga = np.zeros(sb.total_genome + 64, np.uint8)
        rc = lib.ref_align_batch(C.c_int(0), C.c_int(1), P(sb.genome), P(sb.reads),
                                 P(sb.genome_offsets), P(sb.read_offsets), P(sb.edit_offsets),
                                 C.c_int(sb.n), P(sb.dirs), C.c_int(sb.k),
                                 C.c_size_t(sb.total_genome), C.c_int(0), C.c_int(nthreads),
                                 C.c_int(256), P(sc), P(ra), P(ga))
        if rc != 0:
            return {"value": None, "unavailable": "reference host run failed"}
        done += sb.n
        start += sb.n
    dt = time.perf_counter() - t0
    return {"value": done / dt, "cores": nthreads, "candidates": done, "seconds": dt}


def run_reference_arm(args, cfg, rank: int) -> None:
    if rank != 0:
        return
    bs = build_batches(cfg, 0)
    chs = [Chunker(b) for b in bs]
    per_step = []
    for i in range(args.warmup + args.steps):
        cand, secs = 0, 0.0
        for b, ch in zip(bs, chs):
            r = cpu_reference_rate(b, seconds=args.ref_seconds / len(bs), chunker=ch)
            if r.get("value") is None:
                print(json.dumps({"impl": "reference", "unavailable": r.get("unavailable")}))
                return
            cand += r["candidates"]
            secs += r["seconds"]
            cores = r["cores"]
        if i >= args.warmup:
            per_step.append((cand, secs))
    cand = sum(c for c, _ in per_step)
    secs = sum(t for _, t in per_step)
    value = cand / secs
    line = {
        "impl": "reference", "metric": "alignments/s", "value": value, "unit": "alignments/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * secs / len(per_step), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
        "config": {"workload": cfg["workload"], "sample": "consecutive sub-batches of the "
                   f"workload, {args.ref_seconds:.0f} s of host work per step"},
        "cpu_baseline": {"value": value, "unit": "alignments/s", "cores": cores,
                         "kind": "reference", "sample": f"{cand} candidates"},
        "e2e": {"value": value, "unit": "alignments/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


class DeviceBatch:
    """A batch's inputs and outputs resident on the device, with the C-ABI
    views of them."""

    def __init__(self, b, dev, S):
        import torch
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.b = b
        self.g, self.r, self.go, self.ro, self.d = (T(b.genome), T(b.reads), T(b.genome_offsets),
                                                    T(b.read_offsets), T(b.dirs))
        self.scores = torch.zeros(b.n, dtype=torch.int32, device=dev)
        self.ra = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
        self.ga = torch.zeros(b.total_genome + 64, dtype=torch.uint8, device=dev)
        self.sb = S.SaruBatch(self.g.data_ptr(), self.r.data_ptr(), self.go.data_ptr(),
                              self.ro.data_ptr(), self.d.data_ptr(), b.n, b.k, 0, 1, 1, b.m,
                              len(b.genome), b.total_genome)
        self.sr = S.SaruResult(self.scores.data_ptr(), self.ra.data_ptr(), self.ga.data_ptr(),
                               None)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        self.h_in = [(self.g, pin(b.genome)), (self.r, pin(b.reads)), (self.go, pin(b.genome_offsets)),
                     (self.ro, pin(b.read_offsets)), (self.d, pin(b.dirs))]
        self.h_out = [(torch.empty(b.n, dtype=torch.int32).pin_memory(), self.scores),
                      (torch.empty(b.total_genome, dtype=torch.uint8).pin_memory(),
                       self.ra[:b.total_genome]),
                      (torch.empty(b.total_genome, dtype=torch.uint8).pin_memory(),
                       self.ga[:b.total_genome])]

    def h2d(self):
        for d, h in self.h_in:
            d.copy_(h, non_blocking=True)

    def d2h(self):
        for h, d in self.h_out:
            h.copy_(d, non_blocking=True)

    def bytes_in(self):
        return sum(int(h.numel() * h.element_size()) for _, h in self.h_in)

    def bytes_out(self):
        return sum(int(h.numel() * h.element_size()) for h, _ in self.h_out)


def timed(stream, fn, steps, world, dist, dev):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms / steps


def tune_bins(bs, dbs, status, sample: int = 1_000_000) -> dict:
    """Autotunes the launch shape of every (read length, k) bin on the
    first `sample` candidates of the bin itself: the cost model (trained on
    the GPU from the committed B200 sweep) ranks the shapes, the tuner
    times its top 6 and the default, and installs the fastest."""
    from saruman_b200 import autotune as A
    from saruman_b200 import costmodel as CM
    t0 = time.perf_counter()
    model = CM.trained_on_sweep()
    t_train = time.perf_counter() - t0
    out = {}
    for b, d in zip(bs, dbs):
        smp = A.Sample.wrap(b, d.sb, d.sr, status).prefix(min(b.n, sample))
        r = A.tune_bin(smp, model=model, top=6)
        out[f"{b.m},{b.k}"] = {"shape": list(r["best"]), "trials": len(r["ms"]),
                               "ms_sample": r["ms"][r["best"]],
                               "default_ms_sample": r["default_ms"]}
    out["cost_model_train_s"] = t_train
    out["tune_s"] = time.perf_counter() - t0
    return out


class RequestPool:
    """Requests of the serving trace as C-ABI views into pinned host memory.
    Each request takes a contiguous range of reads from every length bin of
    a pre-generated candidate pool (the host filter's output), one gather
    call per bin: the request's read table (reads as sequenced), and per
    candidate its read's row, window start, flag and window end offset; the
    server gathers windows and reads from its resident genome.  Outputs come
    from a pinned ring that requests release in completion order."""

    def __init__(self, bs, tables, S, ring_bytes: int):
        import torch
        self.S = S
        self.bs = bs
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        self.pt = [pin(t.reshape(-1)) for t in tables]
        self.pp = [pin(b.pos) for b in bs]
        self.pd = [pin(b.dirs) for b in bs]
        self.gend = [np.concatenate([[0], b.genome_offsets.astype(np.int64)]) for b in bs]
        self.per_bin = [t.shape[0] for t in tables]
        self.ring = torch.empty(ring_bytes, dtype=torch.uint8).pin_memory()
        self.ring_ptr = self.ring.data_ptr()
        self.ring_bytes = ring_bytes
        self.live = []  # (start, end) of outstanding requests, oldest first

    def make(self, reads: int, rng) -> dict:
        import torch
        S = self.S
        calls, gcalls, keep, cand, out_bytes, spans = [], [], [], 0, 0, []
        h2d = d2h = out_compact = d2h_compact = 0
        for i, b in enumerate(self.bs):
            r = max(1, reads // len(self.bs))
            r0 = int(rng.integers(0, max(1, self.per_bin[i] - r)))
            c0, c1 = (int(x) for x in np.searchsorted(b.ids, [r0, r0 + r]))
            n = c1 - c0
            if n == 0:
                continue
            base = int(self.gend[i][c0])
            go = (self.gend[i][c0 + 1:c1 + 1] - base).astype(np.int32)
            ri = (b.ids[c0:c1] - r0).astype(np.int32)
            t = torch.from_numpy(np.concatenate([go, ri])).pin_memory()
            keep.append(t)
            gbytes = int(go[-1])
            slots = gbytes + b.k * n
            recs = n * S.compact_record_bytes(b.m, b.k)
            spans.append((4 * n, slots + 64, recs))
            out_bytes += (4 * n + 255) // 256 * 256 + 2 * ((slots + 64 + 255) // 256 * 256)
            out_compact += (4 * n + 255) // 256 * 256 + (recs + 255) // 256 * 256
            d2h_compact += 4 * n + recs
            calls.append(S.SaruBatch(0, 0, t.data_ptr(), 0, self.pd[i].data_ptr() + c0, n, b.k,
                                     0, 1, 1, b.m, gbytes, slots))
            gcalls.append(S.SaruGatherCall(self.pt[i].data_ptr() + r0 * b.m, t.data_ptr() + 4 * n,
                                           self.pp[i].data_ptr() + 4 * c0,
                                           self.pd[i].data_ptr() + c0, t.data_ptr(), n, r, b.k,
                                           0, 1, 1, b.m, gbytes, slots))
            cand += n
            h2d += r * b.m + 13 * n
            d2h += 4 * n + 2 * slots
        return dict(calls=calls, gcalls=gcalls, keep=keep, cand=cand, out_bytes=out_bytes,
                    out_compact=out_compact, spans=spans, h2d=h2d, d2h=d2h,
                    d2h_compact=d2h_compact)

    def alloc(self, nbytes: int) -> int | None:
        """Start offset in the ring, or None while the oldest requests hold it."""
        if nbytes > self.ring_bytes:
            raise ValueError("request larger than the output ring")
        if not self.live:
            return 0
        tail, head = self.live[0][0], self.live[-1][1]
        if self.live[-1][0] >= tail:  # not wrapped: free [head, end) and [0, tail)
            if self.ring_bytes - head >= nbytes:
                return head
            return 0 if tail >= nbytes else None
        return head if tail - head >= nbytes else None  # wrapped: free [head, tail)

    def bind(self, req: dict, start: int, compact: bool = False):
        S = self.S
        p = self.ring_ptr + start
        res = []
        for n4, slots, recs in req["spans"]:
            sc = p
            p += (n4 + 255) // 256 * 256
            if compact:
                res.append(S.SaruResult(sc, p, 0, None))
                p += (recs + 255) // 256 * 256
                continue
            ra = p
            p += (slots + 255) // 256 * 256
            ga = p
            p += (slots + 255) // 256 * 256
            res.append(S.SaruResult(sc, ra, ga, None))
        self.live.append((start, start + (req["out_compact"] if compact else req["out_bytes"])))
        n = len(req["calls"])
        import ctypes as C
        req["arr_c"] = (S.SaruBatch * n)(*req["calls"])
        req["arr_r"] = (S.SaruResult * n)(*res)
        req["arr_g"] = (S.SaruGatherCall * n)(*req["gcalls"])
        req["creq"] = S.SaruRequest(req["arr_c"], req["arr_r"], n,
                                    C.cast(req["arr_g"], C.POINTER(S.SaruGatherCall)),
                                    1 if compact else 0)

    def release_oldest(self):
        self.live.pop(0)


def run_trace(S, pool: RequestPool, reqs: list, arrivals_s, pipeline: bool, budget: int,
              max_per_launch: int = 64, compact: bool = False):
    """Submits the requests at their arrival times (seconds after start;
    None = all at once) to a fresh server and returns per-request latency
    from arrival to results on the host, the makespan and the counters."""
    import ctypes as C
    import threading
    srv = S.Server(pipeline=pipeline, max_requests_per_launch=max_per_launch, max_inflight=2,
                   budget_bytes=budget)
    srv.set_genome(pool.genome)
    lib = S.load()
    tickets = [None] * len(reqs)
    done_us = [0] * len(reqs)
    lock = threading.Condition()
    t0 = time.monotonic_ns() // 1000

    def submitter():
        for q, r in enumerate(reqs):
            if arrivals_s is not None:
                delay = t0 / 1e6 + arrivals_s[q] - time.monotonic()
                if delay > 0:
                    time.sleep(delay)
            with lock:
                while True:
                    start = pool.alloc(r["out_compact"] if compact else r["out_bytes"])
                    if start is not None:
                        break
                    lock.wait()
                pool.bind(r, start, compact)
            t = C.c_int64()
            rc = lib.saru_server_submit(srv._h, C.byref(r["creq"]), C.byref(t))
            if rc != S.SARU_OK:
                raise RuntimeError(S.last_error())
            with lock:
                tickets[q] = t.value
                lock.notify_all()

    th = threading.Thread(target=submitter)
    th.start()
    st = S.RequestStats()
    for q in range(len(reqs)):
        with lock:
            while tickets[q] is None:
                lock.wait()
            t = tickets[q]
        rc = lib.saru_server_wait(srv._h, t, 3_600_000, C.byref(st))
        if rc != S.SARU_OK:
            raise RuntimeError(f"request {q}: {rc} {S.last_error()}")
        done_us[q] = st.done_us
        with lock:
            pool.release_oldest()
            lock.notify_all()
    th.join()
    groups, launches = srv.counters()
    srv.close()
    arr_us = [t0 + (int(a * 1e6) if arrivals_s is not None else 0) for a in
              (arrivals_s if arrivals_s is not None else [0] * len(reqs))]
    lat_ms = [(d - a) / 1000 for d, a in zip(done_us, arr_us)]
    makespan = (max(done_us) - t0) / 1e6
    return lat_ms, makespan, groups, launches


def run_serving(args, cfg, rank: int) -> None:
    """Serving workload: the same seeded Poisson trace through the batched
    server and the plain per-request loop, plus both at saturation."""
    import torch
    import saruman_b200 as S
    torch.cuda.set_device(0)
    tables = []
    bs = build_batches(cfg, rank, tables)
    genome = tables.pop()
    S.load()
    rng = np.random.default_rng(4242)
    nreq = args.requests or cfg["requests"]
    sizes = np.exp(rng.uniform(np.log(cfg["min_reads"]), np.log(cfg["max_reads"]), nreq))
    sizes = sizes.astype(np.int64)
    pool = RequestPool(bs, tables, S, ring_bytes=6 << 30)  # largest request: ~0.7 GB out
    pool.genome = genome
    reqs = [pool.make(int(s), rng) for s in sizes]
    n_cand = sum(r["cand"] for r in reqs)
    warm = [pool.make(100_000, rng) for _ in range(max(args.warmup, 3))]
    status = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    tuning = {}
    if not args.no_tune:
        dbs = [DeviceBatch(b, torch.device("cuda:0"), S) for b in bs]
        for d in dbs:
            d.sr.status = status.data_ptr()
        tuning = tune_bins(bs, dbs, status)
        del dbs
        torch.cuda.empty_cache()
    budget = cfg["budget"]
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(budget, free - (8 << 30)))

    # warm-up + plain capacity, closed loop
    _, mk, _, _ = run_trace(S, pool, warm, None, False, budget)
    plain_cap = sum(r["cand"] for r in warm) / mk
    run_trace(S, pool, warm, None, True, budget)

    mean_cand = n_cand / nreq
    lam = cfg["load"] * plain_cap / mean_cand  # requests per second
    gaps = rng.exponential(1.0 / lam, nreq)
    arrivals = np.cumsum(gaps) - gaps[0]
    launches0 = S.kernel_launches()
    with ClockSampler(0) as clk:
        lat_b, mk_b, groups_b, launches_b = run_trace(S, pool, reqs, arrivals, True, budget)
    lat_p, mk_p, groups_p, launches_p = run_trace(S, pool, reqs, arrivals, False, budget)
    sat_b = run_trace(S, pool, reqs, None, True, budget)
    sat_p = run_trace(S, pool, reqs, None, False, budget)
    # compact records instead of slot strings, same trace and arrivals
    lat_bc, mk_bc, _, _ = run_trace(S, pool, reqs, arrivals, True, budget, compact=True)
    lat_pc, mk_pc, _, _ = run_trace(S, pool, reqs, arrivals, False, budget, compact=True)
    sat_bc = run_trace(S, pool, reqs, None, True, budget, compact=True)
    sat_pc = run_trace(S, pool, reqs, None, False, budget, compact=True)
    launches = S.kernel_launches() - launches0

    def pct(v, p):
        return float(np.percentile(np.asarray(v), p))

    h2d = sum(r["h2d"] for r in reqs)
    d2h = sum(r["d2h"] for r in reqs)
    line = {
        "metric": "alignments/s", "value": n_cand / sat_b[1], "unit": "alignments/s",
        "n_gpus": 1, "steps": 1, "warmup": len(warm), "ms_per_step": 1000 * sat_b[1],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
        "data": "synthetic",
        "config": {"workload": cfg["workload"], "requests": nreq, "candidates": n_cand,
                   "genome": "resident on the device (saru_server_set_genome); requests carry "
                             "reads and candidate (read, position, flag, window end) arrays",
                   "reads": int(sizes.sum()), "device_budget_bytes": budget,
                   "offered_load": {"requests_per_s": lam,
                                    "alignments_per_s": lam * mean_cand,
                                    "fraction_of_plain_capacity": cfg["load"]},
                   "step": "the whole trace, submitted at once (saturation)",
                   "tuning": tuning or "default shapes",
                   "timing": "host steady clock, arrival (or submit) to results in pinned host "
                             "memory", "l2": "inputs > L2"},
        "e2e": {"value": n_cand / sat_b[1], "unit": "alignments/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "latency_ms": {"p50": pct(lat_b, 50), "p99": pct(lat_b, 99), "max": max(lat_b),
                       "throughput": n_cand / mk_b, "groups": groups_b,
                       "launches": launches_b},
        "plain": {"value": n_cand / sat_p[1], "latency_ms": {
            "p50": pct(lat_p, 50), "p99": pct(lat_p, 99), "max": max(lat_p),
            "throughput": n_cand / mk_p, "launches": launches_p},
            "what": "one request at a time, one launch per length bin, no copy/compute overlap"},
        "batched_over_plain": sat_p[1] / sat_b[1],
        "p99_plain_over_batched": pct(lat_p, 99) / pct(lat_b, 99),
        "compact": {
            "what": "the same trace with compact records (saru_request.compact) returned "
                    "instead of slot strings",
            "d2h_bytes_per_step": sum(r["d2h_compact"] for r in reqs),
            "value": n_cand / sat_bc[1], "plain_value": n_cand / sat_pc[1],
            "batched_over_plain": sat_pc[1] / sat_bc[1],
            "latency_ms": {"p50": pct(lat_bc, 50), "p99": pct(lat_bc, 99),
                           "throughput": n_cand / mk_bc},
            "plain_latency_ms": {"p50": pct(lat_pc, 50), "p99": pct(lat_pc, 99),
                                 "throughput": n_cand / mk_pc}},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c2")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (no autotuning)")
    ap.add_argument("--filter-reads", type=int, default=200_000,
                    help="reads for the device filter leg (0: skip)")
    ap.add_argument("--shape", default=None,
                    help="W,C,B: install this launch shape for every bin instead of tuning")
    ap.add_argument("--requests", type=int, default=None,
                    help="requests in the serving trace (c5)")
    ap.add_argument("--reads", type=int, default=None,
                    help="override the reads per step (smaller cases for profiling)")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.reads:
        cfg["reads"] = args.reads
        cfg["workload"] += f" (reduced to {args.reads} reads)"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, cfg, rank)
        return
    if args.config == "c5":
        if world > 1:
            raise SystemExit("the serving workload runs on one GPU")
        run_serving(args, cfg, rank)
        return

    import torch
    import torch.distributed as dist
    import saruman_b200 as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    tables = []
    bs = build_batches(cfg, rank, tables)
    genome = tables.pop()
    S.load()
    dbs = [DeviceBatch(b, dev, S) for b in bs]
    n_cand = sum(b.n for b in bs)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    for d in dbs:
        d.sr.status = status.data_ptr()
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    multi = len(dbs) > 1
    int_peak = S.int32_issue_peak() if rank == 0 else None
    # launch shapes first: the scratch sizes depend on them
    if args.shape:
        shape = tuple(int(x) for x in args.shape.split(","))
        for b in bs:
            S.set_tuning(b.m, b.k, *shape)
        tuning = {f"{b.m},{b.k}": {"shape": list(shape), "trials": 0} for b in bs}
    else:
        tuning = tune_bins(bs, dbs, status) if not args.no_tune else {}
    status.zero_()
    if multi:
        nscr = S.multi_scratch_bytes([d.sb for d in dbs])
    else:
        nscr = S.scratch_bytes(bs[0].n, bs[0].m, bs[0].k)
    scratch = torch.empty(nscr, dtype=torch.uint8, device=dev)

    def step_batched():
        if multi:
            S.align_multi_device([d.sb for d in dbs], [d.sr for d in dbs], status.data_ptr(),
                                 scratch.data_ptr(), nscr, sptr)
        else:
            S.align_device(dbs[0].sb, dbs[0].sr, scratch.data_ptr(), nscr, sptr)

    plain_scr = [S.scratch_bytes(d.b.n, d.b.m, d.b.k) for d in dbs] if multi else []
    scratch_plain = (torch.empty(max(plain_scr), dtype=torch.uint8, device=dev)
                     if multi else None)

    def step_plain():  # one launch per length bin, in order
        for d, n1 in zip(dbs, plain_scr):
            S.align_device(d.sb, d.sr, scratch_plain.data_ptr(), n1, sptr)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_batched()
    stream.synchronize()
    if int(status.item()) != 0:
        raise SystemExit(f"kernel status {int(status.item())}")

    # ---- device-resident timing: the step captured once in a CUDA graph --
    graph = torch.cuda.CUDAGraph()
    launches0 = S.kernel_launches()
    with torch.cuda.graph(graph, stream=stream):
        step_batched()
    per_step_launches = S.kernel_launches() - launches0

    def step_graph():
        with torch.cuda.stream(stream):
            graph.replay()

    step_graph()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_step = timed(stream, step_graph, args.steps, world, dist, dev)
    torch.cuda.synchronize()
    if int(status.item()) != 0:
        raise SystemExit(f"kernel status {int(status.item())}")
    launches = per_step_launches * args.steps
    value = world * n_cand / (ms_step * 1e-3)
    plain = None
    if multi:
        for _ in range(2):
            step_plain()
        stream.synchronize()
        ms_plain = timed(stream, step_plain, args.steps, world, dist, dev)
        plain = {"value": world * n_cand / (ms_plain * 1e-3), "ms_per_step": ms_plain,
                 "launches_per_step": len(dbs),
                 "what": "one launch per length bin (saru_align_device), bins in sequence"}

    # ---- end to end through the public API, host buffers ----------------
    e2e_steps = args.e2e_steps or max(1, min(args.steps, 5))

    if multi:
        e2e_what = ("pinned host buffers copied in and out around the batched launch "
                    "(saru_align_multi_device) on one stream")

        def e2e_step():
            with torch.cuda.stream(stream):
                for d in dbs:
                    d.h2d()
                step_batched()
                for d in dbs:
                    d.d2h()

        e2e_step()
        stream.synchronize()
        if world > 1:
            dist.barrier()
        e_ms = timed(stream, e2e_step, e2e_steps, world, dist, dev)
    else:
        # the library's host entry point (saru_align_host) on pinned host
        # buffers: it validates the call on the host, copies it in, aligns
        # and copies the results out, in overlapped slices; synchronous, so
        # it is timed by the host clock between device synchronisations
        e2e_what = ("saru_align_host on pinned host buffers (host validation, copies in, "
                    "kernels and copies out overlapped in slices), host clock")
        d0 = dbs[0]
        hb = dataclasses.replace(bs[0], genome=d0.h_in[0][1].numpy(), reads=d0.h_in[1][1].numpy(),
                                 genome_offsets=d0.h_in[2][1].numpy(),
                                 read_offsets=d0.h_in[3][1].numpy(), dirs=d0.h_in[4][1].numpy())
        hout = S.AlignResult(d0.h_out[0][0].numpy(), d0.h_out[1][0].numpy(),
                             d0.h_out[2][0].numpy())

        def e2e_step():
            S.align_host(hb, out=hout)

        e2e_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t_e = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e_ms = (time.perf_counter() - t_e) * 1e3 / e2e_steps
        if world > 1:
            t = torch.tensor([e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
    e2e_value = world * n_cand / (e_ms * 1e-3)

    # ---- compact result records instead of slot strings (single-bin) -----
    compact = None
    if not multi:
        d0, b0 = dbs[0], bs[0]
        rbytes = S.compact_record_bytes(b0.m, b0.k)
        rec = torch.empty(b0.n * rbytes, dtype=torch.uint8, device=dev)
        h_rec = torch.empty(b0.n * rbytes, dtype=torch.uint8).pin_memory()

        def step_compact():
            S.align_device_compact(d0.sb, d0.scores.data_ptr(), rec.data_ptr(), rbytes,
                                   status.data_ptr(), scratch.data_ptr(), nscr, sptr)

        for _ in range(2):
            step_compact()
        stream.synchronize()
        c_ms = timed(stream, step_compact, args.steps, world, dist, dev)

        # end to end through the host entry point (saru_align_host_compact)
        # on pinned buffers, sliced and overlapped like saru_align_host
        c_out = (d0.h_out[0][0].numpy(), h_rec.numpy())

        def e2e_compact():
            S.align_host_compact(hb, out=c_out)

        e2e_compact()
        torch.cuda.synchronize()
        t_c = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_compact()
        torch.cuda.synchronize()
        ce_ms = (time.perf_counter() - t_c) * 1e3 / e2e_steps
        if world > 1:
            t = torch.tensor([ce_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ce_ms = float(t.item())
        if int(status.item()) != 0:
            raise SystemExit(f"kernel status {int(status.item())} (compact)")
        # the reference's TSV lines from the records, on the host cores
        names = S.name_table([b"read%d" % i for i in range(int(b0.ids.max()) + 1)])
        t0 = time.perf_counter()
        tsv, nf, nr = S.format_tsv_compact(b0, d0.h_out[0][0].numpy(), h_rec.numpy(), rbytes,
                                           names)
        tsv_s = time.perf_counter() - t0
        tsv_leg = {"value": n_cand / tsv_s, "unit": "alignments/s", "lines": nf + nr,
                   "bytes": len(tsv), "seconds": tsv_s, "threads": os.cpu_count(),
                   "what": "saru_format_tsv_compact on the host cores (host clock): the "
                           "reference writer's lines straight from the records"}
        del tsv
        compact = {"value": world * n_cand / (c_ms * 1e-3), "ms_per_step": c_ms,
                   "record_bytes": rbytes,
                   "e2e": {"value": world * n_cand / (ce_ms * 1e-3), "unit": "alignments/s",
                           "h2d_bytes_per_step": d0.bytes_in(),
                           "d2h_bytes_per_step": 4 * b0.n + b0.n * rbytes,
                           "what": "saru_align_host_compact on pinned host buffers, host clock"},
                   "what": "saru_align_device_compact: 2-bit traceback records per candidate "
                           "instead of the slot strings; saru_expand_compact rebuilds the "
                           "slots on the host",
                   "tsv": tsv_leg}

    # ---- candidate generation on the device (the reference's q-gram filter) --
    filt = None
    if not multi and args.filter_reads:
        b0, seqs = bs[0], tables[0][:args.filter_reads]
        with S.Filter(genome, b0.m, b0.k) as f:
            f.run(seqs, 0, 4 * len(seqs) + 1000)  # warm-up: buffers sized for the run
            runs = [f.run(seqs, dr, 4 * len(seqs) + 1000) for dr in (0, 4)]
        ms = sum(r.ms for r in runs)
        filt = {"reads": int(len(seqs)), "strands": 2,
                "value": 2 * len(seqs) / (ms * 1e-3), "unit": "read-strands/s",
                "candidates_per_s": sum(len(r.ids) for r in runs) / (ms * 1e-3),
                "ms": ms, "candidates": sum(len(r.ids) for r in runs),
                "perfect_hits": sum(len(r.perfect_ids) for r in runs),
                "what": "saru_filter_run: the reference's q-gram pair filter, a warp per read, "
                        "on the first reads of the workload, both strands, calls assembled; "
                        "device time incl. read upload and copy-back of the kept positions"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    # ---- roofline --------------------------------------------------------
    peaks = measured_peaks()
    cells = sum(band_cells(b) for b in bs)
    achieved_ops = 6 * cells / (ms_step * 1e-3)
    abytes = sum(algorithmic_bytes(b) for b in bs)
    prof = profile_traffic() if args.config == "c2" else None
    traffic = None
    if prof and prof.get("dram_bytes_per_candidate"):
        traffic = prof["dram_bytes_per_candidate"] * n_cand
    roofline = {
        "bound": "int32",
        "achieved": achieved_ops / 1e12, "peak": int_peak / 1e12 if int_peak and int_peak > 0 else None,
        "unit": "Tops/s", "frac": (achieved_ops / int_peak) if int_peak and int_peak > 0 else None,
        "traffic": traffic,
        "traffic_source": "profiles/band_kernel_c2.json (ncu dram bytes per candidate, small case, "
                          "scaled by candidates)" if traffic else None,
        "peak_source": "measured live by saru_int32_issue_probe on this GPU",
        "ops_per_candidate_definition": "band cells x 6 (m*(2k+1) or m*(4k+1) cells)",
        "hbm": {"achieved_gbs": abytes / (ms_step * 1e-3) / 1e9,
                "peak_gbs": peaks.get("hbm_gbs"),
                "frac": abytes / (ms_step * 1e-3) / 1e9 / peaks["hbm_gbs"],
                "algorithmic_bytes_per_step": abytes,
                "peak_source": "MEASURED_PEAKS.json" if not peaks.get("fallback") else "fallback"},
    }
    cpu = None
    if world == 1:
        cand, secs, cores = 0, 0.0, None
        for b in bs:
            r = cpu_reference_rate(b, seconds=args.cpu_seconds / len(bs))
            if r.get("value") is None:
                cpu = {"value": None, "unavailable": r.get("unavailable")}
                break
            cand += r["candidates"]
            secs += r["seconds"]
            cores = r["cores"]
        if cpu is None:
            cpu = {"value": cand / secs, "unit": "alignments/s", "cores": cores,
                   "kind": "reference",
                   "sample": f"{cand} consecutive candidates of the workload ({len(bs)} bins), "
                             "the reference's own kernel code compiled for the host"}
    line = {
        "metric": "alignments/s", "value": value, "unit": "alignments/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
        "data": "synthetic",
        "config": {"workload": cfg["workload"], "candidates_per_step": n_cand,
                   "reads_per_step": cfg["reads"], "read_lengths": [b.m for b in bs],
                   "k": [b.k for b in bs], "parallelism": f"replicas x{world}",
                   "l2": "inputs 4+ GB > L2, no flush",
                   "tuning": tuning or "default shapes"},
        "gcups_rect": world * sum(rect_cells(b) for b in bs) / (ms_step * 1e-3) / 1e9,
        "gpu_launches": int(launches),
        "launch": "one CUDA graph replay per step "
                  f"({per_step_launches} kernel launch(es) captured)",
        "e2e": {"value": e2e_value, "unit": "alignments/s",
                "h2d_bytes_per_step": sum(d.bytes_in() for d in dbs),
                "d2h_bytes_per_step": sum(d.bytes_out() for d in dbs), "steps": e2e_steps,
                "what": e2e_what},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    if plain:
        line["plain"] = plain
        line["batched_over_plain"] = plain["ms_per_step"] / ms_step
    if filt:
        line["filter"] = filt
    if compact:
        compact["roofline_frac"] = (6 * cells / (compact["ms_per_step"] * 1e-3) / int_peak
                                    if int_peak and int_peak > 0 else None)
        line["compact"] = compact
    print(json.dumps(line))


if __name__ == "__main__":
    main()
