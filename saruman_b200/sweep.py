"""Measures the banded kernel's time for every launch shape of the
autotuner's search space over a grid of (read length, k, candidates) bins
on the current GPU: the training data of the autotuner's cost model
(tuning_sweep_b200.json beside this file was made on a B200 with

    python -m saruman_b200.sweep OUT.json

and copied here).
"""
from __future__ import annotations

import json
import math
import sys
import time
from pathlib import Path

import saruman_b200 as S
from saruman_b200 import autotune as A

LENGTHS = (36, 50, 75, 100, 125, 150, 200, 250)
RATES = (0.03, 0.06, 0.10)
SIZES = (16_000, 128_000, 1_000_000)


def main(out: str) -> None:
    S.load()
    S.clear_tuning()
    rows = []
    t0 = time.time()
    for m in LENGTHS:
        ks = sorted({min(15, max(1, math.ceil(r * m))) for r in RATES})
        for k in ks:
            if m <= 3 * k:
                continue
            full = A.Sample.build(m, k, max(SIZES) // 4 + 1000, seed=1000 + m * 16 + k)
            for n in SIZES:
                smp = full.prefix(n)
                for shape in A.search_space(k):
                    ms = A.time_shape(smp, shape, reps=5)
                    rows.append({"m": m, "k": k, "n": smp.batch.n,
                                 "so_frac": smp.start_gap_fraction(), "shape": list(shape),
                                 "ms": ms})
            print(f"m={m} k={k} done, {len(rows)} rows, {time.time() - t0:.0f} s", flush=True)
    Path(out).write_text(json.dumps({"gpu": A.gpu_name(), "rows": rows}) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
