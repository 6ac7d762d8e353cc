"""The call assembly in batches (CallAssembler::add_reads, the device
filter's path) gives exactly the calls of the reference's read-by-read
assembly (add_read, the path the host restatement pins against the
reference program): random launches of reads with kept, negated (already
submitted), perfect-hit and past-the-genome positions, queue thresholds that
split them into many calls or one, reads split over several launches."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

SRC = r'''
#include <stdio.h>
#include <stdlib.h>
#include <random>
#include "filter_calls.h"
using namespace saru;

static bool same(const FilterCalls &a, const FilterCalls &b) {
  return a.call_begin == b.call_begin && a.ids == b.ids && a.pos == b.pos && a.dirs == b.dirs &&
         a.perfect_ids == b.perfect_ids && a.perfect_pos == b.perfect_pos;
}

int main() {
  std::mt19937 rng(7);
  int bad = 0, calls = 0;
  for (int trial = 0; trial < 400; ++trial) {
    const int m = 36 + (int)(rng() % 120), k = (int)(rng() % 8);
    const int64_t glen = 5000 + (int64_t)(rng() % 100000);
    const uint32_t chunk = 1 + (uint32_t)(rng() % (trial % 3 == 0 ? 20 : 2000));
    const long nreads = 1 + (long)(rng() % 6000);
    std::vector<int32_t> hn(nreads), hq(nreads), pos;
    std::vector<int8_t> flag;
    for (long r = 0; r < nreads; ++r) {
      const int n = (rng() % 4 == 0) ? 0 : (int)(rng() % 12);
      hn[r] = n;
      int q = 0;
      for (int j = 0; j < n; ++j) {
        int8_t f = (int8_t)(rng() % 8);
        int32_t p = 1 + (int32_t)(rng() % (uint32_t)glen);
        const int u = (int)(rng() % 10);
        if (u == 0) { f = (rng() % 2) ? 0 : 4; p = -p; }      // perfect hit
        else if (u == 1) p = -p;                              // already submitted
        else if (u == 2) p = (int32_t)(glen - (rng() % 40));  // window may pass the end
        else ++q;
        pos.push_back(p);
        flag.push_back(f);
      }
      hq[r] = (rng() % 5 == 0) ? (int32_t)(rng() % 3) : q;   // the queue count as reported
    }
    CallAssembler a(m, k, glen, chunk), b(m, k, glen, chunk);
    long at = 0;
    for (long r = 0; r < nreads; ++r) {
      a.add_read((int32_t)r, pos.data() + at, flag.data() + at, hn[r], hq[r]);
      at += hn[r];
    }
    a.finish();
    // the same reads in launches of random sizes
    long r0 = 0;
    at = 0;
    while (r0 < nreads) {
      const long cnt = std::min<long>(nreads - r0, 1 + (long)(rng() % 2500));
      long np = 0;
      for (long i = 0; i < cnt; ++i) np += hn[r0 + i];
      b.add_reads((int32_t)r0, cnt, pos.data() + at, flag.data() + at, hn.data() + r0,
                  hq.data() + r0, 1 + (int)(trial % 5));
      r0 += cnt;
      at += np;
    }
    b.finish();
    if (!same(a.out, b.out)) {
      ++bad;
      printf("trial %d differs: calls %zu/%zu cand %zu/%zu\n", trial, a.out.call_begin.size(),
             b.out.call_begin.size(), a.out.ids.size(), b.out.ids.size());
    }
    calls += (int)a.out.call_begin.size() - 1;
  }
  printf("BAD %d calls %d\n", bad, calls);
  return bad != 0;
}
'''


def test_batched_assembly_equals_read_by_read(tmp_path):
    src = tmp_path / "asm.cpp"
    src.write_text(SRC)
    exe = tmp_path / "asm"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I",
                    str(ROOT / "saruman_b200" / "csrc"), str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "BAD 0" in r.stdout
    assert int(r.stdout.split("calls ")[1]) > 1000  # many calls, split at many flush points
