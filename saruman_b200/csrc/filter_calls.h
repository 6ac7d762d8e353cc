// filter_calls.h -- the reference's alignment calls from the filter's
// per-read positions (host code).
//
// The reference keeps each read's positions in a result hash (reads in the
// order they first keep a position), adds every kept position > 0 to an
// alignment queue, and after each read, once the queue exceeds the chunk
// value, submits one call (src/hash.c:840-850): every read of the hash in
// order, every position > 0 whose window m + so + eo fits the genome
// (src/hash.c:982), which it then negates so no later call repeats it.
// Positions whose window does not fit stay positive and are skipped again
// by every later call.  After the last read the rest goes out as a final
// call (src/hash.c:462).  Perfect hits (flag 0, negative positions) are
// printed by the filter itself and never aligned.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "filter_core.cuh"

namespace saru {

struct FilterCalls {
  std::vector<int64_t> call_begin;  // candidate index where each call starts (+ the end)
  std::vector<int32_t> ids, pos;
  std::vector<int8_t> dirs;
  std::vector<int32_t> perfect_ids, perfect_pos;  // in print order; pos = start (0-based)
};

class CallAssembler {
 public:
  CallAssembler(int m, int k, int64_t genome_len, uint32_t chunk_value) {
    reset(m, k, genome_len, chunk_value);
  }

  // A new run; the storage of earlier runs is kept (filling fresh memory
  // costs as much as the assembly).
  void reset(int m, int k, int64_t genome_len, uint32_t chunk_value) {
    m_ = m;
    k_ = k;
    glen_ = genome_len;
    chunk_ = chunk_value;
    queue_ = 0;
    entries_.clear();
    pos_.clear();
    flag_.clear();
    out.call_begin.assign(1, 0);
    out.ids.clear();
    out.pos.clear();
    out.dirs.clear();
    out.perfect_ids.clear();
    out.perfect_pos.clear();
  }

  // The read's kept positions, in the order the filter kept them.
  void add_read(int32_t id, const int32_t *pos, const int8_t *flag, int n, int queue) {
    if (n > 0) {
      const size_t at = pos_.size();
      entries_.push_back(Entry{id, (uint32_t)at, (uint32_t)n});
      pos_.resize(at + (size_t)n);
      flag_.resize(at + (size_t)n);
      memcpy(&pos_[at], pos, sizeof(int32_t) * (size_t)n);
      memcpy(&flag_[at], flag, (size_t)n);
      for (int i = 0; i < n; ++i)
        if (flag[i] == 0) {  // a perfect hit (kept only with a negative position)
          out.perfect_ids.push_back(id);
          out.perfect_pos.push_back(-pos[i]);
        }
    }
    queue_ += (uint32_t)queue;
    if (queue_ > chunk_) flush();
  }

  // The reads r0 .. r0 + cnt - 1 at once, in read order: read i has hn[i]
  // kept positions at pos/flag + (sum of hn before i) and queued hq[i]
  // positions.  The same calls as add_read for each read in turn: a window
  // that does not fit the genome now never fits later in the run (the limit
  // is fixed), so the pending positions add_read keeps never reach a call
  // and are not kept here; the queue threshold's flush points come from a
  // running sum of hq.  The reads' positions are counted and copied on up to
  // `nthreads` host threads.
  void add_reads(int32_t r0, long cnt, const int32_t *pos, const int8_t *flag,
                 const int32_t *hn, const int32_t *hq, int nthreads) {
    if (!entries_.empty()) {  // reads added one by one before: keep their order
      long at = 0;
      for (long i = 0; i < cnt; ++i) {
        add_read(r0 + (int32_t)i, pos + at, flag + at, hn[i], hq[i]);
        at += hn[i];
      }
      return;
    }
    if (cnt <= 0) return;
    const int nt = (int)std::max(1L, std::min<long>(nthreads, cnt / 4096 + 1));
    std::vector<int64_t> at((size_t)cnt + 1), nc((size_t)cnt + 1), np((size_t)cnt + 1);
    at[0] = 0;
    for (long i = 0; i < cnt; ++i) at[(size_t)i + 1] = at[(size_t)i] + hn[i];
    auto fits = [&](int32_t p, int8_t f) {
      int so = 0, eo = 0;
      flank_of(f, k_, so, eo);
      return (int64_t)(uint32_t)p + m_ + so + eo <= glen_;
    };
    auto parallel = [&](auto body) {
      std::vector<std::thread> th;
      for (int t = 1; t < nt; ++t) th.emplace_back(body, cnt * t / nt, cnt * (t + 1) / nt);
      body(0L, cnt / nt);
      for (auto &x : th) x.join();
    };
    // per read: candidates (positions > 0 whose window fits), perfect hits
    parallel([&](long lo, long hi) {
      for (long i = lo; i < hi; ++i) {
        int64_t c = 0, q = 0;
        for (int64_t j = at[(size_t)i]; j < at[(size_t)i + 1]; ++j) {
          if (flag[j] == 0) ++q;
          if (pos[j] > 0 && fits(pos[j], flag[j])) ++c;
        }
        nc[(size_t)i + 1] = c;
        np[(size_t)i + 1] = q;
      }
    });
    nc[0] = np[0] = 0;
    for (long i = 0; i < cnt; ++i) {
      nc[(size_t)i + 1] += nc[(size_t)i];
      np[(size_t)i + 1] += np[(size_t)i];
    }
    const int64_t c0 = (int64_t)out.ids.size(), p0 = (int64_t)out.perfect_ids.size();
    out.ids.resize((size_t)(c0 + nc[(size_t)cnt]));
    out.pos.resize(out.ids.size());
    out.dirs.resize(out.ids.size());
    out.perfect_ids.resize((size_t)(p0 + np[(size_t)cnt]));
    out.perfect_pos.resize(out.perfect_ids.size());
    parallel([&](long lo, long hi) {
      for (long i = lo; i < hi; ++i) {
        int64_t c = c0 + nc[(size_t)i], q = p0 + np[(size_t)i];
        for (int64_t j = at[(size_t)i]; j < at[(size_t)i + 1]; ++j) {
          if (flag[j] == 0) {
            out.perfect_ids[(size_t)q] = r0 + (int32_t)i;
            out.perfect_pos[(size_t)q++] = -pos[j];
          }
          if (pos[j] > 0 && fits(pos[j], flag[j])) {
            out.ids[(size_t)c] = r0 + (int32_t)i;
            out.pos[(size_t)c] = pos[j];
            out.dirs[(size_t)c++] = flag[j];
          }
        }
      }
    });
    // flush points: after read i once the queued positions exceed the
    // threshold; a call ends there if it holds a candidate
    for (long i = 0; i < cnt; ++i) {
      queue_ += (uint32_t)hq[i];
      if (queue_ > chunk_) close_call(c0 + nc[(size_t)i + 1]);
    }
  }

  void finish() {
    if (!entries_.empty() || pos_.size()) {
      if (queue_ > 0) flush();
      return;
    }
    // the last call, as add_read's finish flushes it: only when positions
    // are queued (else the candidates since the last call are never
    // submitted, as in the reference)
    if (queue_ > 0) {
      close_call((int64_t)out.ids.size());
    } else {
      const size_t end = (size_t)out.call_begin.back();
      out.ids.resize(end);
      out.pos.resize(end);
      out.dirs.resize(end);
    }
  }

  FilterCalls out;

 private:
  // a read's positions: pos_/flag_[at, at + n)
  struct Entry {
    int32_t id;
    uint32_t at, n;
  };

  // A call boundary at candidate `end` (the batched path's flush).
  void close_call(int64_t end) {
    if (end > out.call_begin.back()) out.call_begin.push_back(end);
    queue_ = 0;
  }

  void flush() {
    const int64_t before = (int64_t)out.ids.size();
    // (no reserve of size() + pending here: an exact reserve at every flush
    // reallocates and copies every earlier candidate; push_back grows
    // geometrically)
    size_t keep = 0, kept_values = 0;
    for (size_t e = 0; e < entries_.size(); ++e) {
      const Entry E = entries_[e];
      bool pending = false;
      for (uint32_t i = E.at; i < E.at + E.n; ++i) {
        if (pos_[i] <= 0) continue;
        int so = 0, eo = 0;
        flank_of(flag_[i], k_, so, eo);
        if ((int64_t)(uint32_t)pos_[i] + m_ + so + eo > glen_) {
          pending = true;  // stays positive: looked at again by later calls
          continue;
        }
        out.ids.push_back(E.id);
        out.pos.push_back(pos_[i]);
        out.dirs.push_back(flag_[i]);
        pos_[i] = -pos_[i];
      }
      // reads left with nothing positive can never contribute again; the
      // others move down to the front of the arrays
      if (pending) {
        for (uint32_t i = 0; i < E.n; ++i) {
          pos_[kept_values + i] = pos_[E.at + i];
          flag_[kept_values + i] = flag_[E.at + i];
        }
        entries_[keep++] = Entry{E.id, (uint32_t)kept_values, E.n};
        kept_values += E.n;
      }
    }
    entries_.resize(keep);
    pos_.resize(kept_values);
    flag_.resize(kept_values);
    if ((int64_t)out.ids.size() > before) out.call_begin.push_back((int64_t)out.ids.size());
    queue_ = 0;
  }

  int m_ = 0, k_ = 0;
  int64_t glen_ = 0;
  uint32_t chunk_ = 0;
  uint32_t queue_ = 0;
  std::vector<Entry> entries_;
  std::vector<int32_t> pos_;
  std::vector<int8_t> flag_;
};

}  // namespace saru
