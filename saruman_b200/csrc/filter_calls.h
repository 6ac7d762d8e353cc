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

  void finish() {
    if (queue_ > 0) flush();
  }

  FilterCalls out;

 private:
  // a read's positions: pos_/flag_[at, at + n)
  struct Entry {
    int32_t id;
    uint32_t at, n;
  };

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
