// compact.cpp -- host expansion of compact result records into the
// reference's slot strings (the layout src/cuda-functions.cu:807-824 copies
// back), byte for byte what the banded kernel writes in slot mode.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/saruman_b200.h"
#include "server_internal.h"

namespace {

// Slot of one candidate: the steps in reading order from the cell where the
// traceback stopped, zeros after them.  Returns false if the record does not
// fit the candidate (more steps than its slot, or a walk off its matrix).
bool expand_one(const uint32_t *rec, const char *read, const char *win, int m, int L, int k,
                char *slot_r, char *slot_g) {
  const int cap = L + k;
  const uint32_t hdr = rec[0];
  const int n = (int)(hdr & 0xFFFFu);
  memset(slot_r, 0, (size_t)cap);
  memset(slot_g, 0, (size_t)cap);
  if (n > cap || (hdr & 0x10000u)) return false;
  int row = L, col = m;
  for (int st = 0; st < n; ++st) {
    const uint32_t op = (rec[1 + (st >> 4)] >> (2 * (st & 15))) & 3u;
    const int at = n - 1 - st;  // the string is stored in reading order
    if (op == 1u) {             // DIAG
      if (row < 1 || col < 1) return false;
      slot_r[at] = read[col - 1];
      slot_g[at] = win[row - 1];
      --row;
      --col;
    } else if (op == 2u) {  // UP: gap in the read
      if (row < 1) return false;
      slot_r[at] = '_';
      slot_g[at] = win[row - 1];
      --row;
    } else if (op == 3u) {  // LEFT: gap in the window
      if (col < 1) return false;
      slot_r[at] = read[col - 1];
      slot_g[at] = '_';
      --col;
    } else {
      return false;
    }
  }
  return true;
}

}  // namespace

namespace saru {

// Records from slot strings (the inverse of expand_one): the steps are the
// string's columns in reverse (traceback) order -- '_' in the read string an
// UP step, '_' in the window string a LEFT step, else DIAG.
int records_from_slots(const saru_batch *b, const int32_t *scores, const char *read_aln,
                       const char *genome_aln, uint8_t *records, long record_bytes) {
  for (int64_t t = 0; t < b->n; ++t) {
    const int64_t gs = t ? b->genome_offsets[t - 1] : 0;
    const int L = (int)(b->genome_offsets[t] - gs);
    const int cap = L + b->k;
    const char *sr = read_aln + gs + (int64_t)b->k * t;
    const char *sg = genome_aln + gs + (int64_t)b->k * t;
    uint32_t *rec = reinterpret_cast<uint32_t *>(records + t * record_bytes);
    memset(rec, 0, (size_t)record_bytes);
    if (scores[t] > b->k) continue;
    int n = 0;
    while (n < cap && sr[n] != 0) ++n;
    if (4 + 4 * ((n + 15) / 16) > record_bytes) {
      set_last_error("records_from_slots: a string longer than its record");
      return SARU_E_INVALID;
    }
    for (int i = 0; i < n; ++i) {
      const uint32_t op = sr[i] == '_' ? 2u : (sg[i] == '_' ? 3u : 1u);
      const int st = n - 1 - i;
      rec[1 + (st >> 4)] |= op << (2 * (st & 15));
    }
    rec[0] = (uint32_t)n;
  }
  return SARU_OK;
}

}  // namespace saru

extern "C" int saru_expand_compact(const saru_batch *b, const int32_t *scores,
                                   const uint8_t *records, int64_t record_bytes, char *read_aln,
                                   char *genome_aln, int32_t nthreads) {
  saru::set_last_error("");
  if (!b || b->n < 0 || (b->n > 0 && (!scores || !records || !read_aln || !genome_aln)) ||
      record_bytes < 4 || (record_bytes & 3)) {
    saru::set_last_error("saru_expand_compact: invalid arguments");
    return SARU_E_INVALID;
  }
  const int64_t n = b->n;
  if (n == 0) return SARU_OK;
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if ((int64_t)nt * 4096 > n) nt = (int)std::max<int64_t>(1, n / 4096);
  std::vector<int> bad((size_t)nt, 0);
  auto work = [&](int w) {
    const int64_t lo = n * w / nt, hi = n * (w + 1) / nt;
    for (int64_t t = lo; t < hi; ++t) {
      const int64_t gs = t ? b->genome_offsets[t - 1] : 0;
      const int64_t rs = t ? b->read_offsets[t - 1] : 0;
      const int L = (int)(b->genome_offsets[t] - gs), m = (int)(b->read_offsets[t] - rs);
      const int64_t slot = gs + (int64_t)b->k * t;
      char *sr = read_aln + slot, *sg = genome_aln + slot;
      const uint32_t *rec = reinterpret_cast<const uint32_t *>(records + t * record_bytes);
      if (scores[t] > b->k) {  // no traceback: the kernel leaves the slot zero
        memset(sr, 0, (size_t)(L + b->k));
        memset(sg, 0, (size_t)(L + b->k));
        continue;
      }
      if (!expand_one(rec, b->reads + rs, b->genome + gs, m, L, b->k, sr, sg)) bad[(size_t)w] = 1;
    }
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nt; ++w) th.emplace_back(work, w);
  work(0);
  for (auto &x : th) x.join();
  for (int v : bad)
    if (v) {
      saru::set_last_error("saru_expand_compact: a record does not fit its candidate");
      return SARU_E_INVALID;
    }
  return SARU_OK;
}
