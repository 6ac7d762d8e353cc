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
#include "writer.h"

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

namespace {

struct Shape {
  const saru_batch *b;
  const int32_t *scores;
  const uint8_t *records;
  int64_t rb;
  int64_t slot_start(int64_t t) const {
    return (t ? b->genome_offsets[t - 1] : 0) + (int64_t)b->k * t;
  }
  int cap(int64_t t) const {
    return (int)(b->genome_offsets[t] - (t ? b->genome_offsets[t - 1] : 0)) + b->k;
  }
  const uint32_t *rec(int64_t t) const {
    return reinterpret_cast<const uint32_t *>(records + t * rb);
  }
  bool reported(int64_t t) const { return scores[t] <= b->k; }
  // the slot has no NUL: the writer's forward scans run into the next slot
  bool full(int64_t t) const { return reported(t) && (int)(rec(t)[0] & 0xFFFFu) >= cap(t); }
  // the read string holds a read byte (a DIAG or LEFT step): the writer's
  // backward scan stops inside the slot
  bool has_letter(int64_t t) const {
    if (!reported(t)) return false;
    const int n = (int)(rec(t)[0] & 0xFFFFu);
    for (int w = 0; 16 * w < n; ++w) {
      uint32_t x = rec(t)[1 + w];
      const int left = n - 16 * w;
      if (left < 16) x &= (1u << (2 * left)) - 1u;
      if (x & 0x55555555u) return true;
    }
    return false;
  }
};

struct NameTab {
  const char *names;
  int32_t stride, n;
};

const char *table_name(void *ctx, int32_t id) {
  auto *t = static_cast<NameTab *>(ctx);
  return (id >= 0 && id < t->n) ? t->names + (int64_t)id * t->stride : nullptr;
}

}  // namespace

// TSV lines of a call straight from compact records: each thread expands
// the slots of its candidate range -- widened to the slots the reference
// writer's scans can reach (backwards until a slot with a read byte,
// forwards while a slot has no NUL) -- into its own buffer and runs the
// writer there.  Output in candidate order; returns the bytes needed and
// writes min(needed, cap) bytes to out.
extern "C" int64_t saru_format_tsv_compact(const saru_batch *b, const int32_t *scores,
                                           const uint8_t *records, int64_t record_bytes,
                                           const int32_t *read_ids, const int32_t *genome_pos,
                                           int32_t read_length, const char *names,
                                           int32_t name_stride, int32_t n_names, char *out,
                                           int64_t cap, int32_t *done_fwd, int32_t *done_rev,
                                           int32_t nthreads) {
  saru::set_last_error("");
  if (!b || b->n < 0 || (b->n > 0 && (!scores || !records || !read_ids || !genome_pos)) ||
      record_bytes < 4 || (record_bytes & 3)) {
    saru::set_last_error("saru_format_tsv_compact: invalid arguments");
    return -1;
  }
  const int64_t n = b->n;
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, 64));
  if ((int64_t)nt * 64 > n) nt = (int)std::max<int64_t>(1, n / 64);
  const Shape sh{b, scores, records, record_bytes};
  NameTab tab{names, name_stride, n_names};
  std::vector<std::string> text((size_t)nt);
  std::vector<int32_t> df((size_t)nt, 0), dr((size_t)nt, 0);
  std::vector<int> bad((size_t)nt, 0);
  auto work = [&](int w) {
    const int64_t lo = n * w / nt, hi = n * (w + 1) / nt;
    if (lo >= hi) return;
    int64_t s = lo;  // back to a slot whose read string holds a read byte
    while (s > 0 && !sh.has_letter(s)) --s;
    int64_t e = hi;  // on while the last slot has no NUL
    while (e < n && sh.full(e - 1)) ++e;
    const int64_t wlo = sh.slot_start(s), whi = sh.slot_start(e - 1) + sh.cap(e - 1);
    std::vector<char> ra((size_t)(whi - wlo)), ga((size_t)(whi - wlo));
    for (int64_t t = s; t < e; ++t) {
      const int64_t at = sh.slot_start(t) - wlo;
      const int64_t gs = t ? b->genome_offsets[t - 1] : 0;
      const int64_t rs = t ? b->read_offsets[t - 1] : 0;
      const int L = (int)(b->genome_offsets[t] - gs), m = (int)(b->read_offsets[t] - rs);
      if (!sh.reported(t)) {
        memset(&ra[(size_t)at], 0, (size_t)(L + b->k));
        memset(&ga[(size_t)at], 0, (size_t)(L + b->k));
      } else if (!expand_one(sh.rec(t), b->reads + rs, b->genome + gs, m, L, b->k,
                             &ra[(size_t)at], &ga[(size_t)at])) {
        bad[(size_t)w] = 1;
        return;
      }
    }
    saru::WriterCall wc{scores, ra.data(), ga.data(), b->total_slots, b->genome_offsets,
                        genome_pos, b->dirs, read_ids, b->k, read_length, &table_name, &tab};
    wc.window_lo = wlo;
    wc.window_hi = whi;
    saru::format_range(wc, lo, hi, &text[(size_t)w], &df[(size_t)w], &dr[(size_t)w]);
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nt; ++w) th.emplace_back(work, w);
  work(0);
  for (auto &x : th) x.join();
  for (int v : bad)
    if (v) {
      saru::set_last_error("saru_format_tsv_compact: a record does not fit its candidate");
      return -1;
    }
  int64_t total = 0, at = 0;
  int32_t f = 0, r = 0;
  for (int w = 0; w < nt; ++w) {
    total += (int64_t)text[(size_t)w].size();
    f += df[(size_t)w];
    r += dr[(size_t)w];
  }
  if (out && cap > 0)
    for (int w = 0; w < nt && at < cap; ++w) {
      const int64_t len = std::min<int64_t>((int64_t)text[(size_t)w].size(), cap - at);
      memcpy(out + at, text[(size_t)w].data(), (size_t)len);
      at += len;
    }
  if (done_fwd) *done_fwd = f;
  if (done_rev) *done_rev = r;
  return total;
}
