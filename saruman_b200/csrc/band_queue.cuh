// band_queue.cuh -- lane functions of the banded kernel's queued form.
//
// In the queued form a warp's traceback walks do not run per tile.  After a
// tile's fill, its candidates that score <= k (the only ones the reference
// traces) join a per-warp job queue, and the warp walks 32 queued jobs at a
// time, so the walks run on full warps whatever share of a tile survives
// (46% of a C2 tile scores above k and would idle through a per-tile walk).
//
// * Decision planes live in per-warp plane slots: kQueueSlots per warp, at
//   most 31 held by queued jobs when a fill starts, so a fill always finds
//   32 free slots (one per lane, the lane-th free slot of the warp's mask).
//   A lane whose candidate does not survive frees its slot after the fill;
//   a job frees its slot after its walk.
// * Queue entries (8 bytes: the candidate index, its plane slot, so/eo and
//   m) are held in registers, two per lane (entries l and 32 + l); a fill
//   appends its survivors by shuffles, a pass of 32 moves the upper half
//   down.
// * A walk writes the job's steps as a compact record (2 bits a step; the
//   format of lane_traceback_ops): straight to the caller's records in
//   compact mode, into the warp's region (strided by lane) in slot mode.
// * Slot mode: at the fill, the warp zero-fills the tile's slot ranges in
//   global memory (the reference's memset arena: slots of candidates that
//   score > k stay zero); after a walk pass the warp expands each walked
//   job's record into its slot strings cooperatively: the 32 lanes take 4
//   consecutive string positions each, a warp prefix sum of the steps'
//   column and row advances gives every position its read and window byte.
//
// The functions below are those phases as functions of the lane, shared by
// the kernel (kernels.cu) and the host emulation of its warp loop
// (tests/harness/tile_host.cpp).
#pragma once
#include <stdint.h>

#include "band_tile.cuh"

namespace saru {

constexpr int kQueueSlots = 64;  // plane slots per warp

struct QEntry {
  int32_t t;      // candidate index in its segment's arrays
  uint32_t info;  // bits 0-7 plane slot, 8 so != 0, 9 eo != 0, 10-19 m
};

SARU_HD QEntry make_entry(long t, int slot, const Cand &c) {
  return QEntry{(int32_t)t, (uint32_t)slot | (c.so ? 0x100u : 0u) | (c.eo ? 0x200u : 0u) |
                                ((uint32_t)c.m << 10)};
}

SARU_HD int entry_slot(const QEntry &e) { return (int)(e.info & 0xFFu); }

// The candidate of a queued job (regular: L = m + so + eo, checked at the fill).
SARU_HD Cand entry_cand(const QEntry &e, int k, int first_of_call) {
  Cand c;
  c.k = k;
  c.m = (int)((e.info >> 10) & 0x3FFu);
  c.so = (e.info & 0x100u) ? k : 0;
  c.eo = (e.info & 0x200u) ? k : 0;
  c.L = c.m + c.so + c.eo;
  c.first_of_call = first_of_call && e.t == 0;
  return c;
}

SARU_HD int popc32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}

// Position of the n-th (from 0) set bit of x; x has more than n set bits.
SARU_HD int nth_set_bit(uint32_t x, int n) {
  int pos = 0;
  for (int w = 16; w; w >>= 1) {
    const int c = popc32(x & ((1u << w) - 1u));
    if (n >= c) {
      n -= c;
      x >>= w;
      pos += w;
    }
  }
  return pos;
}

// The plane slot lane `lane` fills into: the lane-th free slot of the warp
// (`free_mask` has at least 32 set bits when a fill starts).
SARU_HD int fill_slot(uint64_t free_mask, int lane) {
  const uint32_t lo = (uint32_t)free_mask, hi = (uint32_t)(free_mask >> 32);
  const int nlo = popc32(lo);
  return lane < nlo ? nth_set_bit(lo, lane) : 32 + nth_set_bit(hi, lane - nlo);
}

// Writes zeros over global dst[lo, hi): 16-byte stores where the address
// is aligned, bytes at the edges (the ranges of neighbouring tiles are
// never touched).
template <class Store16Zero>
SARU_HD void zero_range(uint8_t *dst, long lo, long hi, int lane, Store16Zero st16z) {
  // first / last 16-aligned global address in the range, as indices
  const long first = lo + (long)((16u - ((uintptr_t)(dst + lo) & 15u)) & 15u);
  const long last = hi - (long)((uintptr_t)(dst + hi) & 15u);
  if (first >= last) {
    for (long x = lo + lane; x < hi; x += 32) dst[x] = 0;
    return;
  }
  for (long x = lo + lane; x < first; x += 32) dst[x] = 0;
  const long nv = (last - first) >> 4;
  for (long i = lane; i < nv; i += 32) st16z(dst + first + 16 * i);
  for (long x = last + lane; x < hi; x += 32) dst[x] = 0;
}

// The walk of one job into a compact record: store(w, v) receives words
// 1.. (2-bit steps, 16 a word, traceback order), zeros up to word
// `pad_words` - 1 (0: no padding), and word 0 (step count, bit 16 set if
// the walk left its band or slot).  Returns where it ended.
template <typename T, class LoadPair, class StoreWord>
SARU_HD WalkEnd walk_record(const Cand &c, LoadPair ld, StoreWord store, int pad_words = 0) {
  uint32_t acc = 0;
  int sh = 0, w = 1;
  const WalkEnd e = lane_walk<T>(c, ld, [&](int, uint32_t op, int, int) {
    acc |= op << sh;
    sh += 2;
    if (sh == 32) {
      store(w++, acc);
      acc = 0;
      sh = 0;
    }
  });
  if (sh) store(w++, acc);
  for (; w < pad_words; ++w) store(w, 0u);
  store(0, (uint32_t)e.n | (e.bad ? 0x10000u : 0u));
  return e;
}

// Words between walked records in the warp's region: record j at word
// j * stride.  Odd, so the lanes writing the same word of their records
// hit different banks, and the words of one record are in different banks.
SARU_HD int rec_stride(int max_m, int k) { return (int)(1 + step_words(max_m, k)) | 1; }

// Cooperative expansion of one walked job into its slot strings, round by
// round (a round covers 128 string positions, 4 per lane).  Positions are
// in reading order: position p holds step n - 1 - p of the record.  A DIAG
// step (1) puts read byte `col` against window byte `row`, UP (2) a gap in
// the read against window byte `row`, LEFT (3) read byte `col` against a
// gap; DIAG and LEFT advance the column, DIAG and UP the row, starting from
// the cell where the walk stopped.

// Step of the record at string position p (p < n).  word(w) returns record
// word w.
template <class Word>
SARU_HD uint32_t step_at(Word word, int n, int p) {
  const int s = n - 1 - p;
  return (word(1 + (s >> 4)) >> ((s & 15) * 2)) & 3u;
}

// Column and row advances of lane `lane`'s four positions of a round,
// packed as col | row << 16.
template <class Word>
SARU_HD uint32_t expand_advance(Word word, int n, int base, int lane) {
  uint32_t cc = 0, rr = 0;
  for (int i = 0; i < 4; ++i) {
    const int p = base + 4 * lane + i;
    if (p < n) {
      const uint32_t op = step_at(word, n, p);
      cc += op & 1u;
      rr += (op != 3u) ? 1u : 0u;
    }
  }
  return cc | (rr << 16);
}

// Writes lane `lane`'s four positions; col/row are the read and window
// indices of its first position.  rd(i) / wn(i) read byte i of the read /
// window; out(p, a, b) writes string position p.
template <class Word, class Rd, class Wn, class Out>
SARU_HD void expand_write(Word word, int n, int base, int lane, int col, int row, Rd rd, Wn wn,
                          Out out) {
  for (int i = 0; i < 4; ++i) {
    const int p = base + 4 * lane + i;
    if (p >= n) break;
    const uint32_t op = step_at(word, n, p);
    const uint8_t a = (op & 1u) ? rd(col) : uint8_t('_');
    const uint8_t b = (op != 3u) ? wn(row) : uint8_t('_');
    out(p, a, b);
    col += (int)(op & 1u);
    row += (op != 3u) ? 1 : 0;
  }
}

// Shared-memory slice of the queued form: [reads staging][windows staging]
// [region: codes + masks during a fill, walked records during a pass].
SARU_HD SliceLayout queue_slice_layout(int max_m, int k) {
  SliceLayout L = slice_layout(max_m, k);
  const long code_words = (max_m + 7) / 8;
  const long mwords = mask_words(k, max_m + 2 * k);
  const long cm = 4L * 32 * (code_words + NCODES * mwords);
  const long rec = 4L * 32 * rec_stride(max_m, k);
  L.region_bytes = ((cm > rec ? cm : rec) + 15) & ~15L;
  L.warp_smem = L.rs_bytes + L.ws_bytes + L.region_bytes;
  return L;
}

}  // namespace saru
