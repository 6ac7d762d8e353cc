// filter_core.cuh -- the q-gram pair filter of one read (host and device).
//
// The reference's filter (src/hash.c:348-839) emits, per read and strand,
// the genome positions the aligner is asked to check, with a flag that sets
// the free gaps of the window (1/5: end gap, 2/6: start gap, 3/7: both).
// Its candidate stream decides which alignments exist, their order inside a
// call and, through the queue flushes, where calls begin (and with them the
// first-of-call rule of the traceback), so it is restated here step by step:
//
//  * q-grams of the read at q-gram start positions qpos[0..P): the first
//    half at 0, q, 2q, ...; the second at m - q, m - 2q, ... (src/saruman.c
//    :46-75); their genome positions come from the q-gram index in genome
//    order (src/util.c:462-480), laid out per read chunk as the reference's
//    data array: each list, then a 0 (src/hash.c:404-457).  A position 0
//    reads as the end of its list, as it does there.
//  * for each first-half q-gram a and each of its positions: the read's
//    start genome_start = pos - (a q + 1); a perfect match of the read at
//    genome_start + 1 is recorded as a hit at -(genome_start + 1) (flag 0);
//    then pairs with the later first-half q-grams (error zones -k..k; the
//    scan of each pair's list starts at the index of a's current position,
//    not at 0, exactly as the reference indexes it) and with every
//    second-half q-gram (zones of half-width |half - 1 - b - a|); every pair
//    found raises a counter, and the candidate is recorded when the counter
//    reaches the threshold (src/hash.c:472-807).
//  * recording (src/hash.c:43-176): a read's first position is kept; a later
//    one is dropped if it lies within -k..k of a kept one (or of its negation)
//    with a flag not above its own, replaces the flag of an equal position on
//    the same strand with a lower one, is dropped on an equal position (or
//    negation) on the same strand, else appended; every kept position > 0
//    adds 1 to the alignment queue.
// Comparisons follow the reference's unsigned 32-bit arithmetic.
#pragma once
#include <math.h>
#include <stdint.h>

#include "saru_core.cuh"

namespace saru {

constexpr int kFilterMaxQgrams = 64;

struct FilterShape {
  int m, k, q, P, half, rest, tresh;
  int qpos[kFilterMaxQgrams];
};

// The filter's parameters for reads of length m with up to k errors, in
// the reference's float arithmetic (src/saruman.c:46-75,119).  Returns
// false if the q-gram layout does not fit (q < 1 or more than 64 q-grams).
SARU_HD bool filter_shape(int m, int k, FilterShape *S) {
  S->m = m;
  S->k = k;
  S->q = (int)ceilf((float)m / (float)(k + 1)) - 1;
  if (S->q < 1) return false;
  S->rest = m % S->q;
  const int n1 = m / S->q;
  S->P = S->rest ? 2 * n1 : n1;
  if (S->P > kFilterMaxQgrams) return false;
  S->half = S->P / 2;
  int x = 0;
  for (; x < n1; ++x) S->qpos[x] = x * S->q;
  for (int z = 1; z <= n1 && x < S->P; ++z, ++x) S->qpos[x] = m - z * S->q;
  S->tresh = (int)floorf((float)m / (float)S->q) - k + 1;
  return true;
}

// Positions kept for one read, in the order the reference keeps them.
struct ReadHits {
  int32_t *pos;   // capacity cap
  int8_t *flag;
  int cap;
  int n;          // kept positions
  int queue;      // of them > 0 (the alignment queue increments)
  int overflow;   // more than cap positions
};

// add_start_position (src/hash.c:43-176): 0 new, 1 dropped, 2 appended or
// flag replaced.
SARU_HD int filter_record(ReadHits &h, int k, int tresh, int start, int flag, int possible) {
  if (possible != tresh) return 1;
  const int dir = flag > 3 ? 1 : 0;
  if (h.n == 0) {
    if (h.cap < 1) {
      h.overflow = 1;
      return 1;
    }
    h.pos[0] = start;
    h.flag[0] = (int8_t)flag;
    h.n = 1;
    if (start > 0) ++h.queue;
    return 0;
  }
  for (int c = 0; c < h.n; ++c) {
    const int pc = h.pos[c], fc = h.flag[c];
    const int dc = fc > 3 ? 1 : 0;
    for (int i = -k; i <= k; ++i)
      if ((start + i == pc || start + i == -pc) && fc <= flag) return 1;
    if (pc == start && dc == dir && fc > flag) {
      h.flag[c] = (int8_t)flag;
      return 2;
    }
    if ((pc == start && dc == dir) || (pc == -start && dc == dir)) return 1;
  }
  if (h.n >= h.cap) {
    h.overflow = 1;
    return 1;
  }
  h.pos[h.n] = start;
  h.flag[h.n] = (int8_t)flag;
  ++h.n;
  if (start > 0) ++h.queue;
  return 2;
}

// Matches of `want` among the values a scan of the reference visits, in
// visit order (at most two: the scan's first element can come round again).
//  first pass, list b from index `off`: the value at off, then indices
//    1, 2, ... up to the first 0 -- for a non-empty list, indices 1..len-1 of
//    the list itself (ascending, so one binary search), for an empty one the
//    lists that follow it, walked as the reference walks them;
//  second pass, list from index 0: indices 0..len-1 unless the value at 0 is
//    0 (an empty list, or a first position 0).
// Lists: len(x), at(x, i) (element i of the data array from list x's start,
// past the list included), find(x, lo, want) (an index in [lo, len(x)) of
// list x holding want, or -1).
template <class Lists>
SARU_HD int scan_from(const Lists &L, int x, uint32_t v0, uint32_t want) {
  // v0: the value at the scan's first index (L.at(x, off))
  if (v0 == 0) return 0;
  int hits = v0 == want ? 1 : 0;
  const uint32_t len = L.len(x);
  if (len >= 1) return hits + (L.find(x, 1, want) >= 0 ? 1 : 0);
  for (uint32_t i = 1;; ++i) {  // an empty list: the walk runs into the next lists
    const uint32_t v = L.at(x, i);
    if (v == 0) return hits;
    if (v == want) ++hits;
  }
}

// scan_from over list x from index `off` (nlists: the read's lists),
// the same count in fewer reads of the data array.  An empty list x read
// from off >= 1 starts in list x + 1, which follows its terminating 0:
// the value at off is element off - 1 of list x + 1 (its 0 when off - 1 is
// its length), and the walk from index 1 is list x + 1 from its start to
// its 0.  Positions in a list ascend, so a 0 inside one can only be its
// first element (the walk then stops at once) and the walk's match is one
// search.  Any other case takes scan_from itself.
template <class Lists>
SARU_HD int scan_from_at(const Lists &L, int x, int nlists, uint32_t off, uint32_t want) {
  if (L.len(x) >= 1 || off == 0 || x + 1 >= nlists) return scan_from(L, x, L.at(x, off), want);
  const uint32_t len1 = L.len(x + 1);
  const uint32_t v0 =
      off - 1 < len1 ? L.at(x + 1, off - 1) : (off - 1 == len1 ? 0u : L.at(x, off));
  if (v0 == 0) return 0;
  const int hits = v0 == want ? 1 : 0;
  if (len1 == 0 || L.at(x + 1, 0) == 0) return hits;
  return hits + (L.find(x + 1, 0, want) >= 0 ? 1 : 0);
}

template <class Lists>
SARU_HD int scan_all(const Lists &L, int x, uint32_t want) {
  if (L.at(x, 0) == 0) return 0;
  return L.find(x, 0, want) >= 0 ? 1 : 0;
}

// One read (read bytes as sequenced; reversed and complemented here when
// dr == 4).  L: the read's lists (see scan_from), whose values are genome
// positions: with the genome in chunks, positions in the whole genome (the
// chunk's position `offset` added, src/util.c:481), so only the genome's own
// position 0 reads as a list end.  A start is taken when it lies after the
// chunk's first byte (src/hash.c:545).  perfect(gs1): the genome at gs1 (a
// position in the whole genome) spells the read (strand-adjusted) over m
// bytes.  Kept positions are positions in the whole genome.
template <class Lists, class Perfect>
SARU_HD void filter_read(const FilterShape &S, int dr, const Lists &L, Perfect perfect,
                         ReadHits &h, int offset = 0) {
  const int k = S.k, half = S.half, q = S.q;
  for (int a = 0; a < half; ++a) {
    const int first = a == 0 ? 1 : 0;
    const uint32_t in_read = (uint32_t)a * q + 1;
    uint32_t off = 0;
    uint32_t pa = L.at(a, off);
    while (pa > 0) {
      const int gs = (int)(pa - in_read);
      if (gs + 1 - offset > 0) {
        if (perfect(gs + 1)) filter_record(h, k, S.tresh, -(gs + 1), 0, S.tresh);
        int possible = 1;
        // pairs with the later first-half q-grams; the reference starts each
        // scan at a's current index
        for (int b = a + 1; b < half; ++b) {
          const uint32_t rs = (uint32_t)b * q + 1;
          for (int ez = -k; ez <= k; ++ez) {
            const int hits = scan_from_at(L, b, S.P, off, (uint32_t)gs + rs + (uint32_t)ez);
            for (int t = 0; t < hits; ++t) {
              int flag, start;
              if (b == half - 1 && first) {
                flag = 1 + dr;
                start = gs + 1;
              } else if (a == half - 1) {
                flag = ((int)(pa + q) > S.m ? 3 : 2) + dr;
                start = gs - k + 1;
              } else if (first) {
                flag = 1 + dr;
                start = gs + 1;
              } else {
                flag = 3 + dr;
                start = gs - k + 1;
              }
              ++possible;
              filter_record(h, k, S.tresh, start, flag, possible);
            }
          }
        }
        // pairs with the second-half q-grams
        for (int b = 0; b < half; ++b) {
          int lim = half - 1 - b - a;
          if (lim < 0) lim = -lim;
          const uint32_t ns = (uint32_t)(half - b - 1) * q + 1 + S.rest;
          for (int err = -lim; err <= lim; ++err) {
            const int ae = (b - a < 0) ? -err : err;
            if (!scan_all(L, half + b, (uint32_t)gs + ns + (uint32_t)ae)) continue;
            int flag, start;
            if (b == 0 && first) {
              flag = 1 + dr;
              start = gs + 1;
            } else if (b == 0) {
              flag = ((int)(ns + q) > S.m ? 3 : 2) + dr;
              start = gs - k + 1;
            } else if (first) {
              flag = 1 + dr;
              start = gs + 1;
            } else {
              flag = 3 + dr;
              start = gs - k + 1;
            }
            ++possible;
            filter_record(h, k, S.tresh, start, flag, possible);
          }
        }
      }
      ++off;
      pa = L.at(a, off);
    }
  }
}

}  // namespace saru
