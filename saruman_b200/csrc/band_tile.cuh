// band_tile.cuh -- one warp tile of the banded kernel, as phases.
//
// A warp tile is 32 consecutive candidates, one per lane.  Their reads,
// windows and output slots are three contiguous byte ranges, so the warp
// stages the inputs into its shared-memory slice with 16-byte loads, aligns
// out of shared memory, builds both alignment strings for the whole tile in
// shared memory (zero-filled, as the reference's memset arena leaves them)
// and writes the tile's slot range back with 16-byte stores.  Decision
// planes (2 bits per band cell) go to a global scratch that stays in L2;
// the traceback keeps the next three columns' planes in registers.
//
// The phases are separated by warp barriers in the kernel; written as
// functions of the lane so a host harness can run them lane by lane.
//
// Warp slice layout (bytes, each part 16-aligned):
//   [reads staging RS][windows staging WS][region: codes+masks | outputs]
// The region holds the lane-interleaved code/mask words during the fill
// and the two output strings during the traceback.
#pragma once
#include <stdint.h>

#include "saru_core.cuh"

namespace saru {

struct TileArgs {
  const uint8_t *genome, *reads;
  const int32_t *goff, *roff;
  const int8_t *dirs;
  long n;
  int k, max_m, first_of_call;
  int32_t *scores;
  uint8_t *read_aln, *genome_aln;
  void *planes;       // plane_columns(max_m) * pstride plane pairs (plane_index)
  long pstride;       // lanes of the whole grid
  long pair_mul;      // plane-pair index multiplier: 2 when 32-bit pairs share a
                      // launch with 64-bit ones (one slot size for every lane)
  long rs_bytes, ws_bytes, region_bytes;
  uint8_t *records;  // compact result records instead of slot strings (nullptr: slots)
  long rec_bytes;    // bytes per record (compact_record_bytes)
};

// Byte ranges of a tile in the three arrays.
struct TileSpan {
  long t0, t1;
  long r_lo, r_hi, g_lo, g_hi, s_lo, s_hi;
  long r_base, g_base, o_base_r, o_base_g, o_span_r;
  bool fits;
};

SARU_HD long gstart_at(const int32_t *goff, long t) { return t ? goff[t - 1] : 0; }

// Staging base of global range [lo, ...) of array `p`: byte x sits at
// smem[x - base], with base chosen so that 16-byte aligned global addresses
// map to 16-byte aligned smem offsets.
SARU_HD long stage_base(const void *p, long lo) {
  return lo - (long)(((uintptr_t)((const uint8_t *)p + lo)) & 15u);
}

SARU_HD TileSpan tile_span(const TileArgs &a, long wt) {
  TileSpan s;
  s.t0 = wt * 32;
  s.t1 = s.t0 + 32 < a.n ? s.t0 + 32 : a.n;
  s.r_lo = s.t0 ? a.roff[s.t0 - 1] : 0;
  s.r_hi = a.roff[s.t1 - 1];
  s.g_lo = gstart_at(a.goff, s.t0);
  s.g_hi = a.goff[s.t1 - 1];
  s.s_lo = s.g_lo + (long)a.k * s.t0;
  s.s_hi = s.g_hi + (long)a.k * s.t1;
  const long cnt = s.t1 - s.t0;
  // a tile whose ranges exceed what regular candidates can span is not
  // staged at all (its candidates are reported irregular)
  s.fits = s.r_hi >= s.r_lo && s.g_hi >= s.g_lo && s.r_hi - s.r_lo <= cnt * (long)a.max_m &&
           s.g_hi - s.g_lo <= cnt * (long)(a.max_m + 2 * a.k);
  s.r_base = stage_base(a.reads, s.r_lo);
  s.g_base = stage_base(a.genome, s.g_lo);
  s.o_base_r = stage_base(a.read_aln, s.s_lo);
  s.o_base_g = stage_base(a.genome_aln, s.s_lo);
  s.o_span_r = ((s.s_hi - s.o_base_r) + 15) & ~15L;
  return s;
}

// Copies global bytes [lo, hi) of src into dst (smem) at dst[x - base]:
// 16-byte vectors where the global address is aligned, bytes at the edges.
template <class Load16, class Load1>
SARU_HD void stage_in(uint8_t *dst, const uint8_t *src, long lo, long hi, long base, int lane,
                      Load16 ld16, Load1 ld1) {
  const long a16 = base + ((lo - base + 15) & ~15L);
  const long b16 = base + ((hi - base) & ~15L);
  if (a16 >= b16) {
    for (long x = lo + lane; x < hi; x += 32) dst[x - base] = ld1(src + x);
    return;
  }
  for (long x = lo + lane; x < a16; x += 32) dst[x - base] = ld1(src + x);
  const long nv = (b16 - a16) >> 4;
  for (long i = lane; i < nv; i += 32) ld16(dst + (a16 - base) + 16 * i, src + a16 + 16 * i);
  for (long x = b16 + lane; x < hi; x += 32) dst[x - base] = ld1(src + x);
}

// Writes smem src (holding byte x at src[x - base]) to global dst[lo, hi).
template <class Store16>
SARU_HD void stage_out(uint8_t *dst, const uint8_t *src, long lo, long hi, long base, int lane,
                       Store16 st16) {
  const long a16 = base + ((lo - base + 15) & ~15L);
  const long b16 = base + ((hi - base) & ~15L);
  if (a16 >= b16) {
    for (long x = lo + lane; x < hi; x += 32) dst[x] = src[x - base];
    return;
  }
  for (long x = lo + lane; x < a16; x += 32) dst[x] = src[x - base];
  const long nv = (b16 - a16) >> 4;
  for (long i = lane; i < nv; i += 32) st16(dst + a16 + 16 * i, src + (a16 - base) + 16 * i);
  for (long x = b16 + lane; x < hi; x += 32) dst[x] = src[x - base];
}

// Bytes p..p+3 (little endian) from a byte buffer at any alignment, with
// two aligned 32-bit loads; reads up to 7 bytes past p, which the staging
// slack covers.
SARU_HD uint32_t load4(const uint8_t *p) {
  const uintptr_t a = (uintptr_t)p;
  const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
  return fshr32(w[0], w[1], (uint32_t)(a & 3u) * 8u);
}

// Per-lane state carried from the fill to the traceback.
struct LaneState {
  Cand c;
  long gs, rs;
  int score;
  bool ok;
};

// Fill phase of one lane.  Returns status bits.
template <typename T, class PlaneStore>
SARU_HD int lane_fill(const TileArgs &a, const TileSpan &s, int lane, const uint8_t *st_reads,
                      const uint8_t *st_win, uint32_t *region32, LaneState &ls,
                      PlaneStore store) {
  const long t = s.t0 + lane;
  ls.ok = false;
  ls.score = a.k + 1;
  if (t >= a.n) return 0;
  int status = 0;
  const int k = a.k;
  const int code_words = (a.max_m + 7) / 8;
  const int mwords = mask_words(k, a.max_m + 2 * k);
  Strided codes{region32, lane};
  Strided mask{region32, code_words * 32 + lane};
  Cand &c = ls.c;
  ls.gs = gstart_at(a.goff, t);
  ls.rs = t ? a.roff[t - 1] : 0;
  c.m = int(a.roff[t] - ls.rs);
  c.L = int(a.goff[t] - ls.gs);
  c.k = k;
  flank_of(a.dirs[t], k, c.so, c.eo);
  c.first_of_call = a.first_of_call && t == 0;
  if (!s.fits || c.L != c.m + c.so + c.eo || c.m <= 3 * k || c.m > a.max_m || c.m < 2) {
    status |= 1;  // irregular
  } else {
    const uint8_t *rd = st_reads + (ls.rs - s.r_base);
    const uint8_t *wn = st_win + (ls.gs - s.g_base);
    if (!build_codes_acgt(c, [&](int i) { return load4(rd + i); },
                          [&](int i) { return load4(wn + i); }, codes, mask, mwords) &&
        !build_codes(c, [&](int j) -> uint8_t { return rd[j]; },
                     [&](int p) -> uint8_t { return wn[p]; }, codes, mask, mwords)) {
      status |= 2;  // alphabet
    } else {
      ls.ok = true;
      ls.score = fill_band<T>(c, codes, mask, mwords, store);
    }
  }
  a.scores[t] = ls.score;
  return status;
}

// Decision planes of one column for one lane, stored as an adjacent pair
// so a single load fetches both.
template <typename T>
struct PlanePair {
  T A, B;
};

// Decision planes in the scratch: [column][lane], so the fill's store of a
// column is one contiguous 256-byte (512-byte) run per warp.  (Runs of
// columns per lane would give the traceback's walk better L1 locality, but
// their fill stores touch a sector per lane and measured twice as slow.)
// `mul` spaces 32-bit pairs like 64-bit ones when a launch mixes both.
SARU_HD long plane_columns(int max_m) { return (long)max_m + 1; }  // columns 0..max_m

SARU_HD long plane_index(int j, long pstride, long pslot, long mul) {
  return ((long)j * pstride + pslot) * mul;
}

// Traceback phase of one lane: writes the lane's two strings into its slot
// of the output staging, in reading order (the reference emits from the
// alignment end and reverses in place, src/cuda-functions.cu:306-307; here
// the characters are written from the slot end downwards and the string is
// then moved to the slot start, which leaves the same bytes).
//
// Interior cells (row >= 1, column >= 1) take a branch-free step per loop
// iteration, so the warp stays converged: with the recorded decision as
// bits (a, b) -- DIAG (1,0), UP (0,1), LEFT (1,1), STOP (0,0) -- the read
// string gets a read byte iff a, the window string a window byte unless
// a&b, the column drops iff a, the row drops unless a&b.  The planes of the
// next column are already in registers and the column PF ahead is
// prefetched.  Row 0 and column 0 follow the reference's border rules in a
// short tail loop (see traceback_band in saru_core.cuh).
template <typename T, int PF, class LoadPair, class Prefetch>
SARU_HD int lane_traceback(const TileArgs &a, const TileSpan &s, int lane, const uint8_t *st_reads,
                           const uint8_t *st_win, uint8_t *out_r, uint8_t *out_g,
                           const LaneState &ls, LoadPair ld, Prefetch prefetch) {
  constexpr int BITS = int(sizeof(T) * 8);
  const long t = s.t0 + lane;
  if (t >= a.n || !ls.ok || ls.score > a.k) return 0;
  const Cand &c = ls.c;
  const int roff = (int)(ls.rs - s.r_base) - 1;  // read byte col-1 at st_reads[roff + col]
  const int woff = (int)(ls.gs - s.g_base) - 1;  // window byte row-1 at st_win[woff + row]
  const long slot = ls.gs + (long)a.k * t;
  const int sr = (int)(slot - s.o_base_r);  // slot start in out_r
  const int sg = (int)(slot - s.o_base_g);
  const int cap = c.L + c.k;                 // slot bytes
  int n = 0;                                 // bytes written, from the slot end down
  int row = c.L, col = c.m, b = c.L - c.m + c.k;
  bool bad = false, stop = false;
  // planes of the current column and the next three to the left in
  // registers, so a load is issued three column moves before its use
  PlanePair<T> cur = ld(col);
  PlanePair<T> n1 = ld(col - 1);  // col >= 2 here (m > 3k >= 0 and m >= 2)
  PlanePair<T> n2 = col >= 3 ? ld(col - 2) : PlanePair<T>{};
  PlanePair<T> n3 = col >= 4 ? ld(col - 3) : PlanePair<T>{};
  for (int j = col - 4; j >= 1 && j > col - 4 - PF; --j) prefetch(j);
  // interior: row >= 1 and col >= 1 hold on entry to every iteration
  for (;;) {
    if ((unsigned)b >= (unsigned)BITS) {
      bad = true;
      break;
    }
    const uint32_t da = (uint32_t)((cur.A >> b) & T(1));
    const uint32_t db = (uint32_t)((cur.B >> b) & T(1));
    if ((da | db) == 0) {
      stop = true;
      break;
    }
    if (n >= cap) {
      bad = true;
      break;
    }
    const uint8_t rch = st_reads[roff + col];
    const uint8_t gch = st_win[woff + row];
    ++n;
    out_r[sr + cap - n] = da ? rch : uint8_t('_');
    out_g[sg + cap - n] = (da & db) ? uint8_t('_') : gch;
    row -= (int)(1u - (da & db));
    b += (int)db * ((int)da * 2 - 1);
    if (da) {
      --col;
      cur = n1;
      n1 = n2;
      n2 = n3;
      if (col >= 4) n3 = ld(col - 3);
      if (col - 3 - PF >= 1) prefetch(col - 3 - PF);
    }
    if (row == 0 || col == 0) break;
  }
  if (!bad && !stop) {
    // borders.  Row 0 (col >= 1): the first candidate of a call stops; later
    // ones step left to column 0 (their diagonal/top neighbours are the
    // previous matrix's last row, all > k when m > 3k).  Column 0 holds
    // max(0, row - 2so); only the vertical test can hold there.
    for (;;) {
      if (row == 0) {
        if (col == 0 || c.first_of_call) break;
        if (n >= cap) {
          bad = true;
          break;
        }
        ++n;
        out_r[sr + cap - n] = st_reads[roff + col];
        out_g[sg + cap - n] = '_';
        --col;
        continue;
      }
      // col == 0, row >= 1
      const int v = row - 2 * c.so > 0 ? row - 2 * c.so : 0;
      const int tp = row - 1 - 2 * c.so > 0 ? row - 1 - 2 * c.so : 0;
      const int corr = (c.so && row - 1 <= 2 * c.so + 2) ? 1 : 0;
      if (tp + 1 - corr != v) break;
      if (n >= cap) {
        bad = true;
        break;
      }
      ++n;
      out_r[sr + cap - n] = '_';
      out_g[sg + cap - n] = st_win[woff + row];
      --row;
    }
  }
  // move the string to the slot start; clear what it vacated
  if (n < cap) {
    const int from = cap - n;
    for (int i = 0; i < n; ++i) {
      out_r[sr + i] = out_r[sr + from + i];
      out_g[sg + i] = out_g[sg + from + i];
    }
    for (int i = n; i < cap; ++i) {
      out_r[sr + i] = 0;
      out_g[sg + i] = 0;
    }
  }
  return bad ? 4 : 0;
}

// Compact result record of one candidate (the alternative to its two slot
// strings): word 0 = number of traceback steps n (bits 0-15) and an
// overflow flag (bit 16); words 1.. = the steps in traceback order (from
// the alignment end), 2 bits each, 16 per word: 1 DIAG (read byte against
// window byte), 2 UP (gap in the read), 3 LEFT (gap in the window).  With
// the call's reads and windows the host rebuilds the slot strings exactly
// (saru_expand_compact).  A candidate with score > k has n = 0.
constexpr int kCompactHeaderBytes = 4;

SARU_HD long compact_record_bytes(int max_m, int k) {
  const long steps = (long)max_m + 3L * k;  // L + k <= m + 3k
  return (kCompactHeaderBytes + 4 * ((steps + 15) / 16) + 15) & ~15L;
}

// Traceback of one lane into its compact record (same walk and border rules
// as lane_traceback).  store(w, v) writes word w of candidate t's record.
template <typename T, class LoadPair, class StoreWord>
SARU_HD int lane_traceback_ops(const TileArgs &a, const TileSpan &s, int lane,
                               const LaneState &ls, LoadPair ld, StoreWord store) {
  constexpr int BITS = int(sizeof(T) * 8);
  const long t = s.t0 + lane;
  if (t >= a.n) return 0;
  if (!ls.ok || ls.score > a.k) {
    store(0, 0u);
    return 0;
  }
  const Cand &c = ls.c;
  const int cap = c.L + c.k;
  int n = 0;
  uint32_t acc = 0;
  int row = c.L, col = c.m, b = c.L - c.m + c.k;
  bool bad = false, stop = false;
  auto push = [&](uint32_t op) {
    acc |= op << (2 * (n & 15));
    ++n;
    if ((n & 15) == 0) {
      store(n >> 4, acc);  // words 1.. hold steps 16(w-1) .. 16w-1
      acc = 0;
    }
  };
  PlanePair<T> cur = ld(col);
  PlanePair<T> nxt = ld(col - 1);  // col >= 2 here (m > 3k >= 0 and m >= 2)
  for (;;) {
    if ((unsigned)b >= (unsigned)BITS) {
      bad = true;
      break;
    }
    const uint32_t da = (uint32_t)((cur.A >> b) & T(1));
    const uint32_t db = (uint32_t)((cur.B >> b) & T(1));
    if ((da | db) == 0) {
      stop = true;
      break;
    }
    if (n >= cap) {
      bad = true;
      break;
    }
    push(da | (db << 1));
    row -= (int)(1u - (da & db));
    b += (int)db * ((int)da * 2 - 1);
    if (da) {
      --col;
      cur = nxt;
      if (col >= 2) nxt = ld(col - 1);
    }
    if (row == 0 || col == 0) break;
  }
  if (!bad && !stop) {
    for (;;) {  // borders, as in lane_traceback
      if (row == 0) {
        if (col == 0 || c.first_of_call) break;
        if (n >= cap) {
          bad = true;
          break;
        }
        push(3u);
        --col;
        continue;
      }
      const int v = row - 2 * c.so > 0 ? row - 2 * c.so : 0;
      const int tp = row - 1 - 2 * c.so > 0 ? row - 1 - 2 * c.so : 0;
      const int corr = (c.so && row - 1 <= 2 * c.so + 2) ? 1 : 0;
      if (tp + 1 - corr != v) break;
      if (n >= cap) {
        bad = true;
        break;
      }
      push(2u);
      --row;
    }
  }
  if (n & 15) store((n >> 4) + 1, acc);
  store(0, (uint32_t)n | (bad ? 0x10000u : 0u));
  return bad ? 4 : 0;
}

// Shared-memory slice sizes for a maximum read length and k.
struct SliceLayout {
  long rs_bytes, ws_bytes, region_bytes, warp_smem;
};

SARU_HD SliceLayout slice_layout(int max_m, int k) {
  SliceLayout L;
  const long code_words = (max_m + 7) / 8;
  const long mwords = mask_words(k, max_m + 2 * k);
  // staged bytes, 16 bytes of alignment head and 96 of slack for the word
  // readers (load4 and the 32-position chunks of build_codes_acgt)
  L.rs_bytes = (32L * max_m + 16 + 96 + 15) & ~15L;
  L.ws_bytes = (32L * (max_m + 2 * k) + 16 + 96 + 15) & ~15L;
  const long cm = 4L * 32 * (code_words + NCODES * mwords);
  const long out = 2 * ((32L * (max_m + 3 * k) + 32 + 15) & ~15L);
  L.region_bytes = ((cm > out ? cm : out) + 15) & ~15L;
  L.warp_smem = L.rs_bytes + L.ws_bytes + L.region_bytes;
  return L;
}

}  // namespace saru
