// band_tile.cuh -- one warp tile of the banded kernel, as phases.
//
// A warp tile is 32 consecutive candidates, one per lane.  Their reads,
// windows and output slots are three contiguous byte ranges, so the warp
// stages the inputs into its shared-memory slice with 16-byte loads, aligns
// out of shared memory, builds both alignment strings for the whole tile in
// shared memory (zero-filled, as the reference's memset arena leaves them)
// and writes the tile's slot range back with 16-byte stores.  Decision
// planes (2 bits per band cell) go to a global scratch that stays in L2;
// the traceback keeps the next four columns' planes in flight.
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
  long t0;           // first candidate (a multiple of 32); n is one past the last
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
  s.t0 = a.t0 + wt * 32;
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

// Compact result record of one candidate (the alternative to its two slot
// strings): word 0 = number of traceback steps n (bits 0-15) and an
// overflow flag (bit 16); words 1.. = the steps in traceback order (from
// the alignment end), 2 bits each, 16 per word: 1 DIAG (read byte against
// window byte), 2 UP (gap in the read), 3 LEFT (gap in the window).  With
// the call's reads and windows the host rebuilds the slot strings exactly
// (saru_expand_compact).  A candidate with score > k has n = 0.
constexpr int kCompactHeaderBytes = 4;

// Words of 2-bit steps a traceback can need: a slot holds L + k <= m + 3k.
SARU_HD long step_words(int max_m, int k) { return ((long)max_m + 3L * k + 15) / 16; }

SARU_HD long compact_record_bytes(int max_m, int k) {
  return (kCompactHeaderBytes + 4 * step_words(max_m, k) + 15) & ~15L;
}

// Bytes of a warp's two output strings in its shared slice.
SARU_HD long out_area_bytes(int max_m, int k) {
  return 2 * ((32L * (max_m + 3 * k) + 32 + 15) & ~15L);
}

// Where a traceback walk ended.
struct WalkEnd {
  int n;         // steps
  int row, col;  // the cell it stopped at
  bool bad;      // left the band or the slot
};

// The traceback walk of one lane (the reference's get_alignment,
// src/cuda-functions.cu:108-315, over the band's decision planes).  Each
// step is handed to emit(i, op, row, col): i counts from 0 at the alignment
// end, op is 1 DIAG (read byte col - 1 against window byte row - 1), 2 UP
// (gap in the read, window byte row - 1), 3 LEFT (read byte col - 1, gap in
// the window), and (row, col) is the cell the step leaves.
//
// Interior cells (row >= 1, column >= 1): the recorded decision (a, b) --
// DIAG (1,0), UP (0,1), LEFT (1,1), STOP (0,0) -- is the step; the column
// drops iff a, the band offset moves by +1 (LEFT) or -1 (UP), and the row
// follows from them: row = offset + column - k holds along the walk (it
// holds at the start, row L and column m at offset L - m + k, and every
// step keeps it).  The planes of the next four columns are in flight in
// four registers used in turn: a register is refilled with the column four
// ahead right after the walk leaves its column, and no register is copied
// to another (a copy would wait for its load).  Row 0 and column 0 follow
// the reference's border rules in a short tail loop (see traceback_band in
// saru_core.cuh).
template <typename T, class LoadPair, class Emit>
SARU_HD WalkEnd lane_walk(const Cand &c, LoadPair ld, Emit emit) {
  constexpr int BITS = int(sizeof(T) * 8);
  const int cap = c.L + c.k, k = c.k;
  int n = 0;
  int col = c.m, b = c.L - c.m + c.k;
  int end = 0;  // 1: reached row 0 or column 0, 2: a stop decision, 3: left band or slot
  // the steps at the current column (planes p) up to the one that leaves
  // it; false when the walk's interior ends
  auto column = [&](const PlanePair<T> &p) -> bool {
    for (;;) {
      const bool out = (unsigned)b >= (unsigned)BITS;
      const int bb = b & (BITS - 1);
      const uint32_t da = (uint32_t)(p.A >> bb) & 1u;
      const uint32_t db = (uint32_t)(p.B >> bb) & 1u;
      if (out || (da | db) == 0u || n >= cap) {
        end = (out || (da | db) != 0u) ? 3 : 2;
        return false;
      }
      emit(n++, da | (db << 1), b + col - k, col);
      if (!da) {  // UP: same column, one row up
        --b;
        if (b + col == k) {
          end = 1;
          return false;
        }
        continue;
      }
      b += (int)db;  // LEFT +1, DIAG 0
      --col;
      if (b + col == k || col == 0) {
        end = 1;
        return false;
      }
      return true;
    }
  };
  auto ahead = [&](int j) { return ld(j > 0 ? j : 0); };
  PlanePair<T> p0 = ld(col), p1 = ahead(col - 1), p2 = ahead(col - 2), p3 = ahead(col - 3);
  for (;;) {
    if (!column(p0)) break;
    p0 = ahead(col - 3);
    if (!column(p1)) break;
    p1 = ahead(col - 3);
    if (!column(p2)) break;
    p2 = ahead(col - 3);
    if (!column(p3)) break;
    p3 = ahead(col - 3);
  }
  bool bad = end == 3;
  int row = b + col - k;
  if (end == 1) {
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
        emit(n++, 3u, row, col);
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
      emit(n++, 2u, row, col);
      --row;
    }
  }
  return WalkEnd{n, row, col, bad};
}

// Traceback phase of one lane in slot mode: writes the lane's two strings
// into its slot of the output staging, in reading order.  The reference
// emits from the alignment end and reverses in place
// (src/cuda-functions.cu:306-307); here the characters are written from the
// slot end downwards as the walk goes and the strings are then moved to
// the slot start, which leaves the same bytes.
template <typename T, class LoadPair>
SARU_HD int lane_traceback(const TileArgs &a, const TileSpan &s, int lane, const uint8_t *st_reads,
                           const uint8_t *st_win, uint8_t *out_r, uint8_t *out_g,
                           const LaneState &ls, LoadPair ld) {
  const long t = s.t0 + lane;
  if (t >= a.n || !ls.ok || ls.score > a.k) return 0;
  const int cap = ls.c.L + ls.c.k;  // slot bytes
  const long slot = ls.gs + (long)a.k * t;
  uint8_t *o_r = out_r + (slot - s.o_base_r);
  uint8_t *o_g = out_g + (slot - s.o_base_g);
  const uint8_t *rd = st_reads + (ls.rs - s.r_base) - 1;  // read byte col - 1 at rd[col]
  const uint8_t *wn = st_win + (ls.gs - s.g_base) - 1;    // window byte row - 1 at wn[row]
  uint8_t *e_r = o_r + cap - 1, *e_g = o_g + cap - 1;      // step i at e_r[-i]
  const WalkEnd e = lane_walk<T>(ls.c, ld, [&](int i, uint32_t op, int row, int col) {
    const uint8_t rch = rd[col], gch = wn[row];
    e_r[-i] = (op & 1u) ? rch : uint8_t('_');
    e_g[-i] = op != 3u ? gch : uint8_t('_');
  });
  // move the strings to the slot start; clear what they vacated
  const int n = e.n;
  if (n < cap) {
    const int from = cap - n;
    for (int i = 0; i < n; ++i) {
      o_r[i] = o_r[from + i];
      o_g[i] = o_g[from + i];
    }
    for (int i = n; i < cap; ++i) {
      o_r[i] = 0;
      o_g[i] = 0;
    }
  }
  return e.bad ? 4 : 0;
}

// Traceback of one lane into its compact record.  store(w, v) writes word w
// of candidate t's record.
template <typename T, class LoadPair, class StoreWord>
SARU_HD int lane_traceback_ops(const TileArgs &a, const TileSpan &s, int lane,
                               const LaneState &ls, LoadPair ld, StoreWord store) {
  const long t = s.t0 + lane;
  if (t >= a.n) return 0;
  // every word of the record is written (steps, then zeros), so a record's
  // bytes do not depend on what the buffer held before
  const int nwords = (int)(a.rec_bytes / 4);
  if (!ls.ok || ls.score > a.k) {
    for (int w = 0; w < nwords; ++w) store(w, 0u);
    return 0;
  }
  uint32_t acc = 0;
  int sh = 0, w = 1;
  const WalkEnd e = lane_walk<T>(ls.c, ld, [&](int, uint32_t op, int, int) {
    acc |= op << sh;
    sh += 2;
    if (sh == 32) {  // words 1.. hold steps 16(w-1) .. 16w-1
      store(w++, acc);
      acc = 0;
      sh = 0;
    }
  });
  if (sh) store(w++, acc);
  for (; w < nwords; ++w) store(w, 0u);
  store(0, (uint32_t)e.n | (e.bad ? 0x10000u : 0u));
  return e.bad ? 4 : 0;
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
  const long out = out_area_bytes(max_m, k);
  L.region_bytes = ((cm > out ? cm : out) + 15) & ~15L;
  L.warp_smem = L.rs_bytes + L.ws_bytes + L.region_bytes;
  return L;
}

}  // namespace saru
