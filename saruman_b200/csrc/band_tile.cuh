// band_tile.cuh -- one warp tile of the banded kernel, as phases.
//
// A warp tile is 32 consecutive candidates, one per lane.  Their reads,
// windows and output slots are three contiguous byte ranges, so the warp
// stages the inputs into its shared-memory slice with 16-byte loads, aligns
// out of shared memory, builds both alignment strings for the whole tile in
// shared memory (zero-filled, as the reference's memset arena leaves them)
// and writes the tile's slot range back with 16-byte stores.  Decision
// planes (2 bits per band cell) go to a global scratch that stays in L2;
// the traceback walk keeps the next kRing columns' planes in flight.
//
// The phases are separated by warp barriers in the kernel; written as
// functions of the lane so a host harness can run them lane by lane.
//
// Warp slice layout (bytes, each part 16-aligned):
//   [reads staging RS][windows staging WS][region: codes+masks | outputs]
// The region holds the lane-interleaved code/mask words during the fill,
// the ring of decision planes during the traceback walk and the two output
// strings after it.
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
  void *planes;       // plane_units(max_m, wide) x pstride units of kPlaneUnit bytes
  long pstride;       // lanes of the whole grid
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
  const int code_words = a.max_m / 8 + 1;
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

// Decision planes in the scratch: 16-byte units, [unit][lane], so a warp's
// store of a unit is one contiguous 512-byte run.  A unit holds the pairs
// of two columns of a 32-bit band (column j in unit j >> 1 at byte
// (j & 1) * 8) or of one column of a 64-bit band (unit j): the fill stores
// 16 bytes a lane every other column of a 32-bit band.  (Runs of columns
// per lane would give the traceback's walk better locality, but their fill
// stores touch a sector per lane and measured twice as slow.)
constexpr long kPlaneUnit = 16;

// Units a lane needs for columns 0..max_m.
SARU_HD long plane_units(int max_m, bool wide) {
  return wide ? (long)max_m + 1 : (long)(max_m >> 1) + 1;
}

// Byte offset of column j's pair in unit row 0 of a lane (add the lane's
// slot * kPlaneUnit and the unit row's bytes).
template <typename T>
SARU_HD long plane_unit_of(int j) {
  return sizeof(T) == 4 ? (long)(j >> 1) : (long)j;
}
template <typename T>
SARU_HD long plane_half_of(int j) {
  return sizeof(T) == 4 ? (long)(j & 1) * 8 : 0L;
}

// The fill's plane sink for one lane: put(unit, x, y, z, w) stores one
// 16-byte unit.  A 32-bit band's even column waits in (pa, pb) for the odd
// one; the last column (`last`), if even, goes out with a zero partner.
// Column 0 has no planes (the walk never reads it), so unit 0 carries zeros
// in its first half.
template <typename T, class Put16>
struct PlaneWriter {
  Put16 put;
  uint32_t pa, pb;
  SARU_HD void operator()(int j, T A, T B, bool last) {
    if (sizeof(T) == 4) {
      if (j & 1) {
        put(j >> 1, pa, pb, (uint32_t)A, (uint32_t)B);
      } else {
        pa = (uint32_t)A;
        pb = (uint32_t)B;
        if (last) put(j >> 1, pa, pb, 0u, 0u);
      }
    } else {
      const uint64_t a = (uint64_t)A, b = (uint64_t)B;
      put(j, (uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
    }
  }
};

template <typename T, class Put16>
SARU_HD PlaneWriter<T, Put16> plane_writer(Put16 put) {
  return PlaneWriter<T, Put16>{put, 0u, 0u};
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

// A gap run of a traceback: `len` consecutive UP (gap in the read) or LEFT
// (gap in the window) steps, the first of them step i0 (steps count from 0
// at the alignment end).  Packed in one word: i0 in bits 0-10, len in bits
// 11-21, the step code in bits 22-23 (a slot holds at most 512 + 3 * 15
// steps).
SARU_HD uint32_t gap_run(int i0, int len, uint32_t op) {
  return (uint32_t)i0 | ((uint32_t)len << 11) | (op << 22);
}
SARU_HD int run_first(uint32_t r) { return int(r & 0x7FFu); }
SARU_HD int run_len(uint32_t r) { return int((r >> 11) & 0x7FFu); }
SARU_HD uint32_t run_op(uint32_t r) { return r >> 22; }

// Gap runs one walk can record.  Along the walk a LEFT step, and an UP step
// off the free vertical moves, lowers the cell value by one; the walk starts
// at a value <= k and values are >= 0, so at most k runs hold such a step.
// The free moves (UP on the last column below row L - 2eo, UP on column 1
// for rows <= 2so + 3) and the two border tails (row 0, column 0) start at
// most four runs more.  k <= 15 in the banded kernel.
constexpr int kMaxGapRuns = 20;

// The gap runs of one step code (UP or LEFT) of a walk, in traceback order:
// r[0 .. n) (a per-thread array, written and read once a run) and then
// `open`, the last one (length 0: no run at all), kept in a register: in
// reading order it is the first.
struct GapRuns {
  const uint32_t *r;
  int n;
  uint32_t open;
};

// Appends traceback step `step` to the runs (r, n, open): extends the open
// run when the step follows it, else starts a new one.  False if r is full.
SARU_HD bool add_gap_step(uint32_t *r, int &n, uint32_t &open, int step, uint32_t op) {
  if (run_len(open) && run_first(open) + run_len(open) == step) {
    open += 1u << 11;
    return true;
  }
  bool ok = true;
  if (run_len(open)) {
    if (n < kMaxGapRuns) r[n++] = open;
    else ok = false;
  }
  open = gap_run(step, 1, op);
  return ok;
}

// The decision planes the traceback walk keeps in flight: a ring of kRing
// slots per lane in the warp's region (free between the fill and the
// writing of the strings), slot s of a lane at base[32 * s], column j in
// slot j mod kRing.  fetch(j) starts the copy of column max(j, 0) into its
// slot as one copy group; take(j) waits until no more than kRing - 1 groups
// are in flight (so column j, the oldest, has landed) and reads it.  A
// column's slot is refilled only after the walk has left that column.
constexpr int kRing = 16;

// Region bytes the ring takes: 8-byte plane pairs of a 32-bit band, 16-byte
// ones of a 64-bit band (which a launch shape can ask for at any k).
SARU_HD long ring_bytes(bool wide) { return (long)kRing * 32 * (wide ? 16 : 8); }

template <typename T, class Copy, class Wait>
struct PlaneRing {
  PlanePair<T> *base;  // this lane's slot 0
  Copy copy;           // copy(dst, j): start copying column j's pair to dst, as one group
  Wait wait;           // wait(): the oldest group in flight has landed (of kRing)
  SARU_HD PlanePair<T> *slot(int j) const { return base + 32 * (j & (kRing - 1)); }
  SARU_HD void fetch(int j) const { copy(slot(j), j > 0 ? j : 0); }
  SARU_HD PlanePair<T> take(int j) const {
    wait();
    return *slot(j);
  }
};

template <typename T, class Copy, class Wait>
SARU_HD PlaneRing<T, Copy, Wait> plane_ring(PlanePair<T> *base, Copy copy, Wait wait) {
  return PlaneRing<T, Copy, Wait>{base, copy, wait};
}

// The traceback walk of one lane (the reference's get_alignment,
// src/cuda-functions.cu:108-315, over the band's decision planes), recording
// only its gap runs: every other step is a DIAG step, so the cell where the
// walk ends, its step count and its gap runs give both alignment strings.
//
// Interior cells (row >= 1, column >= 1): the recorded decision (a, b) --
// DIAG (1,0), UP (0,1), LEFT (1,1), STOP (0,0) -- is the step; the column
// drops iff a, the band offset moves by +1 (LEFT) or -1 (UP), and the row
// follows from them: row = offset + column - k holds along the walk (it
// holds at the start, row L and column m at offset L - m + k, and every
// step keeps it).  The step count is m - column + the UP steps so far.  A
// DIAG step that stays off the borders and inside the slot takes the fast
// path: one test of the DIAG bit at the band offset and one bound on the
// column (`stop`, recomputed when the offset or the UP count changes).  The
// planes of the next kRing columns are in flight in the ring: the walk takes
// column col from it and, on leaving the column, asks for column
// col - kRing.  Row 0 and column 0 follow the reference's border rules in a
// short tail loop (see traceback_band in saru_core.cuh).
template <typename T, class Ring>
SARU_HD WalkEnd lane_walk(const Cand &c, const Ring &ring, uint32_t *up_r, uint32_t *left_r,
                          GapRuns &ups, GapRuns &lefts) {
  constexpr int BITS = int(sizeof(T) * 8);
  const int cap = c.L + c.k, k = c.k, m = c.m;
  int col = m, b = c.L - m + k, nup = 0;
  int nu = 0, nl = 0;            // runs in up_r / left_r
  uint32_t ou = 0, ol = 0;       // the open UP / LEFT run
  bool full = false;  // more runs than kMaxGapRuns (not reachable, see above)
  auto gap = [&](int n, uint32_t op) {
    const bool ok = op == (uint32_t)OP_UP ? add_gap_step(up_r, nu, ou, n, op)
                                          : add_gap_step(left_r, nl, ol, n, op);
    if (!ok) full = true;
  };
  T bit = T(0);
  int stop = 0;
  // a DIAG step from column col takes the fast path iff col > stop: then the
  // step is inside the slot (m - col + nup < cap) and lands on neither
  // border (col - 1 >= 1, row - 1 >= 1)
  auto refresh = [&]() {
    bit = (unsigned)b < (unsigned)BITS ? T(1) << b : T(0);
    const int s1 = k - b + 1 > 1 ? k - b + 1 : 1;
    const int s2 = m + nup - cap;
    stop = s1 > s2 ? s1 : s2;
  };
  refresh();
  int end = 0;  // 1: reached row 0 or column 0, 2: a stop decision, 3: left band or slot
  // the steps at the current column (planes p) up to the one that leaves
  // it; false when the walk's interior ends
  auto column = [&](const PlanePair<T> &p) -> bool {
    if ((p.A & ~p.B & bit) != T(0) && col > stop) {
      --col;
      return true;
    }
    for (;;) {
      const bool out = (unsigned)b >= (unsigned)BITS;
      const int bb = b & (BITS - 1);
      const uint32_t da = (uint32_t)(p.A >> bb) & 1u;
      const uint32_t db = (uint32_t)(p.B >> bb) & 1u;
      const int n = m - col + nup;
      if (out || (da | db) == 0u || n >= cap) {
        end = (out || (da | db) != 0u) ? 3 : 2;
        return false;
      }
      if (!da) {  // UP: same column, one row up
        gap(n, OP_UP);
        ++nup;
        --b;
        refresh();
        if (b + col == k) {
          end = 1;
          return false;
        }
        continue;
      }
      if (db) {  // LEFT: one column left, same row
        gap(n, OP_LEFT);
        ++b;
        refresh();
      }
      --col;
      if (b + col == k || col == 0) {
        end = 1;
        return false;
      }
      return true;
    }
  };
  for (int i = 0; i < kRing; ++i) ring.fetch(col - i);
  for (;;) {
    if (!column(ring.take(col))) break;
    ring.fetch(col - (kRing - 1));
  }
  bool bad = end == 3;
  int row = b + col - k;
  if (end == 1) {
    // borders.  Row 0 (col >= 1): the first candidate of a call stops; later
    // ones step left to column 0 (their diagonal/top neighbours are the
    // previous matrix's last row, all > k when m > 3k).  Column 0 holds
    // max(0, row - 2so); only the vertical test can hold there.
    for (;;) {
      const int n = m - col + nup;
      if (row == 0) {
        if (col == 0 || c.first_of_call) break;
        if (n >= cap) {
          bad = true;
          break;
        }
        gap(n, OP_LEFT);
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
      gap(n, OP_UP);
      ++nup;
      --row;
    }
  }
  ups = GapRuns{up_r, nu, ou};
  lefts = GapRuns{left_r, nl, ol};
  return WalkEnd{m - col + nup, row, col, bad || full};
}

// Bytes [lo, hi) of a little-endian word (0 <= lo <= hi <= 4) as a mask.
SARU_HD uint32_t bytes_mask(int lo, int hi) {
  const uint32_t h = hi >= 4 ? 0xFFFFFFFFu : ((1u << (8 * hi)) - 1u);
  const uint32_t l = lo >= 4 ? 0xFFFFFFFFu : ((1u << (8 * lo)) - 1u);
  return h & ~l;
}

// src[x .. x+4) as a word, with the bytes at negative indices zero (nothing
// before src is read).
SARU_HD uint32_t load4_from(const uint8_t *src, int x) {
  if (x >= 0) return load4(src + x);
  return x <= -4 ? 0u : load4(src) << (8 * -x);
}

// ORs a word into shared memory (two lanes may own bytes of one word).
SARU_HD void or_word(uint32_t *w, uint32_t v) {
#if defined(__CUDA_ARCH__)
  atomicOr(w, v);
#else
  *w |= v;
#endif
}

// One alignment string of a lane in reading order at dst[0, n): the bytes
// of src in order, with '_' at the positions of the gap runs g (UP runs for
// the read string, LEFT runs for the window string).  Position p is
// traceback step n - 1 - p, so the runs come in the reverse of their
// recorded order.  Written on dst's word grid with the same instructions in
// every lane: the source streamed through a funnel shift; a word that meets
// a gap merges '_' bytes and the shifted source by byte masks; the two
// edge words, which share bytes with the neighbouring slots (or hold this
// slot's tail, zero already), are ORed in.  Reads up to 7 bytes past the
// last source byte it uses and nothing before src.
SARU_HD void expand_string(uint8_t *dst, int n, const uint8_t *src, const GapRuns g) {
  if (n <= 0) return;
  constexpr int kNone = 0x7FFFFFFF;
  int gs = kNone, ge = kNone;  // the next gap [gs, ge) in reading order
  auto take = [&](uint32_t r) {
    ge = n - run_first(r);
    gs = ge - run_len(r);
  };
  if (run_len(g.open)) take(g.open);
  int gi = g.n;                                 // runs of g.r not taken yet
  uint32_t nxt = gi > 0 ? g.r[gi - 1] : 0u;     // the one after [gs, ge), loaded ahead
  int cum = 0;                                  // gap positions before p
  // the word at positions [p, p+4) from v (its bytes as if no gap met it)
  auto merge_gaps = [&](int p, uint32_t v) -> uint32_t {
    while (gs < p + 4) {
      const int lo = gs > p ? gs - p : 0;
      const int hi = ge < p + 4 ? ge - p : 4;
      cum += hi - lo;
      const uint32_t gm = bytes_mask(lo, hi), am = bytes_mask(hi, 4);
      v = (v & ~(gm | am)) | (0x5F5F5F5Fu & gm) | (load4_from(src, p - cum) & am);
      if (ge > p + 4) break;  // the gap goes on into the next word
      if (run_len(nxt)) {
        take(nxt);
        --gi;
        nxt = gi > 0 ? g.r[gi - 1] : 0u;
      } else {
        gs = ge = kNone;
      }
    }
    return v;
  };
  const int a = (int)((uintptr_t)dst & 3u);
  uint32_t *dw = reinterpret_cast<uint32_t *>(dst - a);
  int p = -a;
  if (a) {  // head word: positions [-a, 4 - a)
    uint32_t v = merge_gaps(p, load4_from(src, p));
    or_word(dw, v & bytes_mask(a, n - p < 4 ? n - p : 4));
    p += 4;
    ++dw;
  }
  // whole words: the source stream restarts after each word that met a gap
  const uint32_t *sw = nullptr;
  uint32_t lo = 0, sh = 0;
  auto restart = [&](int q) {  // the stream at position q (source q - cum)
    const uintptr_t ad = (uintptr_t)(src + (q - cum));
    sw = reinterpret_cast<const uint32_t *>(ad & ~(uintptr_t)3);
    sh = (uint32_t)(ad & 3u) * 8u;
    lo = *sw;
  };
  restart(p);
  for (; p + 4 <= n; p += 4, ++dw) {
    ++sw;
    const uint32_t hi = *sw;
    uint32_t v = fshr32(lo, hi, sh);
    lo = hi;
    if (gs < p + 4) {
      v = merge_gaps(p, v);
      restart(p + 4);
    }
    *dw = v;
  }
  if (p < n) {  // tail word
    const uint32_t v = merge_gaps(p, load4_from(src, p - cum));
    or_word(dw, v & bytes_mask(0, n - p));
  }
}

// What a lane's traceback walk leaves for the writing of its strings.
struct LaneWalk {
  WalkEnd e;
  GapRuns ups, lefts;
  bool walked;  // the lane has an alignment (score <= k)
};

// Traceback walk of one lane in slot mode (the ring in the warp's region).
// up_r / left_r hold the lane's gap runs until its strings are written.
template <typename T, class Ring>
SARU_HD int lane_traceback_walk(const TileArgs &a, const TileSpan &s, int lane,
                                const LaneState &ls, const Ring &ring, uint32_t *up_r,
                                uint32_t *left_r, LaneWalk &w) {
  const long t = s.t0 + lane;
  w.walked = t < a.n && ls.ok && ls.score <= a.k;
  w.e = WalkEnd{0, 0, 0, false};
  w.ups = GapRuns{up_r, 0, 0u};
  w.lefts = GapRuns{left_r, 0, 0u};
  if (!w.walked) return 0;
  w.e = lane_walk<T>(ls.c, ring, up_r, left_r, w.ups, w.lefts);
  return w.e.bad ? 4 : 0;
}

// The lane's two strings written into its slot of the output staging in
// reading order (the reference emits from the alignment end and reverses in
// place, src/cuda-functions.cu:306-307, which leaves the same bytes).  The
// staging is zero-filled before, which gives the slot's tail past the
// strings.  The read string takes read bytes col.., the window string window
// bytes row.., from the cell where the walk ended.
SARU_HD void lane_write_strings(const TileArgs &a, const TileSpan &s, int lane,
                                const uint8_t *st_reads, const uint8_t *st_win, uint8_t *out_r,
                                uint8_t *out_g, const LaneState &ls, const LaneWalk &w) {
  if (!w.walked) return;
  const long slot = ls.gs + (long)a.k * (s.t0 + lane);
  expand_string(out_r + (slot - s.o_base_r), w.e.n, st_reads + (ls.rs - s.r_base) + w.e.col,
                w.ups);
  expand_string(out_g + (slot - s.o_base_g), w.e.n, st_win + (ls.gs - s.g_base) + w.e.row,
                w.lefts);
}

// Lays the runs of g that meet steps [lo, lo + 16) over word (2 bits a
// step), from run index *i on (runs before it end before lo).
SARU_HD uint32_t overlay_runs(uint32_t word, int lo, const GapRuns g, int &i, uint32_t code) {
  auto run_at = [&](int j) -> uint32_t { return j < g.n ? g.r[j] : (j == g.n ? g.open : 0u); };
  while (run_len(run_at(i)) && run_first(run_at(i)) + run_len(run_at(i)) <= lo) ++i;
  for (int j = i;; ++j) {
    const uint32_t r = run_at(j);
    if (!run_len(r) || run_first(r) >= lo + 16) break;
    const int f = run_first(r), e = f + run_len(r) - lo;
    const int s0 = f > lo ? f - lo : 0;  // steps [s0, s1) of this word
    const int s1 = e < 16 ? e : 16;
    const uint32_t mk =
        (s1 >= 16 ? 0xFFFFFFFFu : ((1u << (2 * s1)) - 1u)) & ~((1u << (2 * s0)) - 1u);
    word = (word & ~mk) | (code & mk);
  }
  return word;
}

// Words 1 .. nwords-1 of a compact record from a walk: 2-bit steps in
// traceback order, DIAG (01) except over the gap runs, zero past step n.
template <class StoreWord>
SARU_HD void expand_record(int n, const GapRuns ups, const GapRuns lefts, int nwords,
                           StoreWord store) {
  int ui = 0, li = 0;
  for (int w = 1; w < nwords; ++w) {
    const int lo = 16 * (w - 1);  // first step of word w
    uint32_t word = 0;
    if (lo < n) {
      word = n - lo >= 16 ? 0x55555555u : (0x55555555u & ((1u << (2 * (n - lo))) - 1u));
      word = overlay_runs(word, lo, ups, ui, 0xAAAAAAAAu);
      word = overlay_runs(word, lo, lefts, li, 0xFFFFFFFFu);
    }
    store(w, word);
  }
}

// Traceback of one lane into its compact record.  store(w, v) writes word w
// of candidate t's record.
template <typename T, class Ring, class StoreWord>
SARU_HD int lane_traceback_ops(const TileArgs &a, const TileSpan &s, int lane,
                               const LaneState &ls, const Ring &ring, StoreWord store) {
  const long t = s.t0 + lane;
  if (t >= a.n) return 0;
  // every word of the record is written (steps, then zeros), so a record's
  // bytes do not depend on what the buffer held before
  const int nwords = (int)(a.rec_bytes / 4);
  if (!ls.ok || ls.score > a.k) {
    for (int w = 0; w < nwords; ++w) store(w, 0u);
    return 0;
  }
  uint32_t up_r[kMaxGapRuns], left_r[kMaxGapRuns];
  GapRuns ups, lefts;
  const WalkEnd e = lane_walk<T>(ls.c, ring, up_r, left_r, ups, lefts);
  expand_record(e.n, ups, lefts, nwords, store);
  store(0, (uint32_t)e.n | (e.bad ? 0x10000u : 0u));
  return e.bad ? 4 : 0;
}

// Shared-memory slice sizes for a maximum read length and k.
struct SliceLayout {
  long rs_bytes, ws_bytes, region_bytes, warp_smem;
};

SARU_HD SliceLayout slice_layout(int max_m, int k, bool wide) {
  SliceLayout L;
  const long code_words = max_m / 8 + 1;
  const long mwords = mask_words(k, max_m + 2 * k);
  // staged bytes, 16 bytes of alignment head and 48 of slack for the word
  // readers (load4 reads up to 7 bytes past its position; the 32-position
  // chunks of build_codes_acgt reach 31 positions past a window's end)
  L.rs_bytes = (32L * max_m + 16 + 48 + 15) & ~15L;
  L.ws_bytes = (32L * (max_m + 2 * k) + 16 + 48 + 15) & ~15L;
  const long cm = 4L * 32 * (code_words + NCODES * mwords);
  const long out = out_area_bytes(max_m, k);
  long r = cm > out ? cm : out;
  if (r < ring_bytes(wide)) r = ring_bytes(wide);
  L.region_bytes = (r + 15) & ~15L;
  L.warp_smem = L.rs_bytes + L.ws_bytes + L.region_bytes;
  return L;
}

}  // namespace saru
