// Host emulation of the banded kernel's warp loop (saruman_b200/csrc/
// kernels.cu, saru_band_kernel) over band_tile.cuh, for CPU tests.  Each
// warp's phases run lane by lane in the order the kernel's warp barriers
// impose.  Built with AddressSanitizer and exactly-sized buffers (shared
// slices, planes, inputs, outputs), it checks the kernel's index arithmetic
// on the CPU before the kernel runs on a GPU.  Test infrastructure only.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../saruman_b200/csrc/band_tile.cuh"

using namespace saru;

// Byte offset of column j's plane pair of lane pslot (the kernel's layout).
template <typename T>
static long pair_off(int j, long pstride, long pslot) {
  return (plane_unit_of<T>(j) * pstride + pslot) * kPlaneUnit + plane_half_of<T>(j);
}

// A lane's asynchronous copies (cp.async in the kernel), emulated: a copy
// takes its source bytes when issued and lands only at a wait that covers
// its group; copies landing at one wait land newest first.  So a slot
// refilled before the copy that held it has landed ends up with the older
// bytes, and the oracle comparison fails.
struct AsyncCopies {
  struct C {
    uint8_t *dst;
    uint8_t data[16];
    size_t n;
    long group;
  };
  std::vector<C> pending;
  long open = 0;  // the group the copies issued since the last commit join
  void copy(void *dst, const void *src, size_t n) {
    C c;
    c.dst = static_cast<uint8_t *>(dst);
    memcpy(c.data, src, n);
    c.n = n;
    c.group = open;
    pending.push_back(c);
  }
  void commit() { ++open; }
  void wait(long keep) {  // at most `keep` committed groups stay in flight
    const long limit = open - keep;
    for (long i = (long)pending.size() - 1; i >= 0; --i)
      if (pending[(size_t)i].group < limit)
        memcpy(pending[(size_t)i].dst, pending[(size_t)i].data, pending[(size_t)i].n);
    std::vector<C> rest;
    for (const C &c : pending)
      if (c.group >= limit) rest.push_back(c);
    pending.swap(rest);
  }
  void wait_all() { wait(-1); }
};

// The walk's plane ring of one lane over emulated asynchronous copies (one
// copy group a column, as in the kernel).
template <typename T>
static auto host_ring(uint8_t *region, int lane, const uint8_t *planes, long pstride, long pslot,
                      AsyncCopies *ac) {
  return plane_ring<T>(
      reinterpret_cast<PlanePair<T> *>(region) + lane,
      [=](PlanePair<T> *dst, int j) {
        ac->copy(dst, planes + pair_off<T>(j, pstride, pslot), sizeof(PlanePair<T>));
        ac->commit();
      },
      [=] { ac->wait(kRing - 1); });
}

template <typename T>
static int run(const TileArgs &a0, int nwarps_total) {
  TileArgs a = a0;
  const SliceLayout S = slice_layout(a.max_m, a.k, sizeof(T) == 8);
  a.rs_bytes = S.rs_bytes;
  a.ws_bytes = S.ws_bytes;
  a.region_bytes = S.region_bytes;
  a.pstride = (long)nwarps_total * 32;
  std::vector<uint8_t> planes_v((size_t)plane_units(a.max_m, sizeof(T) == 8) * a.pstride *
                                kPlaneUnit);
  uint8_t *planes = planes_v.data();
  int status = 0;
  auto ld16 = [](uint8_t *d, const uint8_t *g) { memcpy(d, g, 16); };
  auto ld1 = [](const uint8_t *g) -> uint8_t { return *g; };
  auto st16 = [](uint8_t *g, const uint8_t *d) { memcpy(g, d, 16); };
  for (int gwarp = 0; gwarp < nwarps_total; ++gwarp) {
    // the three parts of a warp's shared slice, each its own exactly-sized
    // 16-aligned allocation so an overrun of any part is caught
    uint8_t *st_reads = (uint8_t *)aligned_alloc(16, (size_t)S.rs_bytes);
    uint8_t *st_win = (uint8_t *)aligned_alloc(16, (size_t)S.ws_bytes);
    uint8_t *region = (uint8_t *)aligned_alloc(16, (size_t)S.region_bytes);
    memset(st_reads, 0xA5, (size_t)S.rs_bytes);
    memset(st_win, 0xA5, (size_t)S.ws_bytes);
    memset(region, 0xA5, (size_t)S.region_bytes);
    uint32_t *region32 = reinterpret_cast<uint32_t *>(region);
    for (long wt = gwarp; a.t0 + wt * 32 < a.n; wt += nwarps_total) {
      const TileSpan s = tile_span(a, wt);
      if (!s.fits) {
        for (int lane = 0; lane < 32; ++lane)
          if (s.t0 + lane < a.n) a.scores[s.t0 + lane] = a.k + 1;
        status |= 1;
        continue;
      }
      for (int lane = 0; lane < 32; ++lane) {
        stage_in(st_reads, a.reads, s.r_lo, s.r_hi, s.r_base, lane, ld16, ld1);
        stage_in(st_win, a.genome, s.g_lo, s.g_hi, s.g_base, lane, ld16, ld1);
      }
      LaneState ls[32];
      for (int lane = 0; lane < 32; ++lane) {
        const long pslot = (long)gwarp * 32 + lane;
        status |= lane_fill<T>(
            a, s, lane, st_reads, st_win, region32, ls[lane],
            plane_writer<T>(
                [&](long u, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
                  const uint32_t v[4] = {x, y, z, w};
                  memcpy(planes + (u * a.pstride + pslot) * kPlaneUnit, v, 16);
                }));
      }
      // the walk's plane ring in the region, over emulated asynchronous copies
      if (a.records) {  // compact records straight to the (exactly sized) output
        for (int lane = 0; lane < 32; ++lane) {
          uint32_t *rec = reinterpret_cast<uint32_t *>(a.records + (s.t0 + lane) * a.rec_bytes);
          AsyncCopies ac;
          status |= lane_traceback_ops<T>(
              a, s, lane, ls[lane],
              host_ring<T>(region, lane, planes, a.pstride, (long)gwarp * 32 + lane, &ac),
              [&](int w, uint32_t v) { rec[w] = v; });
          ac.wait_all();
        }
        continue;
      }
      uint32_t up_r[32][kMaxGapRuns], left_r[32][kMaxGapRuns];
      LaneWalk walks[32];
      for (int lane = 0; lane < 32; ++lane) {
        AsyncCopies ac;
        status |= lane_traceback_walk<T>(
            a, s, lane, ls[lane],
            host_ring<T>(region, lane, planes, a.pstride, (long)gwarp * 32 + lane, &ac),
            up_r[lane], left_r[lane], walks[lane]);
        ac.wait_all();
      }
      uint8_t *out_r = region, *out_g = region + s.o_span_r;
      const long out_bytes = out_area_bytes(a.max_m, a.k);
      memset(region, 0, (size_t)out_bytes);
      for (int lane = 0; lane < 32; ++lane)
        lane_write_strings(a, s, lane, st_reads, st_win, out_r, out_g, ls[lane], walks[lane]);
      for (int lane = 0; lane < 32; ++lane) {
        stage_out(a.read_aln, out_r, s.s_lo, s.s_hi, s.o_base_r, lane, st16);
        stage_out(a.genome_aln, out_g, s.s_lo, s.s_hi, s.o_base_g, lane, st16);
      }
    }
    free(st_reads);
    free(st_win);
    free(region);
  }
  return status;
}

// Aligns a call with the emulated kernel.  Buffers are the caller's (the
// Python side passes exactly-sized copies, at chosen misalignments).
extern "C" int tile_align_batch(const uint8_t *genome, const uint8_t *reads, const int *goff,
                                const int *roff, const int8_t *dirs, long n, int k, int max_m,
                                int wide, int first_of_call, int nwarps, int *scores,
                                uint8_t *ra, uint8_t *ga) {
  TileArgs a{genome, reads, goff, roff, dirs, n, k, max_m, first_of_call, scores, ra, ga,
             nullptr, 0, 0, 0, 0};
  return wide ? run<uint64_t>(a, nwarps) : run<uint32_t>(a, nwarps);
}

// The same call in slices of `slice` candidates (a multiple of 32), each a
// launch over candidates [t0, t1) of the whole call, as the host entry
// point streams a large call.
extern "C" int tile_align_slices(const uint8_t *genome, const uint8_t *reads, const int *goff,
                                 const int *roff, const int8_t *dirs, long n, int k, int max_m,
                                 int wide, int first_of_call, int nwarps, long slice, int *scores,
                                 uint8_t *ra, uint8_t *ga) {
  int status = 0;
  for (long t0 = 0; t0 < n; t0 += slice) {
    TileArgs a{genome, reads, goff, roff, dirs, t0 + slice < n ? t0 + slice : n, k, max_m,
               first_of_call, scores, ra, ga, nullptr, 0, 0, 0, 0, nullptr, 0, t0};
    status |= wide ? run<uint64_t>(a, nwarps) : run<uint32_t>(a, nwarps);
  }
  return status;
}

// The same call with compact records (rec_bytes per candidate) instead of
// slot strings.
extern "C" int tile_align_compact(const uint8_t *genome, const uint8_t *reads, const int *goff,
                                  const int *roff, const int8_t *dirs, long n, int k, int max_m,
                                  int wide, int first_of_call, int nwarps, int *scores,
                                  uint8_t *records, long rec_bytes) {
  TileArgs a{genome, reads, goff, roff, dirs, n, k, max_m, first_of_call, scores, nullptr,
             nullptr, nullptr, 0, 0, 0, 0, records, rec_bytes};
  return wide ? run<uint64_t>(a, nwarps) : run<uint32_t>(a, nwarps);
}

// Multi-call launch (saru_band_kernel with a segment table): tiles of all
// segments in table order, the shared slice sized for the largest read
// length and k of the launch, one plane buffer for both band widths.
struct HostSeg {
  const uint8_t *genome, *reads;
  const int *goff, *roff;
  const int8_t *dirs;
  int *scores;
  uint8_t *ra, *ga;
  long n;
  int k, max_m, first_of_call, wide;
};

extern "C" int tile_align_multi(const HostSeg *segs, int nseg, int nwarps_total) {
  int max_m = 0, max_k = 0, wide_any = 0;
  std::vector<long> tile_begin(nseg);
  long tiles = 0;
  for (int i = 0; i < nseg; ++i) {
    tile_begin[i] = tiles;
    tiles += (segs[i].n + 31) / 32;
    if (segs[i].max_m > max_m) max_m = segs[i].max_m;
    if (segs[i].k > max_k) max_k = segs[i].k;
    wide_any |= segs[i].wide;
  }
  const SliceLayout S = slice_layout(max_m, max_k, wide_any != 0);
  const long pstride = (long)nwarps_total * 32;
  // exactly the bytes the launcher reserves for the planes
  std::vector<uint8_t> planes_v((size_t)plane_units(max_m, wide_any != 0) * pstride * kPlaneUnit);
  int status = 0;
  auto ld16 = [](uint8_t *d, const uint8_t *g) { memcpy(d, g, 16); };
  auto ld1 = [](const uint8_t *g) -> uint8_t { return *g; };
  auto st16 = [](uint8_t *g, const uint8_t *d) { memcpy(g, d, 16); };
  struct Slice {
    uint8_t *st_reads, *st_win, *region;
    LaneState ls[32];
    long tile = -1;
    int seg = 0;
    TileSpan span;
  };
  std::vector<Slice> W(nwarps_total);
  for (auto &w : W) {
    w.st_reads = (uint8_t *)aligned_alloc(16, (size_t)S.rs_bytes);
    w.st_win = (uint8_t *)aligned_alloc(16, (size_t)S.ws_bytes);
    w.region = (uint8_t *)aligned_alloc(16, (size_t)S.region_bytes);
  }
  auto targs = [&](int si) {
    const HostSeg &g = segs[si];
    return TileArgs{g.genome, g.reads, g.goff, g.roff, g.dirs, g.n, g.k, g.max_m,
                    g.first_of_call, g.scores, g.ra, g.ga, planes_v.data(), pstride,
                    S.rs_bytes, S.ws_bytes, S.region_bytes};
  };
  // rounds: every warp takes a tile, all fills run, then all tracebacks --
  // the interleaving in which one lane's planes could clobber another's
  for (long base = 0; base < tiles; base += nwarps_total) {
    for (int gw = 0; gw < nwarps_total; ++gw) {
      Slice &w = W[gw];
      w.tile = base + gw < tiles ? base + gw : -1;
      if (w.tile < 0) continue;
      int lo = 0, hi = nseg - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_begin[mid] <= w.tile) lo = mid;
        else hi = mid - 1;
      }
      w.seg = lo;
      const TileArgs a = targs(lo);
      w.span = tile_span(a, w.tile - tile_begin[lo]);
      if (!w.span.fits) {
        status |= 1;
        w.tile = -1;
        continue;
      }
      auto fill = [&](auto tag) {
        using T = decltype(tag);
        uint8_t *planes = planes_v.data();
        for (int lane = 0; lane < 32; ++lane) {
          stage_in(w.st_reads, a.reads, w.span.r_lo, w.span.r_hi, w.span.r_base, lane, ld16, ld1);
          stage_in(w.st_win, a.genome, w.span.g_lo, w.span.g_hi, w.span.g_base, lane, ld16, ld1);
        }
        for (int lane = 0; lane < 32; ++lane) {
          const long pslot = (long)gw * 32 + lane;
          status |= lane_fill<T>(
              a, w.span, lane, w.st_reads, w.st_win, reinterpret_cast<uint32_t *>(w.region),
              w.ls[lane],
              plane_writer<T>(
                  [&](long u, uint32_t x, uint32_t y, uint32_t z, uint32_t q) {
                    const uint32_t v[4] = {x, y, z, q};
                    memcpy(planes + (u * pstride + pslot) * kPlaneUnit, v, 16);
                  }));
        }
      };
      if (segs[lo].wide) fill(uint64_t(0));
      else fill(uint32_t(0));
    }
    for (int gw = 0; gw < nwarps_total; ++gw) {
      Slice &w = W[gw];
      if (w.tile < 0) continue;
      const TileArgs a = targs(w.seg);
      auto trace = [&](auto tag) {
        using T = decltype(tag);
        uint8_t *planes = planes_v.data();
        uint32_t up_r[32][kMaxGapRuns], left_r[32][kMaxGapRuns];
        LaneWalk walks[32];
        for (int lane = 0; lane < 32; ++lane) {
          const long pslot = (long)gw * 32 + lane;
          AsyncCopies ac;
          status |= lane_traceback_walk<T>(
              a, w.span, lane, w.ls[lane],
              host_ring<T>(w.region, lane, planes, pstride, pslot, &ac), up_r[lane],
              left_r[lane], walks[lane]);
          ac.wait_all();
        }
        const long out_bytes = out_area_bytes(a.max_m, a.k);
        memset(w.region, 0, (size_t)out_bytes);
        uint8_t *out_r = w.region, *out_g = w.region + w.span.o_span_r;
        for (int lane = 0; lane < 32; ++lane)
          lane_write_strings(a, w.span, lane, w.st_reads, w.st_win, out_r, out_g, w.ls[lane],
                             walks[lane]);
        for (int lane = 0; lane < 32; ++lane) {
          stage_out(a.read_aln, out_r, w.span.s_lo, w.span.s_hi, w.span.o_base_r, lane, st16);
          stage_out(a.genome_aln, out_g, w.span.s_lo, w.span.s_hi, w.span.o_base_g, lane, st16);
        }
      };
      if (segs[w.seg].wide) trace(uint64_t(0));
      else trace(uint32_t(0));
    }
  }
  for (auto &w : W) {
    free(w.st_reads);
    free(w.st_win);
    free(w.region);
  }
  return status;
}
