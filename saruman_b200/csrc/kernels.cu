// kernels.cu -- sm_100a kernels of the alignment stage.
//
//  saru_band_kernel           the production path: persistent warps over
//                             32-candidate tiles (one lane per candidate),
//                             bit-parallel banded fill (saru_core.cuh) with
//                             2-bit traceback decisions, traceback and slot
//                             strings or compact records on the device; a
//                             launch covers segments (calls, or slices
//                             [t0, t1) of one call) of 32- or 64-bit bands.
//  saru_full_fill_kernel      the exact full-rectangle path for inputs the
//  saru_full_trace_kernel     banded kernel does not cover (other costs,
//                             m <= 3k, k > 15, irregular windows): the
//                             reference's int16 recurrence over a device
//                             arena holding every matrix of the call, then
//                             its traceback over that arena.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "kernels.cuh"
#include "band_tile.cuh"
#include "saru_core.cuh"

namespace saru {

__device__ __forceinline__ long gstart_of(const int32_t *goff, long t) { return t ? goff[t - 1] : 0; }

// ---------------------------------------------------------------------------
// banded kernel: persistent warps over warp tiles (band_tile.cuh)
// ---------------------------------------------------------------------------

// One warp tile of one segment (the phases of band_tile.cuh).
template <typename T>
__device__ __forceinline__ int band_tile(const TileArgs &ta, long wt, int lane, uint8_t *st_reads,
                                         uint8_t *st_win, uint8_t *region, void *planes_v,
                                         long pslot) {
  // this lane's plane units: unit u at lane_units + u * row_bytes (a unit
  // row of the whole grid's lanes is a few MB, so the offset of a unit is a
  // 32-bit product widened by one multiply-add)
  uint8_t *lane_units = reinterpret_cast<uint8_t *>(planes_v) + pslot * kPlaneUnit;
  const uint32_t row_bytes = (uint32_t)(ta.pstride * kPlaneUnit);
  auto pair_at = [&](int j) -> PlanePair<T> * {
    return reinterpret_cast<PlanePair<T> *>(
        lane_units + (unsigned long long)(uint32_t)plane_unit_of<T>(j) * row_bytes +
        plane_half_of<T>(j));
  };
  uint32_t *region32 = reinterpret_cast<uint32_t *>(region);
  auto ld16 = [](uint8_t *d, const uint8_t *g) {
    *reinterpret_cast<uint4 *>(d) = __ldg(reinterpret_cast<const uint4 *>(g));
  };
  auto ld1 = [](const uint8_t *g) -> uint8_t { return __ldg(g); };
  auto st16 = [](uint8_t *g, const uint8_t *d) {
    *reinterpret_cast<uint4 *>(g) = *reinterpret_cast<const uint4 *>(d);
  };
  const TileSpan s = tile_span(ta, wt);
  if (!s.fits) {  // offsets no regular call can have: report, do not stage
    const long t = s.t0 + lane;
    if (t < ta.n) ta.scores[t] = ta.k + 1;
    return 1;
  }
  stage_in(st_reads, ta.reads, s.r_lo, s.r_hi, s.r_base, lane, ld16, ld1);
  stage_in(st_win, ta.genome, s.g_lo, s.g_hi, s.g_base, lane, ld16, ld1);
  __syncwarp();
  LaneState ls;
  int st = lane_fill<T>(
      ta, s, lane, st_reads, st_win, region32, ls,
      plane_writer<T>(
          [&](long u, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
            *reinterpret_cast<uint4 *>(lane_units + (unsigned long long)(uint32_t)u * row_bytes) =
                make_uint4(x, y, z, w);
          }));
  __syncwarp();
  // the traceback walk's plane ring in the region: asynchronous 8- or
  // 16-byte copies from the plane scratch, one copy group per column
  const auto ring = plane_ring<T>(
      reinterpret_cast<PlanePair<T> *>(region) + lane,
      [&](PlanePair<T> *dst, int j) {
        const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
        const size_t g = __cvta_generic_to_global(pair_at(j));
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(g),
                     "n"((int)sizeof(PlanePair<T>))
                     : "memory");
        asm volatile("cp.async.commit_group;\n" ::: "memory");
      },
      [] { asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 1) : "memory"); });
  if (ta.records) {  // compact records straight to global memory
    uint32_t *rec = reinterpret_cast<uint32_t *>(ta.records + (s.t0 + lane) * ta.rec_bytes);
    st |= lane_traceback_ops<T>(ta, s, lane, ls, ring, [&](int w, uint32_t v) { rec[w] = v; });
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    return st;
  }
  uint32_t up_r[kMaxGapRuns], left_r[kMaxGapRuns];
  LaneWalk w;
  st |= lane_traceback_walk<T>(ta, s, lane, ls, ring, up_r, left_r, w);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();
  uint8_t *out_r = region;
  uint8_t *out_g = region + s.o_span_r;
  const long out_bytes = out_area_bytes(ta.max_m, ta.k);
  {
    uint4 *p4 = reinterpret_cast<uint4 *>(region);
    const long nv = out_bytes >> 4;
    for (long i = lane; i < nv; i += 32) p4[i] = make_uint4(0, 0, 0, 0);
  }
  __syncwarp();
  lane_write_strings(ta, s, lane, st_reads, st_win, out_r, out_g, ls, w);
  __syncwarp();
  stage_out(ta.read_aln, out_r, s.s_lo, s.s_hi, s.o_base_r, lane, st16);
  stage_out(ta.genome_aln, out_g, s.s_lo, s.s_hi, s.o_base_g, lane, st16);
  __syncwarp();
  return st;
}

// Persistent warps take 32-candidate tiles from a launch-wide counter; a
// tile belongs to one segment (a call with its own m, k and band width).
// The bounds hold the kernel to 128 registers a thread: above that an SM
// sub-partition's register file holds 3 of these warps instead of 4.
__global__ void __launch_bounds__(128, 4) saru_band_kernel(const __grid_constant__ KernelArgs a) {
  extern __shared__ uint4 smem_v[];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const int WARPS = blockDim.x >> 5;
  uint8_t *ws = reinterpret_cast<uint8_t *>(smem_v) + (long)wid * a.warp_smem;
  uint8_t *st_reads = ws;
  uint8_t *st_win = ws + a.rs_bytes;
  uint8_t *region = st_win + a.ws_bytes;
  const long gwarp = (long)blockIdx.x * WARPS + wid;
  const long pstride = (long)gridDim.x * WARPS * 32;
  const long pslot = gwarp * 32 + lane;
  for (;;) {
    int tile = 0;
    if (lane == 0) tile = atomicAdd(a.counter, 1);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= a.total_tiles) break;
    int lo = 0, hi = a.nseg - 1;  // last segment with tile_begin <= tile
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.segs[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const Segment &g = a.segs[lo];
    const TileArgs ta{g.genome, g.reads, g.goff, g.roff, g.dirs, g.n, g.k, g.max_m,
                      g.first_of_call, g.scores, g.read_aln, g.genome_aln, a.planes, pstride,
                      a.rs_bytes, a.ws_bytes, a.warp_smem - a.rs_bytes - a.ws_bytes,
                      g.records, g.rec_bytes, g.t0};
    const long wt = tile - g.tile_begin;
    int status = g.wide ? band_tile<uint64_t>(ta, wt, lane, st_reads, st_win, region, a.planes, pslot)
                        : band_tile<uint32_t>(ta, wt, lane, st_reads, st_win, region, a.planes, pslot);
    status = __reduce_or_sync(0xffffffffu, status);
    if (status && lane == 0)
      atomicOr(g.status, (status & 1 ? kStatusIrregular : 0) | (status & 2 ? kStatusAlphabet : 0) |
                             (status & 4 ? kStatusOverflow : 0));
  }
}

// ---------------------------------------------------------------------------
// exact full-rectangle path
// ---------------------------------------------------------------------------

__device__ __forceinline__ short min3s(short x, short y, short z) {
  short r = x;
  if (r > y) r = y;
  if (r > z) r = z;
  return r;
}

__global__ void saru_full_fill_kernel(FullArgs a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long gs = gstart_of(a.goff, t), rs = t ? a.roff[t - 1] : 0;
  const long m = a.roff[t] - rs, L = a.goff[t] - gs, W = m + 1;
  int so, eo;
  flank_of(a.dirs[t], a.k, so, eo);
  short *M = a.arena + a.eoff[t];
  const uint8_t *g = a.genome + gs, *r = a.reads + rs;
  for (long j = 0; j <= m; ++j) M[j] = (short)j;
  for (long i = 1; i <= L; ++i) M[i * W] = (short)(i < 2 * so + 1 ? M[(i - 1) * W] : M[(i - 1) * W] + 1);
  for (long i = 0; i < L; ++i) {
    const short *up = M + i * W;
    short *cur = M + (i + 1) * W;
    const uint8_t gi = g[i];
    for (long j = 0; j < m; ++j) {
      const int corr = (j == m - 1 && i >= L - 2 * eo) ? a.mismatch : 0;
      const short d = (short)(up[j] + (gi != r[j] ? a.mismatch : a.match));
      const short l = (short)(cur[j] + a.mismatch);
      const short u = (short)(up[j + 1] + a.mismatch - corr);
      cur[j + 1] = min3s(d, l, u);
    }
  }
  a.scores[t] = M[W * (L + 1) - 1];
}

__device__ __forceinline__ short arena_cell(const FullArgs &a, long P) { return a.arena[P]; }

// The reference traceback (src/cuda-functions.cu:108-315) over the arena of
// absolute cells; stops with an overflow flag instead of leaving the slot.
__global__ void saru_full_trace_kernel(FullArgs a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  if (a.scores[t] > a.k) return;
  const long gs = gstart_of(a.goff, t), rs = t ? a.roff[t - 1] : 0;
  const long m = a.roff[t] - rs, L = a.goff[t] - gs, W = m + 1;
  int so, eo;
  flank_of(a.dirs[t], a.k, so, eo);
  const long base = a.eoff[t];
  const long slot = gs + (long)a.k * t;
  const long slot_end = slot + L + a.k;
  long P = base + (L + 1) * W - 1;
  long ap = slot;
  // the loop bound is on the absolute cell index, as in the reference
  while (P >= W) {
    const short v = arena_cell(a, P);
    short dg, lf, tp;
    if (P % W != 0) {
      dg = arena_cell(a, P - W - 1);
      lf = arena_cell(a, P - 1);
    } else {
      dg = 999;
      lf = 999;
    }
    tp = P != 0 ? arena_cell(a, P - W) : (short)999;
    short width = 0;
    const short width_tmp = (short)((P % W) - 1);
    if (width_tmp > 0) width = width_tmp;
    const short h_tmp = (short)(((P - base - width) / W) - 1);
    const short height = h_tmp > 0 ? h_tmp : 0;
    const int corr =
        ((width == m - 1 && height >= L - 2 * eo) || (so && width == 0 && height <= (so + 1) * 2))
            ? a.mismatch
            : 0;
    const long gi = gs + height, ri = rs + width;
    uint8_t gch = 0, rch = 0;
    if (gi >= 0 && gi < a.genome_bytes) gch = a.genome[gi];
    else atomicOr(a.status, kStatusUndefined);
    if (ri >= 0 && ri < a.read_bytes) rch = a.reads[ri];
    else atomicOr(a.status, kStatusUndefined);
    uint8_t oa, ob;
    long step;
    if (dg + a.mismatch == v) {
      oa = rch; ob = gch; step = W + 1;
    } else if (dg + a.match == v && gch == rch) {
      oa = rch; ob = gch; step = W + 1;
    } else if (tp + a.mismatch - corr == v) {
      oa = '_'; ob = gch; step = W;
    } else if (lf + a.mismatch == v) {
      oa = rch; ob = '_'; step = 1;
    } else {
      break;
    }
    if (ap >= slot_end) {
      atomicOr(a.status, kStatusOverflow);
      break;
    }
    a.read_aln[ap] = oa;
    a.genome_aln[ap] = ob;
    ++ap;
    P -= step;
  }
  for (long i = slot, j = ap - 1; i < j; ++i, --j) {
    uint8_t x = a.read_aln[i]; a.read_aln[i] = a.read_aln[j]; a.read_aln[j] = x;
    x = a.genome_aln[i]; a.genome_aln[i] = a.genome_aln[j]; a.genome_aln[j] = x;
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

constexpr long kMaxCtaSmem = 227 * 1024;  // opt-in shared memory per block on sm_100

BandLayout band_layout(int max_m, int k, int warps_req, bool wide) {
  const SliceLayout S = slice_layout(max_m, k, wide);
  BandLayout L;
  L.rs_bytes = S.rs_bytes;
  L.ws_bytes = S.ws_bytes;
  L.region_bytes = S.region_bytes;
  L.warp_smem = S.warp_smem;
  long w = kMaxCtaSmem / S.warp_smem;
  L.warps = (int)(w >= 4 ? 4 : (w >= 2 ? 2 : (w >= 1 ? 1 : 0)));
  if (warps_req >= 1 && warps_req < L.warps) L.warps = warps_req;
  L.cta_smem = S.warp_smem * L.warps;
  return L;
}

namespace {
// The opt-in shared-memory limit is an attribute of the kernel on one
// device: set once per device, under a lock, before the first launch there.
std::mutex g_attr_mu;
uint64_t g_attr_done;  // bit d set once device d allows it

cudaError_t allow_smem() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if ((g_attr_done >> dev) & 1u) return cudaSuccess;
  e = cudaFuncSetAttribute(saru_band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kMaxCtaSmem);
  if (e == cudaSuccess) g_attr_done |= 1ull << dev;
  return e;
}
}  // namespace

cudaError_t launch_band_kernel(KernelArgs &a, cudaStream_t s) {
  const BandLayout L = band_layout(a.max_m, a.max_k, a.warps_req, a.wide_any != 0);
  if (L.warps < 1 || a.nseg < 1 || a.nseg > kMaxSegs) return cudaErrorInvalidValue;
  // allow the largest slice once per device; each launch asks for its own
  // size (a per-launch attribute would race between concurrent callers)
  cudaError_t e = allow_smem();
  if (e != cudaSuccess) return e;
  a.rs_bytes = L.rs_bytes;
  a.ws_bytes = L.ws_bytes;
  a.warp_smem = L.warp_smem;
  e = cudaMemsetAsync(a.counter, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  saru_band_kernel<<<(unsigned)a.grid, 32 * L.warps, L.cta_smem, s>>>(a);
  return cudaGetLastError();
}

long band_grid(int sms, long n, const BandLayout &L, int smem_per_sm, int ctas_cap) {
  const long per_cta = 32L * (L.warps > 0 ? L.warps : 1);
  const long tiles = (n + per_cta - 1) / per_cta;
  long per_sm = smem_per_sm / (L.cta_smem + 1024);
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 16) per_sm = 16;
  if (ctas_cap >= 1 && per_sm > ctas_cap) per_sm = ctas_cap;
  const long g = (long)sms * per_sm;
  return tiles < g ? (tiles > 0 ? tiles : 1) : g;
}

size_t band_scratch_bytes(long grid, int max_m, int k, bool wide, int warps_req) {
  const BandLayout L = band_layout(max_m, k, warps_req, wide);
  return kCounterBytes + (size_t)grid * 32 * (L.warps > 0 ? L.warps : 1) *
                             (size_t)plane_units(max_m, wide) * kPlaneUnit;
}

cudaError_t launch_full_kernels(const FullArgs &a, cudaStream_t s) {
  const int cta = 128;
  const unsigned grid = (unsigned)((a.n + cta - 1) / cta);
  if (grid == 0) return cudaSuccess;
  saru_full_fill_kernel<<<grid, cta, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  saru_full_trace_kernel<<<grid, cta, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace saru
