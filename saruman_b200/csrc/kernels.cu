// kernels.cu -- sm_100a kernels of the alignment stage.
//
//  saru_band_kernel<T, CTA>   the production path: one thread per candidate,
//                             bit-parallel banded fill (saru_core.cuh) with
//                             2-bit traceback decisions, traceback and slot
//                             output on the device.
//  saru_full_fill_kernel      the exact full-rectangle path for inputs the
//  saru_full_trace_kernel     banded kernel does not cover (other costs,
//                             m <= 3k, k > 15, irregular windows): the
//                             reference's int16 recurrence over a device
//                             arena holding every matrix of the call, then
//                             its traceback over that arena.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"
#include "saru_core.cuh"

namespace saru {

__device__ __forceinline__ long gstart_of(const int32_t *goff, long t) { return t ? goff[t - 1] : 0; }

// ---------------------------------------------------------------------------
// banded kernel
// ---------------------------------------------------------------------------

// Cooperative zero fill of bytes [lo, hi): 16-byte stores for the aligned
// middle, byte stores at the edges.
__device__ __forceinline__ void zero_range(uint8_t *base, long lo, long hi, int tid, int nthr) {
  const long a16 = (lo + 15) & ~15L, b16 = hi & ~15L;
  if (a16 >= b16) {
    for (long i = lo + tid; i < hi; i += nthr) base[i] = 0;
    return;
  }
  for (long i = lo + tid; i < a16; i += nthr) base[i] = 0;
  uint4 *v = reinterpret_cast<uint4 *>(base + a16);
  const long nv = (b16 - a16) >> 4;
  for (long i = tid; i < nv; i += nthr) v[i] = make_uint4(0, 0, 0, 0);
  for (long i = b16 + tid; i < hi; i += nthr) base[i] = 0;
}

template <typename T, int CTA>
__global__ void __launch_bounds__(CTA) saru_band_kernel(KernelArgs a) {
  extern __shared__ uint32_t smem[];
  const int tid = threadIdx.x;
  const long slot_id = (long)blockIdx.x * CTA + tid;
  const long sstride = (long)gridDim.x * CTA;
  const int k = a.k;
  const int code_words = (a.max_m + 7) / 8;
  const int mwords = mask_words(k, a.max_m + 2 * k);
  Strided codes{smem + tid, CTA};
  Strided mask{smem + code_words * CTA + tid, CTA};
  T *planes = reinterpret_cast<T *>(a.scratch);
  uint32_t ops[kMaxOpWords];

  for (long tile = blockIdx.x; tile * CTA < a.n; tile += gridDim.x) {
    const long t = tile * CTA + tid;
    {
      // zero the tile's slot bytes (a contiguous range) before any thread
      // writes its strings into them
      const long t0 = tile * CTA, t1 = (t0 + CTA < a.n ? t0 + CTA : a.n);
      const long lo = gstart_of(a.goff, t0) + (long)k * t0;
      const long hi = (long)a.goff[t1 - 1] + (long)k * t1;
      zero_range(a.read_aln, lo, hi, tid, CTA);
      zero_range(a.genome_aln, lo, hi, tid, CTA);
      __syncthreads();
    }
    if (t >= a.n) continue;
    const long gs = gstart_of(a.goff, t), rs = t ? a.roff[t - 1] : 0;
    Cand c;
    c.m = int(a.roff[t] - rs);
    c.L = int(a.goff[t] - gs);
    c.k = k;
    flank_of(a.dirs[t], k, c.so, c.eo);
    c.first_of_call = a.first_of_call && t == 0;
    if (c.L != c.m + c.so + c.eo || c.m <= 3 * k || c.m > a.max_m) {
      atomicOr(a.status, kStatusIrregular);
      a.scores[t] = k + 1;
      continue;
    }
    const uint8_t *rd = a.reads + rs;
    const uint8_t *wn = a.genome + gs;
    auto rdf = [&](int j) -> uint8_t { return __ldg(rd + j); };
    auto wnf = [&](int p) -> uint8_t { return __ldg(wn + p); };
    if (!build_codes(c, rdf, wnf, codes, mask, mwords)) {
      atomicOr(a.status, kStatusAlphabet);
      a.scores[t] = k + 1;
      continue;
    }
    const int score = fill_band<T>(c, codes, mask, mwords, [&](int j, T A, T B) {
      planes[(2 * (long)j) * sstride + slot_id] = A;
      planes[(2 * (long)j + 1) * sstride + slot_id] = B;
    });
    a.scores[t] = score;
    if (score > k) continue;
    int nsteps = 0;
    bool bad = false;
    const int maxs = max_steps(c);
    traceback_band(
        c,
        [&](int j, int b) -> int {
          if (b < 0 || b >= int(sizeof(T) * 8)) {
            bad = true;
            return OP_STOP;
          }
          const T A = planes[(2 * (long)j) * sstride + slot_id];
          const T B = planes[(2 * (long)j + 1) * sstride + slot_id];
          return int((A >> b) & T(1)) | (int((B >> b) & T(1)) << 1);
        },
        [&](int op, int, int) {
          if (nsteps < maxs) {
            if ((nsteps & 15) == 0) ops[nsteps >> 4] = 0;
            ops[nsteps >> 4] |= uint32_t(op) << ((nsteps & 15) * 2);
          }
          ++nsteps;
        });
    if (bad || nsteps > maxs) {
      atomicOr(a.status, kStatusOverflow);
      continue;
    }
    uint8_t *ra = a.read_aln + gs + (long)k * t;
    uint8_t *ga = a.genome_aln + gs + (long)k * t;
    emit_forward(c, ops, nsteps, rdf, wnf, [&](int pos, uint8_t x, uint8_t y) {
      ra[pos] = x;
      ga[pos] = y;
    });
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

template <typename T, int CTA>
static cudaError_t launch_band(const KernelArgs &a, int sms, cudaStream_t s) {
  const size_t smem = band_smem_bytes(a.max_m, a.k, CTA);
  auto kern = saru_band_kernel<T, CTA>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long tiles = (a.n + CTA - 1) / CTA;
  long grid = a.grid > 0 ? a.grid : tiles;
  if (grid > tiles) grid = tiles;
  (void)sms;
  kern<<<(unsigned)grid, CTA, smem, s>>>(a);
  return cudaGetLastError();
}

size_t band_smem_bytes(int max_m, int k, int cta) {
  const int code_words = (max_m + 7) / 8;
  const int mwords = mask_words(k, max_m + 2 * k);
  return sizeof(uint32_t) * (size_t)cta * (size_t)(code_words + NCODES * mwords);
}

cudaError_t launch_band_kernel(const KernelArgs &a, int cta, int sms, cudaStream_t s) {
  if (a.wide) {
    if (cta == 64) return launch_band<uint64_t, 64>(a, sms, s);
    return launch_band<uint64_t, 128>(a, sms, s);
  }
  if (cta == 64) return launch_band<uint32_t, 64>(a, sms, s);
  return launch_band<uint32_t, 128>(a, sms, s);
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
