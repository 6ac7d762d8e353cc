// filter.cu -- the q-gram pair filter on the device.
//
//  index    every q-gram of the resident genome, hashed (64-bit FNV-1a of its
//           bytes) and sorted with its position (a stable radix sort keeps
//           each q-gram's positions in genome order, as the reference's
//           index lists them, src/util.c:462-480); equal hashes of unequal
//           q-grams are reported, not trusted.
//  lookup   one thread per (read, q-gram): the q-gram of the strand-adjusted
//           read, its run in the sorted index (checked against the genome
//           bytes) and, by an exclusive scan per read chunk, its list's
//           offset in the reference's data array (lists in q-gram order per
//           read, each followed by a 0, src/hash.c:404-457).
//  filter   one warp per read, reads taken most estimated work first:
//           filter_read (filter_core.cuh) over that layout, its pair items
//           spread over the lanes, the read's kept positions into its slice
//           of a scratch.
//  calls    the kept positions, packed, copied back and assembled into the
//           reference's calls on the host (filter_calls.h).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <future>
#include <thread>
#include <vector>

#include "../../include/saruman_b200.h"
#include "filter_calls.h"
#include "filter_core.cuh"
#include "server_internal.h"

namespace {

using namespace saru;

constexpr int kHitsPerRead = 4096;   // kept positions per read and strand
constexpr int kReadsPerLaunch = 1 << 16;

__host__ __device__ inline uint64_t qgram_hash(const uint8_t *p, int q) {
  uint64_t h = 1469598103934665603ull;  // FNV-1a 64
  for (int i = 0; i < q; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

__device__ inline uint8_t comp_byte(uint8_t c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return c;
  }
}

__global__ void k_qgram_hash(const uint8_t *g, long npos, int q, uint64_t *hash, uint32_t *pos) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npos;
       p += (long)gridDim.x * blockDim.x) {
    hash[p] = qgram_hash(g + p, q);
    pos[p] = (uint32_t)p;
  }
}

__global__ void k_index_check(const uint64_t *hash, const uint32_t *pos, long n, const uint8_t *g,
                              int q, int *flag) {
  for (long i = 1 + blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    if (hash[i] != hash[i - 1]) continue;
    const uint8_t *a = g + pos[i], *b = g + pos[i - 1];
    for (int j = 0; j < q; ++j)
      if (a[j] != b[j]) {
        atomicOr(flag, 1);
        break;
      }
  }
}

// byte i of the read as its strand aligns it (reverse complement for dr 4)
__device__ inline uint8_t strand_byte(const uint8_t *read, int m, int dr, int i) {
  return dr == 4 ? comp_byte(read[m - 1 - i]) : read[i];
}

struct LookupArgs {
  const uint8_t *reads;  // nreads x m, as sequenced
  long nreads;
  int dr;
  FilterShape S;
  const uint8_t *genome;
  const uint64_t *hash;
  const uint32_t *pos;
  long nidx;
  long *lo;       // nreads x P: first index of the q-gram's run
  long *count;    // nreads x P: list length + 1 (its terminating 0)
};

__global__ void k_lookup(LookupArgs a) {
  const long total = a.nreads * a.S.P;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long r = t / a.S.P;
    const int x = (int)(t % a.S.P);
    const uint8_t *rd = a.reads + r * a.S.m;
    uint8_t key[kFilterMaxQgrams * 4];
    const int q = a.S.q;
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < q; ++i) {
      key[i] = strand_byte(rd, a.S.m, a.dr, a.S.qpos[x] + i);
      h ^= key[i];
      h *= 1099511628211ull;
    }
    long l = 0, u = a.nidx;  // first index with hash >= h
    while (l < u) {
      const long mid = (l + u) >> 1;
      if (a.hash[mid] < h) l = mid + 1;
      else u = mid;
    }
    long e = l, u2 = a.nidx;  // first index with hash > h
    while (e < u2) {
      const long mid = (e + u2) >> 1;
      if (a.hash[mid] <= h) e = mid + 1;
      else u2 = mid;
    }
    long len = e - l;
    if (len > 0) {  // a hash shared with another q-gram: no list
      const uint8_t *gq = a.genome + a.pos[l];
      for (int i = 0; i < q; ++i)
        if (gq[i] != key[i]) {
          len = 0;
          break;
        }
    }
    a.lo[t] = l;
    a.count[t] = len + 1;
  }
}

struct FilterArgs {
  const uint8_t *reads;
  long r0, r1;      // reads of this launch
  long chunk;       // reads per chunk of the reference's data array (its chunk value)
  long nreads;
  int dr;
  FilterShape S;
  const uint8_t *genome;
  long glen;
  const uint32_t *pos;
  const long *lo, *count, *offs;  // per (read, q-gram); offs: exclusive scan of count
  int32_t *hit_pos;               // (r1 - r0) x kHitsPerRead
  int8_t *hit_flag;
  int32_t *n, *queue;             // per read of the launch
  int *status;
  const int32_t *order;           // the launch's reads (0-based in it), most work first
  uint32_t offset;                // genome position of the chunk's first byte
  uint32_t zone_magic;            // ceil(2^32 / (2k + 1)): item / zones by a multiply
};

// The read's lists on the device: the sorted index's run for each q-gram,
// and the data array's flattened offsets for looks past a list.
struct DevLists {
  const FilterArgs *a;
  long base, c0, c1, cend;
  int P;
  const long *lo, *cnt, *offs;  // this read's lists (shared-memory copies)
  uint32_t off;                 // the chunk's genome position: values are whole-genome positions
  __device__ uint32_t len(int x) const { return (uint32_t)(cnt[x] - 1); }
  __device__ uint32_t at(int x, uint32_t i) const {
    const long t = base + x;
    const long c = cnt[x];
    if ((long)i + 1 < c) return a->pos[lo[x] + i] + off;
    if ((long)i + 1 == c) return 0u;
    const long j = offs[x] + (long)i;  // past the list: what follows it
    if (j >= cend) return 0u;
    long l = t;  // the list holding j: a few lists on, or found by bisection
    const long last = c1 * P - 1;
    int step = 0;
    while (l < last && a->offs[l + 1] <= j && step < 8) {
      ++l;
      ++step;
    }
    if (l < last && a->offs[l + 1] <= j) {
      long u = last;
      while (l < u) {
        const long mid = (l + u + 1) >> 1;
        if (a->offs[mid] <= j) l = mid;
        else u = mid - 1;
      }
    }
    const long w = j - a->offs[l];
    return w + 1 < a->count[l] ? a->pos[a->lo[l] + w] + off : 0u;
  }
  __device__ int find(int x, uint32_t from, uint32_t want) const {
    const long end = lo[x] + cnt[x] - 1;  // ascending positions
    long l = lo[x] + from, u = end;
    while (l < u) {
      const long mid = (l + u) >> 1;
      if (a->pos[mid] + off < want) l = mid + 1;
      else u = mid;
    }
    return (l < end && a->pos[l] + off == want) ? (int)(l - lo[x]) : -1;
  }
};

// filter_record (filter_core.cuh) by a whole warp: every lane carries the
// same n, queue and overflow; the kept entries are examined 32 at a time and
// the first that decides (dropped, flag replaced, or dropped as equal) wins,
// as in the sequential loop; with none deciding, lane 0 appends.
__device__ inline void warp_record(ReadHits &h, int lane, int k, int start, int flag) {
  const int dir = flag > 3 ? 1 : 0;
  for (int c0 = 0; c0 < h.n; c0 += 32) {
    const int c = c0 + lane;
    int code = 0;
    if (c < h.n) {
      const int pc = h.pos[c], fc = h.flag[c];
      const int dc = fc > 3 ? 1 : 0;
      const long d1 = (long)pc - start, d2 = -(long)pc - start;
      if (fc <= flag && ((d1 >= -k && d1 <= k) || (d2 >= -k && d2 <= k))) code = 1;
      else if (pc == start && dc == dir && fc > flag) code = 2;
      else if ((pc == start || pc == -start) && dc == dir) code = 3;
    }
    const unsigned any = __ballot_sync(0xffffffffu, code != 0);
    if (any) {
      if (lane == __ffs(any) - 1 && code == 2) h.flag[c] = (int8_t)flag;
      __syncwarp();
      return;
    }
  }
  if (h.n >= h.cap) {
    h.overflow = 1;
    return;
  }
  if (lane == 0) {
    h.pos[h.n] = start;
    h.flag[h.n] = (int8_t)flag;
  }
  ++h.n;
  if (start > 0) ++h.queue;
  __syncwarp();
}

// One warp per read: filter_read (filter_core.cuh) with its pair scans
// spread over the lanes.  For one position of q-gram a the reference counts
// the pairs it finds, in a fixed order (first pass b ascending, zones
// ascending; second pass b ascending, zones ascending; a first-pass scan can
// count its first element twice) and records only the hit that brings the
// count to the threshold.  The lanes evaluate 32 of those items at a time; a
// warp prefix sum over their hit counts finds that hit, and the warp records
// it (and the perfect hit before it) with warp_record, in the reference's
// order.  Warps take the launch's reads in the order `order` gives (most
// estimated work first), so long reads start early and short ones fill in.
__global__ void __launch_bounds__(128) k_filter(FilterArgs fa) {
  const int lane = threadIdx.x & 31;
  const long wi = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32;
  if (wi >= fa.r1 - fa.r0) return;  // the whole warp
  const long lr = fa.order[wi];
  const long r = fa.r0 + lr;
  const FilterShape &S = fa.S;
  const int P = S.P, k = S.k, half = S.half, q = S.q, m = S.m, dr = fa.dr;
  const long c0 = (r / fa.chunk) * fa.chunk, c1 = min(c0 + fa.chunk, fa.nreads);
  __shared__ long s_lo[4][kFilterMaxQgrams], s_cnt[4][kFilterMaxQgrams],
      s_offs[4][kFilterMaxQgrams];
  const int w = threadIdx.x >> 5;
  for (int x = lane; x < P; x += 32) {
    s_lo[w][x] = fa.lo[r * P + x];
    s_cnt[w][x] = fa.count[r * P + x];
    s_offs[w][x] = fa.offs[r * P + x];
  }
  __syncwarp();
  const DevLists L{&fa, r * P, c0, c1, fa.offs[c1 * P - 1] + fa.count[c1 * P - 1], P,
                   s_lo[w], s_cnt[w], s_offs[w], fa.offset};
  const int goff = (int)fa.offset;
  const uint8_t *rd = fa.reads + r * m;
  ReadHits h{fa.hit_pos + lr * kHitsPerRead, fa.hit_flag + lr * kHitsPerRead, kHitsPerRead, 0, 0,
             0};
  const int zones = 2 * k + 1;
  const int need = S.tresh - 1;  // hits before the one that reaches the threshold
  for (int a = 0; a < half; ++a) {
    const int first = a == 0 ? 1 : 0;
    const uint32_t in_read = (uint32_t)a * q + 1;
    const int n1 = (half - 1 - a) * zones;
    int n2 = 0;
    for (int b = 0; b < half; ++b) n2 += 2 * abs(half - 1 - b - a) + 1;
    uint32_t off = 0;
    uint32_t pa = L.at(a, off);
    while (pa > 0) {
      const int gs = (int)(pa - in_read);
      if (gs + 1 - goff > 0) {  // a start after the chunk's first byte
        const long g1 = gs + 1, l1 = g1 - goff;  // in the genome, in the chunk
        bool eq = l1 + m <= fa.glen;
        for (int i = lane; eq && i < m; i += 32) eq = fa.genome[l1 + i] == strand_byte(rd, m, dr, i);
        if (__all_sync(0xffffffffu, eq)) warp_record(h, lane, k, -(int)g1, 0);
        int seen = 0;
        for (int b0 = 0; need >= 1 && b0 < n1 + n2; b0 += 32) {
          const int item = b0 + lane;
          int hits = 0, flag = 0, start = 0;
          if (item < n1) {
            // item / zones as a multiply-high (an integer division by a
            // variable is a reciprocal estimate and corrections)
            const int zq = (int)__umulhi((uint32_t)item, fa.zone_magic);
            const int b = a + 1 + zq, ez = item - zq * zones - k;
            const uint32_t want = (uint32_t)gs + (uint32_t)b * q + 1 + (uint32_t)ez;
            hits = scan_from_at(L, b, P, off, want);
            if (b == half - 1 && first) {
              flag = 1 + dr;
              start = gs + 1;
            } else if (a == half - 1) {
              flag = ((int)(pa + q) > m ? 3 : 2) + dr;
              start = gs - k + 1;
            } else if (first) {
              flag = 1 + dr;
              start = gs + 1;
            } else {
              flag = 3 + dr;
              start = gs - k + 1;
            }
          } else if (item < n1 + n2) {
            int rest = item - n1, b = 0;
            for (;; ++b) {
              const int w = 2 * abs(half - 1 - b - a) + 1;
              if (rest < w) break;
              rest -= w;
            }
            const int lim = abs(half - 1 - b - a);
            const int err = rest - lim;
            const int ae = (b - a < 0) ? -err : err;
            const uint32_t ns = (uint32_t)(half - b - 1) * q + 1 + S.rest;
            hits = scan_all(L, half + b, (uint32_t)gs + ns + (uint32_t)ae);
            if (b == 0 && first) {
              flag = 1 + dr;
              start = gs + 1;
            } else if (b == 0) {
              flag = ((int)(ns + q) > m ? 3 : 2) + dr;
              start = gs - k + 1;
            } else if (first) {
              flag = 1 + dr;
              start = gs + 1;
            } else {
              flag = 3 + dr;
              start = gs - k + 1;
            }
          }
          int incl = hits;  // inclusive prefix over the lanes
          for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
          }
          const int total = __shfl_sync(0xffffffffu, incl, 31);
          if (seen + total >= need) {
            const unsigned who = __ballot_sync(0xffffffffu, hits > 0 && seen + incl >= need &&
                                                               seen + incl - hits < need);
            const int src = __ffs(who) - 1;
            const int f = __shfl_sync(0xffffffffu, flag, src);
            const int st = __shfl_sync(0xffffffffu, start, src);
            warp_record(h, lane, k, st, f);
            break;
          }
          seen += total;
        }
      }
      ++off;
      pa = L.at(a, off);
    }
  }
  if (lane == 0) {
    fa.n[lr] = h.n;
    fa.queue[lr] = h.queue;
    if (h.overflow) atomicOr(fa.status, 1);
  }
}

// A read's estimated filter work: for each first-half q-gram, its positions
// times the warp steps of its pair items (an upper bound: a position stops
// once its count reaches the threshold).
__global__ void k_work(const long *count, long r0, long cnt, FilterShape S, uint32_t *key,
                       int32_t *idx) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < cnt;
       i += (long)gridDim.x * blockDim.x) {
    const long r = r0 + i;
    unsigned long long w = 0;
    for (int a = 0; a < S.half; ++a) {
      int items = (S.half - 1 - a) * (2 * S.k + 1);
      for (int b = 0; b < S.half; ++b) items += 2 * abs(S.half - 1 - b - a) + 1;
      w += (unsigned long long)(count[r * S.P + a] - 1) * (1 + (items + 31) / 32);
    }
    key[i] = (uint32_t)(w < 0xffffffffull ? w : 0xffffffffull);
    idx[i] = (int32_t)i;
  }
}

__global__ void k_pack(const int32_t *hit_pos, const int8_t *hit_flag, const int32_t *n,
                       const long *at, long nr, int32_t *out_pos, int8_t *out_flag) {
  for (long r = blockIdx.x; r < nr; r += gridDim.x)
    for (int i = threadIdx.x; i < n[r]; i += blockDim.x) {
      out_pos[at[r] + i] = hit_pos[r * kHitsPerRead + i];
      out_flag[at[r] + i] = hit_flag[r * kHitsPerRead + i];
    }
}

__global__ void k_widen(const int32_t *n, long nr, long *out) {
  for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < nr;
       r += (long)gridDim.x * blockDim.x)
    out[r] = n[r];
}

// Device memory that grows, stream-ordered on the filter's stream: a
// growth neither waits for the device's other work (a plain cudaFree
// synchronizes the whole device, so one filter's growth stalled the
// aligner and the other filters of a server) nor for the host.  `slack`
// extra elements are taken on a growth, for buffers sized by the request.
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t count, cudaStream_t s, size_t slack = 0) {
    if (count <= n) return cudaSuccess;
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
    const size_t want = count + slack;
    const cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&p), want * sizeof(T) + 64, s);
    if (e == cudaSuccess) n = want;
    else p = nullptr;
    return e;
  }
  void release(cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
};

// Pinned host memory that grows: copies back from the device into it run
// at full speed and without staging.
template <typename T>
struct HBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t count) {
    if (count <= n) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    const size_t want = std::max(count + count / 2, 2 * n) + 64;
    const cudaError_t e = cudaMallocHost(&p, want * sizeof(T));
    if (e == cudaSuccess) n = want;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
};

}  // namespace

struct saru_filter {
  int device = 0, m = 0, k = 0;
  FilterShape S{};
  long glen = 0, nidx = 0;
  int64_t offset = 0, limit = -1;  // the chunk's genome position; windows end by limit
  uint32_t zone_magic = 0;         // ceil(2^32 / (2k + 1)), checked exact for every item
  cudaStream_t s = nullptr;
  DBuf<uint8_t> genome, reads, temp;
  DBuf<uint64_t> hash, hash_s;
  DBuf<uint32_t> pos, pos_s;
  DBuf<long> lo, count, offs, at, nwide;
  DBuf<int32_t> hit_pos, n, queue, packed_pos, widx;
  DBuf<uint32_t> wkey;
  DBuf<int8_t> hit_flag, packed_flag;
  DBuf<int> status;
  // a launch's counts and kept positions, copied back; two sets, so one
  // launch's calls are assembled on the host while the next one runs
  HBuf<int32_t> h_n[2], h_q[2], h_pos[2];
  HBuf<int8_t> h_flag[2];
  CallAssembler asmb{0, 0, 0, 1};  // the last run's calls (asmb.out), storage kept
  float last_ms = 0.f;
};

namespace {

int fail(const char *what, cudaError_t e) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  saru::set_last_error(msg.c_str());
  return SARU_E_CUDA;
}

}  // namespace

extern "C" {

saru_filter *saru_filter_create(const char *genome, int64_t genome_len, int32_t read_length,
                                int32_t k, int32_t device) {
  saru::set_last_error("");
  if (device < 0 && cudaGetDevice(&device) != cudaSuccess) device = 0;  // the current one
  auto *f = new saru_filter();
  f->device = device;
  f->m = read_length;
  f->k = k;
  f->glen = genome_len;
  if (!genome || genome_len < 1 || read_length < 2 || k < 0 ||
      !filter_shape(read_length, k, &f->S) || f->S.q > 4 * kFilterMaxQgrams) {
    saru::set_last_error("saru_filter_create: a genome, read_length >= 2, k >= 0 and a q-gram "
                         "layout of at most 64 q-grams");
    delete f;
    return nullptr;
  }
  {  // the kernel divides pair items by 2k + 1 with a multiply-high: exact
     // for every item index a read can have (checked here)
    const uint32_t zones = 2u * (uint32_t)k + 1u;
    f->zone_magic = (uint32_t)(((1ull << 32) + zones - 1) / zones);
    const uint32_t items = (uint32_t)(f->S.half * (zones + 2u * (uint32_t)f->S.half + 1u));
    for (uint32_t i = 0; i <= items; ++i)
      if ((uint32_t)(((uint64_t)i * f->zone_magic) >> 32) != i / zones) {
        saru::set_last_error("saru_filter_create: no exact multiply for the item division");
        delete f;
        return nullptr;
      }
  }
  const int q = f->S.q;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->s, cudaStreamNonBlocking);
  f->nidx = genome_len >= q ? genome_len - q + 1 : 0;
  const long n = f->nidx;
  if (e == cudaSuccess) e = f->genome.ensure((size_t)genome_len, f->s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(f->genome.p, genome, (size_t)genome_len, cudaMemcpyHostToDevice, f->s);
  if (e == cudaSuccess && n > 0) {
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t *)nullptr, (uint64_t *)nullptr,
                                    (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, 64,
                                    f->s);
    if ((e = f->hash.ensure(n, f->s)) == cudaSuccess &&
        (e = f->hash_s.ensure(n, f->s)) == cudaSuccess &&
        (e = f->pos.ensure(n, f->s)) == cudaSuccess &&
        (e = f->pos_s.ensure(n, f->s)) == cudaSuccess &&
        (e = f->temp.ensure(tb, f->s)) == cudaSuccess &&
        (e = f->status.ensure(1, f->s)) == cudaSuccess) {
      k_qgram_hash<<<1184, 256, 0, f->s>>>(f->genome.p, n, q, f->hash.p, f->pos.p);
      e = cudaGetLastError();
      if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(f->temp.p, tb, f->hash.p, f->hash_s.p, f->pos.p,
                                            f->pos_s.p, (int)n, 0, 64, f->s);
      if (e == cudaSuccess) e = cudaMemsetAsync(f->status.p, 0, sizeof(int), f->s);
      if (e == cudaSuccess) {
        k_index_check<<<1184, 256, 0, f->s>>>(f->hash_s.p, f->pos_s.p, n, f->genome.p, q,
                                              f->status.p);
        e = cudaGetLastError();
      }
      int flag = 0;
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(&flag, f->status.p, sizeof(int), cudaMemcpyDeviceToHost, f->s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(f->s);
      if (e == cudaSuccess && flag) {
        saru::set_last_error("saru_filter_create: two different q-grams share a 64-bit hash");
        saru_filter_destroy(f);
        return nullptr;
      }
      f->hash.release(f->s);
      f->pos.release(f->s);
    }
  }
  // the genome (saru_filter_genome) is usable on any stream once this returns
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->s);
  if (e != cudaSuccess) {
    fail("saru_filter_create", e);
    saru_filter_destroy(f);
    return nullptr;
  }
  saru::count_launch();
  return f;
}

int saru_filter_run(saru_filter *f, const char *reads, int32_t nreads, int32_t do_reverse,
                    uint32_t chunk_value, int64_t *counts) {
  saru::set_last_error("");
  if (!f || !counts || nreads < 0 || (nreads > 0 && !reads) || chunk_value < 1 ||
      (do_reverse != 0 && do_reverse != 4)) {
    saru::set_last_error("saru_filter_run: reads, chunk_value >= 1, do_reverse 0 or 4");
    return SARU_E_INVALID;
  }
  const long read_chunk = (long)chunk_value;  // the data array's chunk of reads
  cudaSetDevice(f->device);
  const FilterShape &S = f->S;
  const long nr = nreads, P = S.P, m = f->m;
  CallAssembler &asmb = f->asmb;
  asmb.reset(f->m, f->k, f->limit >= 0 ? f->limit : f->glen, chunk_value);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = cudaSuccess;
  int rc = SARU_OK;
  float ms = 0.f;
  if (nr > 0) {
    const long lists = nr * P;
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (long *)nullptr, (long *)nullptr, (int)lists,
                                  f->s);
    size_t tb2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb2, (long *)nullptr, (long *)nullptr,
                                  (int)kReadsPerLaunch, f->s);
    size_t tb3 = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tb3, (uint32_t *)nullptr,
                                              (uint32_t *)nullptr, (int32_t *)nullptr,
                                              (int32_t *)nullptr, (int)kReadsPerLaunch, 0, 32,
                                              f->s);
    const long batch = std::min<long>(nr, kReadsPerLaunch);
    // buffers sized by the request's reads take half again on a growth;
    // those sized by a launch stop growing at kReadsPerLaunch reads
    cudaStream_t s = f->s;
    if ((e = f->reads.ensure((size_t)(nr * m), s, (size_t)(nr * m) / 2)) != cudaSuccess ||
        (e = f->lo.ensure(lists, s, lists / 2)) != cudaSuccess ||
        (e = f->count.ensure(lists, s, lists / 2)) != cudaSuccess ||
        (e = f->offs.ensure(lists, s, lists / 2)) != cudaSuccess ||
        (e = f->temp.ensure(std::max(std::max(tb, tb2), tb3), s)) != cudaSuccess ||
        (e = f->wkey.ensure((size_t)batch * 2, s)) != cudaSuccess ||
        (e = f->widx.ensure((size_t)batch * 2, s)) != cudaSuccess ||
        (e = f->hit_pos.ensure((size_t)batch * kHitsPerRead, s)) != cudaSuccess ||
        (e = f->hit_flag.ensure((size_t)batch * kHitsPerRead, s)) != cudaSuccess ||
        (e = f->n.ensure(batch, s)) != cudaSuccess || (e = f->queue.ensure(batch, s)) != cudaSuccess ||
        (e = f->at.ensure(batch, s)) != cudaSuccess || (e = f->nwide.ensure(batch, s)) != cudaSuccess ||
        (e = f->status.ensure(1, s)) != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail("saru_filter_run", e);
    }
    cudaEventRecord(e0, f->s);
    e = cudaMemcpyAsync(f->reads.p, reads, (size_t)(nr * m), cudaMemcpyHostToDevice, f->s);
    LookupArgs la{f->reads.p, nr, do_reverse, S, f->genome.p, f->hash_s.p, f->pos_s.p,
                  f->nidx, f->lo.p, f->count.p};
    if (e == cudaSuccess) {
      k_lookup<<<(unsigned)std::min<long>((lists + 255) / 256, 65535), 256, 0, f->s>>>(la);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cub::DeviceScan::ExclusiveSum(f->temp.p, tb, f->count.p, f->offs.p, (int)lists, f->s);
    // one scan over all reads: each chunk's lists stay contiguous, and the
    // filter bounds its look past a list by its chunk's end
    if (e == cudaSuccess) e = cudaMemsetAsync(f->status.p, 0, sizeof(int), f->s);
    // the calls of launch i are assembled on the host (one launch at a time,
    // in read order) while launch i + 1 runs on the device
    std::future<void> assembling;
    auto wait_assembly = [&]() {
      if (assembling.valid()) assembling.get();
    };
    for (long r0 = 0, li = 0; r0 < nr && e == cudaSuccess; r0 += batch, ++li) {
      const long r1 = std::min(nr, r0 + batch), cnt = r1 - r0;
      const int set = (int)(li & 1);
      k_work<<<(unsigned)((cnt + 255) / 256), 256, 0, f->s>>>(f->count.p, r0, cnt, S, f->wkey.p,
                                                              f->widx.p);
      e = cudaGetLastError();
      if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairsDescending(f->temp.p, tb3, f->wkey.p,
                                                      f->wkey.p + batch, f->widx.p,
                                                      f->widx.p + batch, (int)cnt, 0, 32, f->s);
      if (e != cudaSuccess) break;
      FilterArgs fa{f->reads.p, r0, r1, read_chunk, nr, do_reverse, S, f->genome.p,
                    f->glen, f->pos_s.p, f->lo.p, f->count.p, f->offs.p, f->hit_pos.p,
                    f->hit_flag.p, f->n.p, f->queue.p, f->status.p, f->widx.p + batch,
                    (uint32_t)f->offset, f->zone_magic};
      k_filter<<<(unsigned)((cnt + 3) / 4), 128, 0, f->s>>>(fa);  // a warp per read
      e = cudaGetLastError();
      if (e != cudaSuccess) break;
      k_widen<<<(unsigned)((cnt + 255) / 256), 256, 0, f->s>>>(f->n.p, cnt, f->nwide.p);
      e = cub::DeviceScan::ExclusiveSum(f->temp.p, tb2, f->nwide.p, f->at.p, (int)cnt, f->s);
      if ((e = f->h_n[set].ensure((size_t)batch)) != cudaSuccess ||
          (e = f->h_q[set].ensure((size_t)batch)) != cudaSuccess)
        break;
      int32_t *hn = f->h_n[set].p, *hq = f->h_q[set].p;
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(hn, f->n.p, 4 * cnt, cudaMemcpyDeviceToHost, f->s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(hq, f->queue.p, 4 * cnt, cudaMemcpyDeviceToHost, f->s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(f->s);
      if (e != cudaSuccess) break;
      long total = 0;
      for (long i = 0; i < cnt; ++i) total += hn[(size_t)i];
      if ((e = f->packed_pos.ensure((size_t)total + 1, s, (size_t)total / 2)) != cudaSuccess ||
          (e = f->packed_flag.ensure((size_t)total + 1, s, (size_t)total / 2)) != cudaSuccess)
        break;
      k_pack<<<(unsigned)std::min<long>(cnt, 65535), 128, 0, f->s>>>(
          f->hit_pos.p, f->hit_flag.p, f->n.p, f->at.p, cnt, f->packed_pos.p, f->packed_flag.p);
      e = cudaGetLastError();
      if (e != cudaSuccess || (e = f->h_pos[set].ensure((size_t)total + 1)) != cudaSuccess ||
          (e = f->h_flag[set].ensure((size_t)total + 1)) != cudaSuccess)
        break;
      int32_t *hpos = f->h_pos[set].p;
      int8_t *hflag = f->h_flag[set].p;
      e = cudaMemcpyAsync(hpos, f->packed_pos.p, 4 * (size_t)total, cudaMemcpyDeviceToHost, f->s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(hflag, f->packed_flag.p, (size_t)total,
                            cudaMemcpyDeviceToHost, f->s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(f->s);
      if (e != cudaSuccess) break;
      wait_assembly();  // the last launch's calls first (and its staging set is free)
      assembling = std::async(std::launch::async, [&asmb, r0, cnt, hpos, hflag, hn, hq]() {
        // the launch's reads at once, counted and copied on the host cores
        // (the same calls as read-by-read assembly: test_filter_assembly.py)
        const int hw = (int)std::thread::hardware_concurrency();
        asmb.add_reads((int32_t)r0, cnt, hpos, hflag, hn, hq, hw > 0 ? hw : 1);
      });
      saru::count_launch();
    }
    wait_assembly();
    int flag = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&flag, f->status.p, sizeof(int), cudaMemcpyDeviceToHost, f->s);
    cudaEventRecord(e1, f->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(f->s);
    if (e != cudaSuccess) rc = fail("saru_filter_run", e);
    else if (flag) {
      saru::set_last_error("saru_filter_run: a read kept more positions than the filter holds");
      rc = SARU_E_OVERFLOW;
    }
    if (rc == SARU_OK) cudaEventElapsedTime(&ms, e0, e1);
  }
  asmb.finish();
  f->last_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  counts[0] = (int64_t)f->asmb.out.call_begin.size() - 1;
  counts[1] = (int64_t)f->asmb.out.ids.size();
  counts[2] = (int64_t)f->asmb.out.perfect_ids.size();
  return rc;
}

int saru_filter_results(const saru_filter *f, int64_t *call_begin, int32_t *ids, int32_t *pos,
                        int8_t *dirs, int32_t *perfect_ids, int32_t *perfect_pos) {
  if (!f) return SARU_E_INVALID;
  const FilterCalls &c = f->asmb.out;
  if (call_begin) memcpy(call_begin, c.call_begin.data(), c.call_begin.size() * 8);
  if (ids) memcpy(ids, c.ids.data(), c.ids.size() * 4);
  if (pos) memcpy(pos, c.pos.data(), c.pos.size() * 4);
  if (dirs) memcpy(dirs, c.dirs.data(), c.dirs.size());
  if (perfect_ids) memcpy(perfect_ids, c.perfect_ids.data(), c.perfect_ids.size() * 4);
  if (perfect_pos) memcpy(perfect_pos, c.perfect_pos.data(), c.perfect_pos.size() * 4);
  return SARU_OK;
}

double saru_filter_last_ms(const saru_filter *f) { return f ? f->last_ms : -1.0; }

const char *saru_filter_genome(const saru_filter *f) {
  return f ? reinterpret_cast<const char *>(f->genome.p) : nullptr;
}

int saru_filter_set_chunk(saru_filter *f, int64_t offset, int64_t limit) {
  saru::set_last_error("");
  if (!f || offset < 0 || limit < offset || offset + f->glen > (int64_t)UINT32_MAX) {
    saru::set_last_error("saru_filter_set_chunk: offset >= 0, limit >= offset, positions in 32 bits");
    return SARU_E_INVALID;
  }
  f->offset = offset;
  f->limit = limit;
  return SARU_OK;
}

void saru_filter_destroy(saru_filter *f) {
  if (!f) return;
  int caller_dev = 0;  // the caller's current device, restored before returning
  const bool had_dev = cudaGetDevice(&caller_dev) == cudaSuccess;
  cudaSetDevice(f->device);
  if (f->s) cudaStreamSynchronize(f->s);
  f->genome.release(f->s);
  f->reads.release(f->s);
  f->temp.release(f->s);
  f->hash.release(f->s);
  f->hash_s.release(f->s);
  f->pos.release(f->s);
  f->pos_s.release(f->s);
  f->lo.release(f->s);
  f->count.release(f->s);
  f->offs.release(f->s);
  f->at.release(f->s);
  f->nwide.release(f->s);
  f->hit_pos.release(f->s);
  f->n.release(f->s);
  f->queue.release(f->s);
  f->packed_pos.release(f->s);
  f->hit_flag.release(f->s);
  f->packed_flag.release(f->s);
  f->status.release(f->s);
  for (int i = 0; i < 2; ++i) {
    f->h_n[i].release();
    f->h_q[i].release();
    f->h_pos[i].release();
    f->h_flag[i].release();
  }
  f->wkey.release(f->s);
  f->widx.release(f->s);
  if (f->s) {
    cudaStreamSynchronize(f->s);  // the stream-ordered frees
    cudaStreamDestroy(f->s);
  }
  delete f;
  if (had_dev) cudaSetDevice(caller_dev);
}

}  // extern "C"
