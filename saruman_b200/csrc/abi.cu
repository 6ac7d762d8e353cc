// abi.cu -- host side of libsaruman_b200.so: the reference's C entry points
// (include/saruman_b200.h part 1) and the batch entry points (part 2).
//
// Flow of one call (reference: src/cuda-functions.cu:586-1049):
//   validate the call layout on the host and pick the kernel path
//   H2D of windows, reads, offsets and flags on the caller's lane stream
//   banded kernel (or the exact full-rectangle kernels) writes scores and
//     the two alignment-slot arrays, zero-filled, in the reference layout
//   D2H of scores and slots; the TSV writer runs on the host
// Each lane (forward / reverse caller) owns a stream and grow-only device
// buffers, so the two reference threads run concurrently without locks on
// the GPU path.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/saruman_b200.h"

#ifndef SARU_STATIC_SCRATCH_BYTES
#define SARU_STATIC_SCRATCH_BYTES (32u << 20)
#endif
#include "band_tile.cuh"
#include "kernels.cuh"
#include "saru_core.cuh"
#include "server_internal.h"
#include "writer.h"

// ---------------------------------------------------------------------------
// Globals of the reference's host program.  The reference defines them in
// its headers (src/saruman.h:55-66, src/util.h:312-343, src/cuda-functions.h
// :31-32); a program linked from those sources supplies its own copies,
// which take precedence over these through ELF symbol interposition.  These
// definitions let the library load on its own (tests, other callers).
// ---------------------------------------------------------------------------
extern "C" {
struct read_name_hash;
struct read_name_hash *read_names = nullptr;
unsigned short int read_length_value = 0;
unsigned short int be_verbose_value = 0;
unsigned short int use_gpu_value = 5000;
unsigned long int cuda_memory_per_thread = 0;
unsigned int forward_alignments_done = 0;
unsigned int reverse_alignments_done = 0;
unsigned int forward_alignment_candidates = 0;
unsigned int reverse_alignment_candidates = 0;
char *forward_output_control = nullptr;
char *reverse_output_control = nullptr;
char *main_alloc_ptr_for = nullptr;
char *main_alloc_ptr_rev = nullptr;
float alignment_time[2] = {0.f, 0.f};
}

namespace {

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
thread_local uint64_t g_thread_launches = 0;  // launches enqueued by this thread
std::mutex g_out_mu;  // stdout lines and the shared counters

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

#define SARU_CUDA(call)                                                            \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return SARU_E_CUDA;                                                          \
    }                                                                              \
  } while (0)

struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  int ensure(size_t bytes) {
    if (bytes <= n) return SARU_OK;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    size_t want = bytes + bytes / 8 + 4096;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of %zu bytes failed", want);
      return SARU_E_NOMEM;
    }
    n = want;
    return SARU_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <typename T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};

struct Lane {
  int device = -1;
  cudaStream_t stream = nullptr;          // copies in (and the unsplit path)
  cudaStream_t s_run = nullptr, s_out = nullptr;  // split calls: kernels, copies out
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_run = nullptr;             // a slice aligned
  std::vector<cudaEvent_t> ev_in;            // a slice's inputs landed (one per slice)
  DevBuf genome, reads, goff, roff, dirs, scores, ra, ga, scratch, status, eoff, arena, records;
  int *status_host = nullptr;  // pinned
  std::mutex mu;

  int init(int dev) {
    if (device == dev && stream) return SARU_OK;
    if (device >= 0) release();  // buffers and streams of another device
    SARU_CUDA(cudaSetDevice(dev));
    SARU_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SARU_CUDA(cudaStreamCreateWithFlags(&s_run, cudaStreamNonBlocking));
    SARU_CUDA(cudaStreamCreateWithFlags(&s_out, cudaStreamNonBlocking));
    SARU_CUDA(cudaEventCreate(&ev0));
    SARU_CUDA(cudaEventCreate(&ev1));
    SARU_CUDA(cudaEventCreateWithFlags(&ev_run, cudaEventDisableTiming));
    SARU_CUDA(cudaMallocHost(&status_host, sizeof(int)));
    device = dev;
    return SARU_OK;
  }
  void release() {
    if (device < 0) return;
    int caller_dev = 0;  // the caller's current device, restored below
    const bool had_dev = cudaGetDevice(&caller_dev) == cudaSuccess;
    cudaSetDevice(device);
    for (DevBuf *b : {&genome, &reads, &goff, &roff, &dirs, &scores, &ra, &ga, &scratch, &status,
                      &eoff, &arena, &records})
      b->release();
    if (status_host) cudaFreeHost(status_host);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : ev_in) cudaEventDestroy(e);
    ev_in.clear();
    if (ev_run) cudaEventDestroy(ev_run);
    if (stream) cudaStreamDestroy(stream);
    if (s_run) cudaStreamDestroy(s_run);
    if (s_out) cudaStreamDestroy(s_out);
    status_host = nullptr;
    ev0 = ev1 = ev_run = nullptr;
    stream = s_run = s_out = nullptr;
    device = -1;
    if (had_dev) cudaSetDevice(caller_dev);
  }
};

Lane g_lanes[3];  // legacy forward, legacy reverse, request server

// The GPU of a host call: the one the reference chose (use_gpu_value, set
// by get_cuda_infos or -u), else the calling thread's current device (one
// process per GPU sets its own).
int current_device() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return -1;
  }
  int d = 0;
  if (use_gpu_value < 5000) d = use_gpu_value;
  else if (cudaGetDevice(&d) != cudaSuccess) d = 0;
  if (d < 0 || d >= count) d = 0;
  return d;
}

int sm_count(int dev) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

// ---------------------------------------------------------------------------
// path selection
// ---------------------------------------------------------------------------

struct Plan {
  bool band = false;   // banded kernel
  bool wide = false;   // 64-bit band
  int max_m = 0;
  int64_t total_cells = 0;  // full-rectangle arena cells
};

// Host-side check of a host batch: the banded kernel needs unit costs, one
// read length m > 3k with m <= kMaxBandM, k <= 15, and windows of exactly
// m + so + eo bytes (the layout src/hash.c:986-1059 builds).
// One range of candidates of plan_host's pass.
struct PlanPart {
  int64_t cells = 0;
  int max_m = 0, m_first = -1, bad = -1;
  bool uniform = true, regular = true, start_gap = false;
};

// (in locals, stored once at the end: the parts of the threads share cache
// lines)
void plan_range(const saru_batch *b, int lo, int hi, PlanPart *out) {
  const int k = b->k;
  const int32_t *go = b->genome_offsets, *ro = b->read_offsets;
  const int8_t *dirs = b->dirs;
  int64_t prev_g = lo ? go[lo - 1] : 0;
  int64_t prev_r = lo ? ro[lo - 1] : 0;
  PlanPart p;
  for (int t = lo; t < hi; ++t) {
    const int64_t L = (int64_t)go[t] - prev_g;
    const int64_t m = (int64_t)ro[t] - prev_r;
    if (L <= 0 || m <= 0 || L > 32000 || m > 32000) {
      p.bad = t;
      break;
    }
    prev_g = go[t];
    prev_r = ro[t];
    if (p.m_first < 0) p.m_first = (int)m;
    p.uniform &= m == p.m_first;
    if (m > p.max_m) p.max_m = (int)m;
    int so, eo;
    saru::flank_of(dirs[t], k, so, eo);
    p.start_gap |= so != 0;
    p.regular &= L == m + so + eo;
    p.cells += (m + 1) * (L + 1);
  }
  *out = p;
}

// plan_range over candidates [lo, hi), split over host threads for long
// ranges; the parts merged in order (bad: the first invalid candidate).
PlanPart plan_span(const saru_batch *b, int lo, int hi) {
  const long n = hi - lo;
  int nt = (int)std::min<long>(16, std::max<long>(1, n / 65536));
  const int hw = (int)std::thread::hardware_concurrency();
  if (hw > 0 && nt > hw) nt = hw;
  std::vector<PlanPart> parts((size_t)nt);
  auto range = [&](int i) {
    plan_range(b, (int)(lo + n * i / nt), (int)(lo + n * (i + 1) / nt), &parts[(size_t)i]);
  };
  if (nt == 1) {
    range(0);
  } else {
    std::vector<std::thread> th;
    for (int i = 1; i < nt; ++i) th.emplace_back(range, i);
    range(0);
    for (auto &x : th) x.join();
  }
  PlanPart all;
  for (const PlanPart &p : parts) {
    if (p.bad >= 0) {
      all.bad = p.bad;
      break;
    }
    all.cells += p.cells;
    if (p.m_first >= 0) {
      if (all.m_first < 0) all.m_first = p.m_first;
      if (p.m_first != all.m_first || !p.uniform) all.uniform = false;
    }
    all.regular = all.regular && p.regular;
    all.start_gap = all.start_gap || p.start_gap;
    all.max_m = std::max(all.max_m, p.max_m);
  }
  return all;
}

int bad_candidate(const saru_batch *b, int t) {
  const int64_t L = (int64_t)b->genome_offsets[t] - (t ? b->genome_offsets[t - 1] : 0);
  const int64_t m = (int64_t)b->read_offsets[t] - (t ? b->read_offsets[t - 1] : 0);
  set_error("invalid batch: candidate %d has window %lld, read %lld", t, (long long)L,
            (long long)m);
  return SARU_E_INVALID;
}

int plan_host(const saru_batch *b, Plan *pl) {
  if (b->n < 0 || b->k < 0) {
    set_error("invalid batch: n=%d k=%d", b->n, b->k);
    return SARU_E_INVALID;
  }
  const int n = b->n, k = b->k;
  const PlanPart all = plan_span(b, 0, n);
  if (all.bad >= 0) return bad_candidate(b, all.bad);
  const int64_t cells = all.cells;
  const bool uniform = all.uniform, regular = all.regular, any_start_gap = all.start_gap;
  const int max_m = all.max_m;
  const int64_t prev_g = n ? b->genome_offsets[n - 1] : 0;
  const int64_t prev_r = n ? b->read_offsets[n - 1] : 0;
  if (n > 0 && (prev_g != b->genome_bytes || prev_g > INT32_MAX || prev_r > INT32_MAX)) {
    set_error("invalid batch: genome_bytes %lld does not match offsets (%lld)",
              (long long)b->genome_bytes, (long long)prev_g);
    return SARU_E_INVALID;
  }
  if (b->total_slots != prev_g + (int64_t)k * n) {
    set_error("invalid batch: total_slots %lld != sum(L + k) = %lld", (long long)b->total_slots,
              (long long)(prev_g + (int64_t)k * n));
    return SARU_E_INVALID;
  }
  pl->max_m = max_m;
  pl->total_cells = cells;
  pl->band = b->match == 0 && b->mismatch == 1 && uniform && regular && k <= 15 &&
             max_m > 3 * k && max_m <= saru::kMaxBandM && max_m >= 2;
  pl->wide = k > 7 && any_start_gap;
  return SARU_OK;
}

int smem_per_sm(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  return v > 0 ? v : 228 * 1024;
}

// persistent grid of the banded kernel: as many CTAs as fit on the GPU
// Launch shapes chosen per (read length, k) by the autotuner (saru_tuning_set);
// classes without an entry keep the default shape.
std::mutex g_tune_mu;
std::map<std::pair<int, int>, saru::Tuning> g_tune;

saru::Tuning tuning_for(int max_m, int k) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find({max_m, k});
  return it == g_tune.end() ? saru::Tuning{} : it->second;
}

long band_grid(int dev, long n, int max_m, int k) {
  const saru::Tuning tn = tuning_for(max_m, k);
  // the band may be 64-bit when k > 7 or when the tuning asks for it
  const bool wide = k > 7 || tn.word_bits == 64;
  return saru::band_grid(sm_count(dev), n, saru::band_layout(max_m, k, tn.warps, wide),
                         smem_per_sm(dev), tn.ctas_per_sm);
}

size_t band_scratch_bytes(long grid, int max_m, int k, bool wide) {
  const saru::Tuning tn = tuning_for(max_m, k);
  return saru::band_scratch_bytes(grid, max_m, k, wide || tn.word_bits == 64, tn.warps);
}

// Enqueues the banded kernel on device buffers: calls[0..ncalls) as the
// segments of one launch (the single-call entry points pass one).  Scratch:
// the tile counter, then the decision planes of the persistent grid.
using saru::CompactOut;

// t0 > 0 (a multiple of 32, one call): align candidates t0 .. n - 1 only.
int run_band_multi(const saru_batch *calls, const saru_result *res, int ncalls, const Plan &pl,
                   void *scratch, size_t scratch_bytes, int *status_dev, int dev,
                   cudaStream_t s, long max_grid = 0, const CompactOut *cmp = nullptr,
                   long t0 = 0) {
  if (ncalls < 1 || ncalls > saru::kMaxSegs) {
    set_error("%d calls in one launch (1..%d)", ncalls, saru::kMaxSegs);
    return SARU_E_INVALID;
  }
  if (t0 < 0 || (t0 & 31) || (t0 > 0 && ncalls != 1)) {
    set_error("a slice of a call starts at a multiple of 32 (%ld)", t0);
    return SARU_E_INVALID;
  }
  // heavier segments first: the counter hands out tiles in segment order, so
  // the tail of the launch is made of the cheapest tiles
  std::vector<int> order((size_t)ncalls);
  for (int i = 0; i < ncalls; ++i) order[(size_t)i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return (long)calls[x].max_read_length * (calls[x].k + 1) >
           (long)calls[y].max_read_length * (calls[y].k + 1);
  });
  static thread_local saru::KernelArgs a;  // ~19 KB: not on the stack
  memset(&a, 0, sizeof(a));
  long tiles = 0, total_n = 0;
  int max_m = 0, max_k = 0, wide_any = 0;
  for (int q = 0; q < ncalls; ++q) {
    max_m = std::max(max_m, calls[q].max_read_length);
    max_k = std::max(max_k, calls[q].k);
  }
  const saru::Tuning tn = tuning_for(max_m, max_k);
  for (int q = 0; q < ncalls; ++q) {
    const saru_batch *b = &calls[order[(size_t)q]];
    const saru_result *r = &res[order[(size_t)q]];
    saru::Segment &g = a.segs[a.nseg++];
    g.genome = reinterpret_cast<const uint8_t *>(b->genome);
    g.reads = reinterpret_cast<const uint8_t *>(b->reads);
    g.goff = b->genome_offsets;
    g.roff = b->read_offsets;
    g.dirs = b->dirs;
    g.scores = r->scores;
    g.read_aln = reinterpret_cast<uint8_t *>(r->read_aln);
    g.genome_aln = reinterpret_cast<uint8_t *>(r->genome_aln);
    g.status = r->status ? r->status : status_dev;
    if (cmp) {
      g.records = cmp[order[(size_t)q]].records;
      g.rec_bytes = cmp[order[(size_t)q]].rec_bytes;
    }
    g.n = b->n;
    g.t0 = t0 < b->n ? t0 : b->n;
    g.tile_begin = tiles;
    g.k = b->k;
    g.max_m = b->max_read_length;
    g.first_of_call = b->first_of_call;
    g.wide = (b->k > 7 && (ncalls > 1 || pl.wide)) || tn.word_bits == 64;
    tiles += (b->n - g.t0 + 31) / 32;
    total_n += b->n - g.t0;
    wide_any |= g.wide;
  }
  if (tiles == 0) return SARU_OK;
  a.total_tiles = tiles;
  a.max_m = max_m;
  a.max_k = max_k;
  a.wide_any = wide_any;
  a.warps_req = tn.warps;
  a.grid = saru::band_grid(sm_count(dev), total_n,
                           saru::band_layout(max_m, max_k, tn.warps, wide_any != 0),
                           smem_per_sm(dev), tn.ctas_per_sm);
  if (max_grid > 0 && a.grid > max_grid) a.grid = max_grid;
  const size_t need = saru::band_scratch_bytes(a.grid, max_m, max_k, wide_any != 0, tn.warps);
  if (need > scratch_bytes) {
    set_error("scratch too small: %zu < %zu", scratch_bytes, need);
    return SARU_E_INVALID;
  }
  if (reinterpret_cast<uintptr_t>(scratch) & 15u) {  // the kernel copies 16-byte plane pairs
    set_error("scratch must be 16-byte aligned");
    return SARU_E_INVALID;
  }
  a.counter = reinterpret_cast<int *>(scratch);
  a.planes = reinterpret_cast<uint8_t *>(scratch) + saru::kCounterBytes;
  SARU_CUDA(saru::launch_band_kernel(a, s));
  g_launches.fetch_add(1);
  g_thread_launches += 1;
  return SARU_OK;
}

// Calls of a multi-call request are grouped into layout classes (read-length
// bucket x band width): one launch sizes its shared-memory slice for its
// longest read, so mixing 36 bp and 150 bp calls in one launch would run the
// short ones at the long ones' occupancy.  Each class gets its own persistent
// launch; the launches run concurrently on forked streams.
struct LaunchClass {
  std::vector<int> calls;
  int max_m = 0, max_k = 0;
  bool wide = false;
  long n = 0, grid = 0;
  size_t scratch_off = 0, scratch_bytes = 0;
};

int length_bucket(int m) {
  // about 25% apart: a class's slice is at most ~25% larger than a member needs
  static const int edges[] = {40, 48, 64, 80, 96, 112, 128, 160, 192, 240, 288, 352, 416, 512};
  for (int e : edges)
    if (m <= e) return e;
  return m;
}

std::vector<LaunchClass> plan_classes(const saru_batch *calls, int ncalls, int dev) {
  std::vector<LaunchClass> cls;
  std::vector<std::pair<int, int>> keys;
  for (int i = 0; i < ncalls; ++i) {
    const std::pair<int, int> key(length_bucket(calls[i].max_read_length), calls[i].k > 7);
    size_t c = 0;
    while (c < keys.size() && keys[c] != key) ++c;
    if (c == keys.size()) {
      keys.push_back(key);
      cls.emplace_back();
    }
    LaunchClass &L = cls[c];
    L.calls.push_back(i);
    L.max_m = std::max(L.max_m, calls[i].max_read_length);
    L.max_k = std::max(L.max_k, calls[i].k);
    L.wide = L.wide || calls[i].k > 7;
    L.n += calls[i].n;
  }
  size_t off = 0;
  for (auto &L : cls) {
    L.grid = band_grid(dev, L.n, L.max_m, L.max_k);
    L.scratch_bytes = band_scratch_bytes(L.grid, L.max_m, L.max_k, L.wide);
    L.scratch_off = off;
    off += (L.scratch_bytes + 255) & ~size_t(255);
  }
  return cls;
}

size_t classes_scratch_bytes(const std::vector<LaunchClass> &cls) {
  size_t t = 0;
  for (const auto &L : cls) t += (L.scratch_bytes + 255) & ~size_t(255);
  return t;
}

// Streams and events for the concurrent class launches of one device.
struct ClassStreams {
  std::mutex mu;
  int dev = -1;
  cudaEvent_t fork = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  int ensure(int d, size_t n) {
    if (dev != d) {
      if (dev >= 0) return SARU_E_INVALID;
      dev = d;
      SARU_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    }
    while (streams.size() < n) {
      cudaStream_t st;
      cudaEvent_t ev;
      SARU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      SARU_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      streams.push_back(st);
      joins.push_back(ev);
    }
    return SARU_OK;
  }
};
ClassStreams g_class_streams[64];

int run_band_classes(const saru_batch *calls, const saru_result *res, int ncalls, void *scratch,
                     size_t scratch_bytes, int *status_dev, int dev, cudaStream_t s,
                     const CompactOut *cmp = nullptr) {
  const std::vector<LaunchClass> cls = plan_classes(calls, ncalls, dev);
  if (classes_scratch_bytes(cls) > scratch_bytes) {
    set_error("scratch too small: %zu < %zu", scratch_bytes, classes_scratch_bytes(cls));
    return SARU_E_INVALID;
  }
  auto launch = [&](const LaunchClass &L, cudaStream_t st) {
    Plan pl;  // a class of k > 7 calls runs 64-bit band words, even with one call
    pl.band = true;
    pl.wide = L.wide;
    std::vector<saru_batch> cb;
    std::vector<saru_result> cr;
    std::vector<CompactOut> cc;
    for (int i : L.calls) {
      cb.push_back(calls[i]);
      cr.push_back(res[i]);
      if (cmp) cc.push_back(cmp[i]);
    }
    return run_band_multi(cb.data(), cr.data(), (int)cb.size(), pl,
                          static_cast<uint8_t *>(scratch) + L.scratch_off, L.scratch_bytes,
                          status_dev, dev, st, 0, cmp ? cc.data() : nullptr);
  };
  if (cls.size() == 1) return launch(cls[0], s);
  if (dev < 0 || dev >= 64) return SARU_E_INVALID;
  ClassStreams &CS = g_class_streams[dev];
  std::lock_guard<std::mutex> lk(CS.mu);
  int rc = CS.ensure(dev, cls.size());
  if (rc) return rc;
  SARU_CUDA(cudaEventRecord(CS.fork, s));
  for (size_t c = 0; c < cls.size(); ++c) {
    SARU_CUDA(cudaStreamWaitEvent(CS.streams[c], CS.fork, 0));
    if ((rc = launch(cls[c], CS.streams[c]))) return rc;
    SARU_CUDA(cudaEventRecord(CS.joins[c], CS.streams[c]));
    SARU_CUDA(cudaStreamWaitEvent(s, CS.joins[c], 0));
  }
  return SARU_OK;
}

int run_band(const saru_batch *b, const Plan &pl, const saru_result *r, void *scratch,
             size_t scratch_bytes, int *status_dev, int dev, cudaStream_t s,
             long max_grid = 0, const CompactOut *cmp = nullptr, long t0 = 0) {
  if (b->n == 0) return SARU_OK;
  saru_batch one = *b;
  one.max_read_length = pl.max_m;
  return run_band_multi(&one, r, 1, pl, scratch, scratch_bytes, status_dev, dev, s, max_grid,
                        cmp, t0);
}

// Host batch -> device buffers of `lane`, returns device-side view (with
// copy false: the buffers only, the caller copies).
int upload(Lane &L, const saru_batch *b, saru_batch *db, bool copy = true) {
  const size_t n = (size_t)b->n;
  int rc;
  if ((rc = L.genome.ensure((size_t)b->genome_bytes + 64))) return rc;
  if ((rc = L.reads.ensure((size_t)(n ? b->read_offsets[n - 1] : 0) + 64))) return rc;
  if ((rc = L.goff.ensure(4 * n + 64))) return rc;
  if ((rc = L.roff.ensure(4 * n + 64))) return rc;
  if ((rc = L.dirs.ensure(n + 64))) return rc;
  cudaStream_t s = L.stream;
  if (n && copy) {
    SARU_CUDA(cudaMemcpyAsync(L.genome.p, b->genome, (size_t)b->genome_bytes, cudaMemcpyHostToDevice, s));
    SARU_CUDA(cudaMemcpyAsync(L.reads.p, b->reads, (size_t)b->read_offsets[n - 1], cudaMemcpyHostToDevice, s));
    SARU_CUDA(cudaMemcpyAsync(L.goff.p, b->genome_offsets, 4 * n, cudaMemcpyHostToDevice, s));
    SARU_CUDA(cudaMemcpyAsync(L.roff.p, b->read_offsets, 4 * n, cudaMemcpyHostToDevice, s));
    SARU_CUDA(cudaMemcpyAsync(L.dirs.p, b->dirs, n, cudaMemcpyHostToDevice, s));
  }
  *db = *b;
  db->genome = L.genome.as<const char>();
  db->reads = L.reads.as<const char>();
  db->genome_offsets = L.goff.as<const int32_t>();
  db->read_offsets = L.roff.as<const int32_t>();
  db->dirs = L.dirs.as<const int8_t>();
  return SARU_OK;
}

// The exact full-rectangle path on lane buffers (whole call).
int run_full(Lane &L, const saru_batch *hb, const saru_batch *db, const Plan &pl,
             const saru_result *dr) {
  const size_t n = (size_t)hb->n;
  int rc;
  std::vector<int64_t> eoff(n);
  int64_t acc = 0;
  for (size_t t = 0; t < n; ++t) {
    eoff[t] = acc;
    const int64_t L_ = (int64_t)hb->genome_offsets[t] - (t ? hb->genome_offsets[t - 1] : 0);
    const int64_t m_ = (int64_t)hb->read_offsets[t] - (t ? hb->read_offsets[t - 1] : 0);
    acc += (m_ + 1) * (L_ + 1);
  }
  if (acc > INT32_MAX) {
    set_error("call too large for the reference's int cell index (%lld cells)", (long long)acc);
    return SARU_E_INVALID;
  }
  if ((rc = L.eoff.ensure(8 * n + 64))) return rc;
  if ((rc = L.arena.ensure(2 * (size_t)acc + 64))) return rc;
  cudaStream_t s = L.stream;
  SARU_CUDA(cudaMemcpyAsync(L.eoff.p, eoff.data(), 8 * n, cudaMemcpyHostToDevice, s));
  SARU_CUDA(cudaMemsetAsync(dr->read_aln, 0, (size_t)hb->total_slots, s));
  SARU_CUDA(cudaMemsetAsync(dr->genome_aln, 0, (size_t)hb->total_slots, s));
  saru::FullArgs a{};
  a.genome = reinterpret_cast<const uint8_t *>(db->genome);
  a.reads = reinterpret_cast<const uint8_t *>(db->reads);
  a.goff = db->genome_offsets;
  a.roff = db->read_offsets;
  a.dirs = db->dirs;
  a.eoff = L.eoff.as<const int64_t>();
  a.n = hb->n;
  a.k = hb->k;
  a.match = hb->match;
  a.mismatch = hb->mismatch;
  a.first_of_call = hb->first_of_call;
  a.genome_bytes = hb->genome_bytes;
  a.read_bytes = n ? hb->read_offsets[n - 1] : 0;
  a.arena = L.arena.as<short>();
  a.scores = dr->scores;
  a.read_aln = reinterpret_cast<uint8_t *>(dr->read_aln);
  a.genome_aln = reinterpret_cast<uint8_t *>(dr->genome_aln);
  a.status = L.status.as<int>();
  (void)pl;
  SARU_CUDA(saru::launch_full_kernels(a, s));
  g_launches.fetch_add(2);
  g_thread_launches += 2;
  return SARU_OK;
}

// A call of at least 2 * kSplitMin candidates from host memory is split
// into slices of whole tiles.  The copies in of every slice are issued
// first (one event each), and the host's pass over the call (plan_host)
// runs while they stream; then, for a banded call, the kernel of slice i
// waits for its inputs and the copies out of slice i wait for its kernel,
// so copies in, kernels and copies out overlap on three streams (the
// reference copies everything in, aligns, copies everything out).  Each
// slice is a launch over candidates [t0, t1) of the whole call on the
// device, so its tiles, and every output byte, are the ones the unsplit
// launch makes; only candidate 0 of the call takes the first-of-call rule.
// With pinned host buffers the copies run asynchronously; with pageable
// ones they are correct but serialised.
constexpr long kSplitMin = 1L << 18;
constexpr long kSplitParts = 32;

long split_chunk(long n) {
  const long c = ((n + kSplitParts - 1) / kSplitParts + 31) & ~31L;
  return c < kSplitMin ? kSplitMin : c;
}

// The slice edges of a large call, checked before its copies are issued:
// each copy reads the caller's arrays between two edges, so the offsets
// there must not decrease and must end at the sizes the call states.
int check_slice_edges(const saru_batch *b, long chunk) {
  const long n = b->n;
  int64_t pg = 0, pr = 0;
  for (long t1 = std::min(n, chunk);; t1 = std::min(n, t1 + chunk)) {
    const int64_t g = b->genome_offsets[t1 - 1], r = b->read_offsets[t1 - 1];
    if (g < pg || r < pr) {
      set_error("invalid batch: offsets decrease before candidate %ld", t1 - 1);
      return SARU_E_INVALID;
    }
    pg = g;
    pr = r;
    if (t1 == n) break;
  }
  if (pg != b->genome_bytes || pg > INT32_MAX || pr > INT32_MAX) {
    set_error("invalid batch: genome_bytes %lld does not match offsets (%lld)",
              (long long)b->genome_bytes, (long long)pg);
    return SARU_E_INVALID;
  }
  if (b->total_slots != pg + (int64_t)b->k * n) {
    set_error("invalid batch: total_slots %lld != sum(L + k) = %lld", (long long)b->total_slots,
              (long long)(pg + (int64_t)b->k * n));
    return SARU_E_INVALID;
  }
  return SARU_OK;
}

// Copies in, slice by slice, on the lane's first stream.
int upload_slices(Lane &L, const saru_batch *b, long chunk) {
  const long n = b->n;
  const size_t nslices = (size_t)((n + chunk - 1) / chunk);
  while (L.ev_in.size() < nslices) {
    cudaEvent_t e;
    SARU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    L.ev_in.push_back(e);
  }
  cudaStream_t si = L.stream;
  const int32_t *go = b->genome_offsets, *ro = b->read_offsets;
  for (long t0 = 0, i = 0; t0 < n; t0 += chunk, ++i) {
    const long t1 = std::min(n, t0 + chunk);
    const long g0 = t0 ? go[t0 - 1] : 0, g1 = go[t1 - 1];
    const long r0 = t0 ? ro[t0 - 1] : 0, r1 = ro[t1 - 1];
    SARU_CUDA(cudaMemcpyAsync(L.genome.as<char>() + g0, b->genome + g0, (size_t)(g1 - g0),
                              cudaMemcpyHostToDevice, si));
    SARU_CUDA(cudaMemcpyAsync(L.reads.as<char>() + r0, b->reads + r0, (size_t)(r1 - r0),
                              cudaMemcpyHostToDevice, si));
    SARU_CUDA(cudaMemcpyAsync(L.goff.as<int32_t>() + t0, go + t0, 4 * (size_t)(t1 - t0),
                              cudaMemcpyHostToDevice, si));
    SARU_CUDA(cudaMemcpyAsync(L.roff.as<int32_t>() + t0, ro + t0, 4 * (size_t)(t1 - t0),
                              cudaMemcpyHostToDevice, si));
    SARU_CUDA(cudaMemcpyAsync(L.dirs.as<int8_t>() + t0, b->dirs + t0, (size_t)(t1 - t0),
                              cudaMemcpyHostToDevice, si));
    SARU_CUDA(cudaEventRecord(L.ev_in[(size_t)i], si));
  }
  return SARU_OK;
}

// Kernels and copies out of the slices (after upload_slices), each slice
// checked on the host (plan_range, threaded) just before its launch, so the
// first kernels and copies out start while later slices are checked.  The
// banded path was chosen from facts known up front (unit costs, k <= 15, the
// first read's length); a slice whose reads differ in length or whose
// windows are not m + so + eo sets *exact and launches stop (the call then
// takes the exact path whole); an invalid candidate anywhere is an error.
// Host outputs of a call in compact records (saru_align_host_compact).
struct HostCompact {
  int32_t *scores;
  uint8_t *records;
  long rec_bytes;
};

int band_slices(Lane &L, const saru_batch *b, int m0, const saru_batch &db,
                const saru_result &dr, const saru_result *r, int dev, long chunk, bool *exact,
                const HostCompact *hc) {
  const long n = b->n, k = b->k;
  int rc;
  Plan pl;
  pl.band = true;
  pl.max_m = m0;
  const long grid = band_grid(dev, chunk, m0, b->k);
  if ((rc = L.scratch.ensure(band_scratch_bytes(grid, m0, b->k, k > 7)))) return rc;
  cudaStream_t sr = L.s_run, so = L.s_out;
  const int32_t *go = b->genome_offsets;
  const CompactOut dcmp{L.records.as<uint8_t>(), hc ? hc->rec_bytes : 0};
  *exact = false;
  int bad = -1;
  for (long t0 = 0, i = 0; t0 < n; t0 += chunk, ++i) {
    const long t1 = std::min(n, t0 + chunk);
    const PlanPart part = plan_span(b, (int)t0, (int)t1);
    if (part.bad >= 0) {
      bad = part.bad;
      break;
    }
    if (!part.uniform || part.m_first != m0 || !part.regular) *exact = true;
    if (*exact) continue;  // check the rest, launch no more
    pl.wide = k > 7 && part.start_gap;
    const long g0 = t0 ? go[t0 - 1] : 0, g1 = go[t1 - 1];
    SARU_CUDA(cudaStreamWaitEvent(sr, L.ev_in[(size_t)i], 0));
    saru_batch slice = db;
    slice.n = (int32_t)t1;
    if ((rc = run_band(&slice, pl, &dr, L.scratch.p, L.scratch.n, L.status.as<int>(), dev, sr, 0,
                       hc ? &dcmp : nullptr, t0)))
      return rc;
    SARU_CUDA(cudaEventRecord(L.ev_run, sr));
    SARU_CUDA(cudaStreamWaitEvent(so, L.ev_run, 0));
    if (hc) {
      SARU_CUDA(cudaMemcpyAsync(hc->scores + t0, dr.scores + t0, 4 * (size_t)(t1 - t0),
                                cudaMemcpyDeviceToHost, so));
      SARU_CUDA(cudaMemcpyAsync(hc->records + t0 * hc->rec_bytes,
                                L.records.as<uint8_t>() + t0 * hc->rec_bytes,
                                (size_t)((t1 - t0) * hc->rec_bytes), cudaMemcpyDeviceToHost, so));
      continue;
    }
    const long s0 = g0 + k * t0, s1 = g1 + k * t1;
    SARU_CUDA(cudaMemcpyAsync(r->scores + t0, dr.scores + t0, 4 * (size_t)(t1 - t0),
                              cudaMemcpyDeviceToHost, so));
    SARU_CUDA(cudaMemcpyAsync(r->read_aln + s0, dr.read_aln + s0, (size_t)(s1 - s0),
                              cudaMemcpyDeviceToHost, so));
    SARU_CUDA(cudaMemcpyAsync(r->genome_aln + s0, dr.genome_aln + s0, (size_t)(s1 - s0),
                              cudaMemcpyDeviceToHost, so));
  }
  SARU_CUDA(cudaMemcpyAsync(L.status_host, L.status.p, sizeof(int), cudaMemcpyDeviceToHost, so));
  SARU_CUDA(cudaEventRecord(L.ev1, so));
  // every stream of the lane is idle before returning (the copies read and
  // write the caller's buffers)
  SARU_CUDA(cudaStreamSynchronize(L.stream));
  SARU_CUDA(cudaStreamSynchronize(sr));
  SARU_CUDA(cudaStreamSynchronize(so));
  if (bad >= 0) return bad_candidate(b, bad);
  return SARU_OK;
}

// A host call: slot strings into r, or (hc) compact records.
int align_host_impl(const saru_batch *b, saru_result *r, Lane &L, float *ms_out,
                    const HostCompact *hc = nullptr) {
  Plan pl;
  int rc;
  const bool big = b->n >= 2 * kSplitMin && b->k >= 0;
  const long chunk = big ? split_chunk(b->n) : 0;
  if (!big && (rc = plan_host(b, &pl))) return rc;
  if (big && (rc = check_slice_edges(b, chunk))) return rc;
  const int dev = current_device();
  if (dev < 0) {
    set_error("no CUDA device");
    return SARU_E_CUDA;
  }
  if ((rc = L.init(dev))) return rc;
  SARU_CUDA(cudaSetDevice(dev));
  if (b->n == 0) return SARU_OK;
  cudaStream_t s = L.stream;
  SARU_CUDA(cudaEventRecord(L.ev0, s));
  const size_t n = (size_t)b->n;
  saru_batch db;
  if ((rc = upload(L, b, &db, !big))) return rc;
  if ((rc = L.scores.ensure(4 * n + 64))) return rc;
  if ((rc = L.ra.ensure((size_t)b->total_slots + 64))) return rc;
  if ((rc = L.ga.ensure((size_t)b->total_slots + 64))) return rc;
  if ((rc = L.status.ensure(64))) return rc;
  if (hc && (rc = L.records.ensure(n * (size_t)hc->rec_bytes + 64))) return rc;
  saru_result dr{L.scores.as<int32_t>(), L.ra.as<char>(), L.ga.as<char>(), L.status.as<int32_t>()};
  const CompactOut dcmp{L.records.as<uint8_t>(), hc ? hc->rec_bytes : 0};
  SARU_CUDA(cudaMemsetAsync(L.status.p, 0, sizeof(int), s));
  bool split = false;
  if (big) {  // copies in first; the host's checks run while they stream
    if ((rc = upload_slices(L, b, chunk))) return rc;
    const int m0 = b->read_offsets[0];
    split = b->match == 0 && b->mismatch == 1 && b->k <= 15 && m0 > 3 * b->k &&
            m0 <= saru::kMaxBandM && m0 >= 2;
    if (split && hc && hc->rec_bytes < saru::compact_record_bytes(m0, b->k)) {
      cudaStreamSynchronize(s);
      set_error("record_bytes %ld < saru_compact_record_bytes(%d, %d)", hc->rec_bytes, m0, b->k);
      return SARU_E_INVALID;
    }
    bool exact = false;
    if (split && (rc = band_slices(L, b, m0, db, dr, r, dev, chunk, &exact, hc))) return rc;
    if (!split || exact) {
      split = false;
      if ((rc = plan_host(b, &pl))) {
        cudaStreamSynchronize(s);
        return rc;
      }
      pl.band = false;  // the exact path, whole
    }
  }
  bool full = !pl.band && !split, copied = false;
  if (split) {
    const int st = *L.status_host;
    if (st & (saru::kStatusAlphabet | saru::kStatusIrregular)) {
      full = true;  // rare bytes or layouts: redo the call on the exact path
      SARU_CUDA(cudaMemsetAsync(L.status.p, 0, sizeof(int), s));
    } else if (st & saru::kStatusOverflow) {
      set_error("banded traceback left its band (status %d)", st);
      return SARU_E_OVERFLOW;
    } else {
      copied = true;
    }
  } else if (pl.band) {
    if (hc && hc->rec_bytes < saru::compact_record_bytes(pl.max_m, b->k)) {
      set_error("record_bytes %ld < saru_compact_record_bytes(%d, %d)", hc->rec_bytes, pl.max_m,
                b->k);
      return SARU_E_INVALID;
    }
    const long grid = band_grid(dev, b->n, pl.max_m, b->k);
    if ((rc = L.scratch.ensure(band_scratch_bytes(grid, pl.max_m, b->k, pl.wide)))) return rc;
    if ((rc = run_band(&db, pl, &dr, L.scratch.p, L.scratch.n, L.status.as<int>(), dev, s, 0,
                       hc ? &dcmp : nullptr)))
      return rc;
    SARU_CUDA(cudaMemcpyAsync(L.status_host, L.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaStreamSynchronize(s));
    const int st = *L.status_host;
    if (st & (saru::kStatusAlphabet | saru::kStatusIrregular)) {
      full = true;  // rare bytes or layouts: redo the call on the exact path
      SARU_CUDA(cudaMemsetAsync(L.status.p, 0, sizeof(int), s));
    } else if (st & saru::kStatusOverflow) {
      set_error("banded traceback left its band (status %d)", st);
      return SARU_E_OVERFLOW;
    }
  }
  if (full) {
    if ((rc = run_full(L, b, &db, pl, &dr))) return rc;
    SARU_CUDA(cudaMemcpyAsync(L.status_host, L.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  if (!copied && hc && !full) {  // banded, unsplit: the records
    SARU_CUDA(cudaMemcpyAsync(hc->scores, dr.scores, 4 * n, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaMemcpyAsync(hc->records, L.records.p, n * (size_t)hc->rec_bytes,
                              cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaEventRecord(L.ev1, s));
    SARU_CUDA(cudaStreamSynchronize(s));
  } else if (!copied && hc) {  // the exact path's slots, turned into records on the host
    std::vector<char> ra((size_t)b->total_slots + 64), ga((size_t)b->total_slots + 64);
    SARU_CUDA(cudaMemcpyAsync(hc->scores, dr.scores, 4 * n, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaMemcpyAsync(ra.data(), dr.read_aln, (size_t)b->total_slots, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaMemcpyAsync(ga.data(), dr.genome_aln, (size_t)b->total_slots, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaEventRecord(L.ev1, s));
    SARU_CUDA(cudaStreamSynchronize(s));
    if ((rc = saru::records_from_slots(b, hc->scores, ra.data(), ga.data(), hc->records,
                                       hc->rec_bytes)))
      return rc;
  } else if (!copied) {
    SARU_CUDA(cudaMemcpyAsync(r->scores, dr.scores, 4 * n, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaMemcpyAsync(r->read_aln, dr.read_aln, (size_t)b->total_slots, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaMemcpyAsync(r->genome_aln, dr.genome_aln, (size_t)b->total_slots, cudaMemcpyDeviceToHost, s));
    SARU_CUDA(cudaEventRecord(L.ev1, s));
    SARU_CUDA(cudaStreamSynchronize(s));
  }
  if (full && (*L.status_host & saru::kStatusOverflow)) {
    set_error("a traceback left its slot; the reference result depends on thread order");
    return SARU_E_OVERFLOW;
  }
  if (ms_out) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, L.ev0, L.ev1);
    *ms_out = ms;
  }
  return SARU_OK;
}

// uthash application-order walk of the caller's read_names table.  Element
// layout of struct read_name_hash (src/util.h:350-354): int read_number;
// char name[60]; UT_hash_handle hh; the handle's third pointer `next`
// (src/uthash.h, UT_hash_handle) links the elements in insertion order.
struct NameIndex {
  std::vector<const char *> by_id;  // element of each read id (nullptr: none)
  const void *head = nullptr;
  static const char *lookup(void *ctx, int32_t id) {
    auto *ni = static_cast<NameIndex *>(ctx);
    if (id < 0 || (size_t)id >= ni->by_id.size() || !ni->by_id[(size_t)id]) return nullptr;
    return ni->by_id[(size_t)id] + sizeof(int);
  }
  void build(const void *h) {
    by_id.clear();
    head = h;
    const char *e = static_cast<const char *>(h);
    size_t guard = 0;
    while (e && guard++ < (size_t)1 << 31) {
      const int id = *reinterpret_cast<const int *>(e);
      if (id >= 0) {
        if ((size_t)id >= by_id.size()) by_id.resize((size_t)id + 1, nullptr);
        by_id[(size_t)id] = e;
      }
      const void *next = *reinterpret_cast<void *const *>(e + 64 + 2 * sizeof(void *));
      e = static_cast<const char *>(next);
    }
  }
  // true if every read id of ids[0..n) whose candidate prints (score <= k)
  // has an element that still holds that id
  bool covers(const void *h, const int32_t *ids, const int32_t *scores, int n, int k) const {
    if (h != head) return false;
    for (int v = 0; v < n; ++v) {
      if (scores[v] > k) continue;
      const int32_t id = ids[v];
      if (id < 0 || (size_t)id >= by_id.size() || !by_id[(size_t)id] ||
          *reinterpret_cast<const int *>(by_id[(size_t)id]) != id)
        return false;
    }
    return true;
  }
};

// The caller's read_names table, walked once and kept while it still holds
// the ids a call prints (the reference builds one table per read batch and
// makes many calls against it; walking a list of millions of reads per call
// would cost more than the call).
// Shared while a call's lines are formatted (the two strands' calls format
// at once), exclusive while the index is rebuilt.
std::shared_mutex g_names_mu;
NameIndex g_names;

// Grow-only pinned host buffer.
struct PinnedBuf {
  void *p = nullptr;
  size_t n = 0;
  int ensure(size_t bytes) {
    if (bytes <= n) return SARU_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    const size_t want = bytes + bytes / 8 + 4096;
    if (cudaMallocHost(&p, want) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMallocHost of %zu bytes failed", want);
      return SARU_E_NOMEM;
    }
    n = want;
    return SARU_OK;
  }
  template <typename T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};
PinnedBuf g_legacy_out[2][3];  // per legacy lane: scores, read strings, window strings

}  // namespace

// hooks for the request server (server.cpp)
namespace saru {
uint64_t thread_launches() { return g_thread_launches; }
void count_launch() {
  g_launches.fetch_add(1);
  g_thread_launches += 1;
}
void set_last_error(const char *msg) { g_last_error = msg; }
int redo_on_host_path(const saru_batch *b, saru_result *r) {
  Lane &L = g_lanes[2];
  std::lock_guard<std::mutex> lk(L.mu);
  return align_host_impl(b, r, L, nullptr);
}
int align_multi_mixed(const saru_batch *calls, const saru_result *results,
                      const CompactOut *cmp, int32_t ncalls, int32_t *status, void *scratch,
                      size_t scratch_bytes, void *stream) {
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  return run_band_classes(calls, results, ncalls, scratch, scratch_bytes, status, dev,
                          reinterpret_cast<cudaStream_t>(stream), cmp);
}
}  // namespace saru

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char *saru_last_error(void) { return g_last_error.c_str(); }

uint64_t saru_kernel_launches(void) { return g_launches.load(); }

int saru_tuning_set(int32_t read_length, int32_t k, const saru_tuning *t) {
  g_last_error.clear();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (!t) {
    g_tune.erase({read_length, k});
    return SARU_OK;
  }
  if (t->warps_per_cta < 0 || t->warps_per_cta > 4 || t->ctas_per_sm < 0 ||
      t->ctas_per_sm > 16 || (t->word_bits != 0 && t->word_bits != 32 && t->word_bits != 64) ||
      (t->word_bits == 32 && k > 7)) {
    set_error("saru_tuning_set: warps_per_cta 0..4, ctas_per_sm 0..16, word_bits 0/32/64 "
              "(32 only for k <= 7)");
    return SARU_E_INVALID;
  }
  saru::Tuning tn;
  tn.warps = t->warps_per_cta;
  tn.ctas_per_sm = t->ctas_per_sm;
  tn.word_bits = t->word_bits;
  g_tune[{read_length, k}] = tn;
  return SARU_OK;
}

int saru_tuning_get(int32_t read_length, int32_t k, saru_tuning *t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find({read_length, k});
  if (it == g_tune.end()) {
    if (t) *t = saru_tuning{0, 0, 0};
    return 0;
  }
  if (t) *t = saru_tuning{it->second.warps, it->second.ctas_per_sm, it->second.word_bits};
  return 1;
}

void saru_tuning_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
}

size_t saru_scratch_bytes(int32_t n, int32_t read_length, int32_t k, int wide) {
  int dev = current_device();
  if (dev < 0) dev = 0;
  return band_scratch_bytes(band_grid(dev, n, read_length, k), read_length, k, wide != 0);
}

int saru_align_host(const saru_batch *batch, saru_result *result, int lane) {
  g_last_error.clear();
  Lane &L = g_lanes[lane ? 1 : 0];
  std::lock_guard<std::mutex> lk(L.mu);
  return align_host_impl(batch, result, L, nullptr);
}

int saru_align_host_compact(const saru_batch *batch, int32_t *scores, uint8_t *records,
                            int64_t record_bytes, int32_t lane) {
  g_last_error.clear();
  if (!batch || batch->n < 0 || batch->k < 0 || (batch->n > 0 && (!scores || !records)) ||
      (record_bytes & 15) || record_bytes < 16) {
    set_error("saru_align_host_compact: a batch, scores, records and record_bytes a multiple "
              "of 16 (saru_compact_record_bytes)");
    return SARU_E_INVALID;
  }
  Lane &L = g_lanes[lane ? 1 : 0];
  std::lock_guard<std::mutex> lk(L.mu);
  const HostCompact hc{scores, records, (long)record_bytes};
  return align_host_impl(batch, nullptr, L, nullptr, &hc);
}

int saru_align_device(const saru_batch *batch, saru_result *result, void *scratch,
                      size_t scratch_bytes, void *stream) {
  g_last_error.clear();
  if (batch->n < 0 || batch->k < 0 || batch->k > 15 || batch->match != 0 ||
      batch->mismatch != 1 || batch->max_read_length < 2 ||
      batch->max_read_length > saru::kMaxBandM || !result->status) {
    set_error("saru_align_device: needs unit costs, k <= 15, 2 <= max_read_length <= %d and a "
              "status word",
              saru::kMaxBandM);
    return SARU_E_INVALID;
  }
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  Plan pl;
  pl.band = true;
  pl.max_m = batch->max_read_length;
  pl.wide = batch->k > 7;
  return run_band(batch, pl, result, scratch, scratch_bytes, result->status, dev,
                  reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Entry point without any device allocation.  Its scratch (the banded
// kernel's decision planes) is this file-scope device array, present on
// every GPU that loads the library for the life of the process.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = SARU_STATIC_SCRATCH_BYTES;
__device__ __align__(256) uint8_t g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void *g_static_ptr[kMaxDevices] = {};

// Device address of g_static_scratch on `dev` (the current device).  In host
// code the array's name is only a stand-in, so the address is asked for once
// per device with that device current.
int static_scratch_ptr(int dev, void **out) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device %d out of range", dev);
    return SARU_E_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress(g_static_scratch): %s", cudaGetErrorString(e));
      return SARU_E_CUDA;
    }
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return SARU_OK;
}

}  // namespace

namespace {
// The TSV lines of a legacy call, formatted on the host cores in ordered
// ranges of candidates and written in candidate order, then the output
// controls and counters (src/cuda-functions.cu:827-1006).
void legacy_write(const saru_batch &b, PinnedBuf *hb, const int *read_id_array,
                  const int *genome_pos_array, const char *direction_array, int error, int lane,
                  float ms) {
  const int n = b.n;
  const int32_t *scores = hb[0].as<int32_t>();
  std::shared_lock<std::shared_mutex> names_lk(g_names_mu);
  if (!g_names.covers(read_names, read_id_array, scores, n, error)) {
    names_lk.unlock();
    {
      std::unique_lock<std::shared_mutex> build_lk(g_names_mu);
      if (!g_names.covers(read_names, read_id_array, scores, n, error)) g_names.build(read_names);
    }
    names_lk.lock();
  }
  saru::WriterCall w{scores, hb[1].as<char>(), hb[2].as<char>(), b.total_slots,
                     b.genome_offsets, genome_pos_array,
                     reinterpret_cast<const int8_t *>(direction_array), read_id_array, error,
                     (int32_t)read_length_value, &NameIndex::lookup, &g_names};
  const int hw = (int)std::thread::hardware_concurrency();
  int nt = std::max(1, std::min(hw > 0 ? hw : 1, n / 16384 + 1));
  std::vector<std::string> text((size_t)nt);
  std::vector<int32_t> df((size_t)nt, 0), dr((size_t)nt, 0);
  auto part = [&](int i) {
    const int64_t lo = (int64_t)n * i / nt, hi = (int64_t)n * (i + 1) / nt;
    text[(size_t)i].reserve((size_t)(hi - lo) * 64);
    saru::format_range(w, lo, hi, &text[(size_t)i], &df[(size_t)i], &dr[(size_t)i]);
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nt; ++i) th.emplace_back(part, i);
  part(0);
  for (auto &t : th) t.join();
  std::lock_guard<std::mutex> lk(g_out_mu);
  for (const std::string &t : text) fwrite(t.data(), 1, t.size(), stdout);
  for (int v = 0; v < n; ++v) {
    if (scores[v] > error) continue;
    const int id = read_id_array[v];
    if (direction_array[v] > 3) {
      if (reverse_output_control) reverse_output_control[id] = 1;
    } else if (forward_output_control) {
      forward_output_control[id] = 1;
    }
  }
  for (int i = 0; i < nt; ++i) {
    forward_alignments_done += (unsigned)df[(size_t)i];
    reverse_alignments_done += (unsigned)dr[(size_t)i];
  }
  alignment_time[lane] += ms;
}
}  // namespace

extern "C" {

int saru_align_device_static(const saru_batch *batch, saru_result *result, void *stream) {
  g_last_error.clear();
  if (batch->n < 0 || batch->k < 0 || batch->k > 15 || batch->match != 0 ||
      batch->mismatch != 1 || batch->max_read_length < 2 ||
      batch->max_read_length > saru::kMaxBandM || !result->status) {
    set_error("saru_align_device_static: needs unit costs, k <= 15, 2 <= max_read_length <= %d "
              "and a status word",
              saru::kMaxBandM);
    return SARU_E_INVALID;
  }
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  void *scratch = nullptr;
  int rc = static_scratch_ptr(dev, &scratch);
  if (rc) return rc;
  Plan pl;
  pl.band = true;
  pl.max_m = batch->max_read_length;
  pl.wide = batch->k > 7;
  // as many persistent CTAs as the array holds planes for (each CTA's warps
  // need their own slice); a batch that cannot get even one CTA is refused
  const size_t per_cta = band_scratch_bytes(1, pl.max_m, batch->k, pl.wide);
  const long max_grid = (long)(kStaticScratchBytes / (per_cta ? per_cta : 1));
  if (max_grid < 1) {
    set_error("saru_align_device_static: one thread block needs %zu bytes of scratch, the "
              "static array holds %zu",
              per_cta, kStaticScratchBytes);
    return SARU_E_INVALID;
  }
  return run_band(batch, pl, result, scratch, kStaticScratchBytes, result->status, dev,
                  reinterpret_cast<cudaStream_t>(stream), max_grid);
}

int64_t saru_compact_record_bytes(int32_t max_read_length, int32_t k) {
  if (max_read_length < 1 || k < 0) return -1;
  return saru::compact_record_bytes(max_read_length, k);
}

int saru_align_device_compact(const saru_batch *batch, int32_t *scores, uint8_t *records,
                              int64_t record_bytes, int32_t *status, void *scratch,
                              size_t scratch_bytes, void *stream) {
  g_last_error.clear();
  if (batch->n < 0 || batch->k < 0 || batch->k > 15 || batch->match != 0 ||
      batch->mismatch != 1 || batch->max_read_length < 2 ||
      batch->max_read_length > saru::kMaxBandM || !status || !scores ||
      (batch->n > 0 && !records) ||
      record_bytes < saru::compact_record_bytes(batch->max_read_length, batch->k) ||
      (record_bytes & 15)) {
    set_error("saru_align_device_compact: needs unit costs, k <= 15, 2 <= max_read_length <= "
              "%d, scores, records of at least saru_compact_record_bytes (a multiple of 16) "
              "and a status word",
              saru::kMaxBandM);
    return SARU_E_INVALID;
  }
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  Plan pl;
  pl.band = true;
  pl.max_m = batch->max_read_length;
  pl.wide = batch->k > 7;
  const saru_result r{scores, nullptr, nullptr, status};
  const CompactOut cmp{records, (long)record_bytes};
  return run_band(batch, pl, &r, scratch, scratch_bytes, status, dev,
                  reinterpret_cast<cudaStream_t>(stream), 0, &cmp);
}

int saru_align_multi_device_compact(const saru_batch *calls, saru_result *results,
                                    int32_t ncalls, int32_t *status, void *scratch,
                                    size_t scratch_bytes, void *stream) {
  g_last_error.clear();
  if (ncalls < 1 || ncalls > saru::kMaxSegs || !status || !results) {
    set_error("saru_align_multi_device_compact: 1..%d calls, results and a status word",
              saru::kMaxSegs);
    return SARU_E_INVALID;
  }
  std::vector<CompactOut> cmp((size_t)ncalls);
  for (int i = 0; i < ncalls; ++i) {
    const saru_batch *b = &calls[i];
    if (b->n < 0 || b->k < 0 || b->k > 15 || b->match != 0 || b->mismatch != 1 ||
        b->max_read_length < 2 || b->max_read_length > saru::kMaxBandM ||
        (b->n > 0 && !results[i].read_aln)) {
      set_error("saru_align_multi_device_compact: call %d needs unit costs, k <= 15, "
                "2 <= max_read_length <= %d and a records array",
                i, saru::kMaxBandM);
      return SARU_E_INVALID;
    }
    cmp[(size_t)i] = CompactOut{reinterpret_cast<uint8_t *>(results[i].read_aln),
                                (long)saru::compact_record_bytes(b->max_read_length, b->k)};
  }
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  return run_band_classes(calls, results, ncalls, scratch, scratch_bytes, status, dev,
                          reinterpret_cast<cudaStream_t>(stream), cmp.data());
}

size_t saru_multi_scratch_bytes(const saru_batch *calls, int32_t ncalls) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  return classes_scratch_bytes(plan_classes(calls, ncalls, dev));
}

int saru_align_multi_device(const saru_batch *calls, saru_result *results, int32_t ncalls,
                            int32_t *status, void *scratch, size_t scratch_bytes, void *stream) {
  g_last_error.clear();
  if (ncalls < 1 || ncalls > saru::kMaxSegs || !status) {
    set_error("saru_align_multi_device: 1..%d calls and a status word", saru::kMaxSegs);
    return SARU_E_INVALID;
  }
  for (int i = 0; i < ncalls; ++i) {
    const saru_batch *b = &calls[i];
    if (b->n < 0 || b->k < 0 || b->k > 15 || b->match != 0 || b->mismatch != 1 ||
        b->max_read_length < 2 || b->max_read_length > saru::kMaxBandM) {
      set_error("saru_align_multi_device: call %d needs unit costs, k <= 15 and "
                "2 <= max_read_length <= %d",
                i, saru::kMaxBandM);
      return SARU_E_INVALID;
    }
  }
  int dev = 0;
  SARU_CUDA(cudaGetDevice(&dev));
  return run_band_classes(calls, results, ncalls, scratch, scratch_bytes, status, dev,
                          reinterpret_cast<cudaStream_t>(stream));
}

int64_t saru_format_tsv(const saru_batch *batch, const saru_result *result,
                        const int32_t *read_ids, const int32_t *genome_pos, int32_t read_length,
                        const char *names, int32_t name_stride, int32_t n_names, char *out,
                        int64_t cap, int32_t *done_fwd, int32_t *done_rev) {
  struct Tab {
    const char *names;
    int32_t stride, n;
    static const char *get(void *c, int32_t id) {
      auto *t = static_cast<Tab *>(c);
      return (id >= 0 && id < t->n) ? t->names + (int64_t)id * t->stride : nullptr;
    }
  } tab{names, name_stride, n_names};
  saru::WriterCall w{result->scores, result->read_aln, result->genome_aln, batch->total_slots,
                     batch->genome_offsets, genome_pos, batch->dirs, read_ids, batch->k,
                     read_length, &Tab::get, &tab};
  // ordered ranges of candidates on the host cores, concatenated in order
  const int64_t n = batch->n;
  const int hw = (int)std::thread::hardware_concurrency();
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw > 0 ? hw : 1, n / 16384 + 1));
  std::vector<std::string> text((size_t)nt);
  std::vector<int32_t> df((size_t)nt, 0), dr((size_t)nt, 0);
  auto part = [&](int i) {
    saru::format_range(w, n * i / nt, n * (i + 1) / nt, &text[(size_t)i], &df[(size_t)i],
                       &dr[(size_t)i]);
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nt; ++i) th.emplace_back(part, i);
  part(0);
  for (auto &t : th) t.join();
  int64_t total = 0;
  int32_t f = 0, r = 0;
  for (int i = 0; i < nt; ++i) {
    const std::string &t = text[(size_t)i];
    if (out && total < cap)
      memcpy(out + total, t.data(), (size_t)std::min<int64_t>((int64_t)t.size(), cap - total));
    total += (int64_t)t.size();
    f += df[(size_t)i];
    r += dr[(size_t)i];
  }
  if (done_fwd) *done_fwd = f;
  if (done_rev) *done_rev = r;
  return total;
}

void cuda_allocate_memory(int do_reverse) {
  const int lane = do_reverse == 4 ? 1 : 0;
  const int dev = current_device();
  if (dev < 0) {
    fprintf(stderr, "saruman_b200: no CUDA device\n");
    return;
  }
  std::lock_guard<std::mutex> lk(g_lanes[lane].mu);
  if (g_lanes[lane].init(dev) != SARU_OK) {
    fprintf(stderr, "saruman_b200: %s\n", g_last_error.c_str());
    return;
  }
  // the reference keeps its arena base in these globals; here they mark the
  // lane as prepared (memory is allocated per call, on demand)
  char *marker = reinterpret_cast<char *>(g_lanes[lane].stream);
  if (lane) main_alloc_ptr_rev = marker;
  else main_alloc_ptr_for = marker;
}

void cuda_free_memory(int do_reverse) {
  const int lane = do_reverse ? 1 : 0;
  std::lock_guard<std::mutex> lk(g_lanes[lane].mu);
  g_lanes[lane].release();
  if (lane) main_alloc_ptr_rev = nullptr;
  else main_alloc_ptr_for = nullptr;
}

unsigned long int get_cuda_infos(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    count = 0;
  }
  fprintf(stderr, "\n=== CUDA hardware ===\n");
  fprintf(stderr, "Detected %d GPU(s):\n\n", count);
  size_t most_free = 0;
  int best = 0, i;
  int caller_dev = 0;  // restored after the scan: the caller's current device
  const bool had_dev = cudaGetDevice(&caller_dev) == cudaSuccess;
  for (i = 0; i < count; ++i) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, i);
    size_t fr = 0, tot = 0;
    cudaSetDevice(i);
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fprintf(stderr, "GPU %d: %s\t", i, prop.name);
      fprintf(stderr, "Could not get memory information from GPU.\nShutting down.\n");
      exit(-1);
    }
    if (fr > most_free) {
      most_free = fr;
      best = i;
    }
    fprintf(stderr, "GPU %d: %s\t", i, prop.name);
    fprintf(stderr, "[%*lu/%*lu MB available]\n", 4, (unsigned long)(fr / (1024 * 1024)), 4,
            (unsigned long)(tot / (1024 * 1024)));
  }
  if (had_dev && count > 0) cudaSetDevice(caller_dev);
  if (most_free < 128000000UL) {
    fprintf(stderr, "\n-> SARUMAN was not able to find a GPU with enough VRAM available! (available: %lu MB)\n",
            (unsigned long)(most_free / (1024 * 1024)));
    exit(1);
  } else if (use_gpu_value <= i) {
    fprintf(stderr, "\n-> SARUMAN was forced to run on GPU %d\n", use_gpu_value);
  } else {
    fprintf(stderr, "\n-> SARUMAN will run on GPU %d\n", best);
    use_gpu_value = (unsigned short)best;
  }
  return (unsigned long)most_free;
}

void cuda_needleman_wunsch(int match, int mismatch, char *genome_sequences_on_host,
                           char *read_sequences_on_host, int *genome_offsets, int *read_offsets,
                           int *edit_offsets, int sample_size, int *read_id_array,
                           int *genome_pos_array, char *direction_array, int error,
                           size_t total_genome_array_size, size_t total_read_sequence_array_size,
                           size_t total_edit_matrix_size, int do_reverse) {
  (void)edit_offsets;
  (void)total_read_sequence_array_size;
  (void)total_edit_matrix_size;
  g_last_error.clear();
  fprintf(stderr, "\t\t-> starting CUDA kernel with %d samples from %s thread\n", sample_size,
          (do_reverse ? "reverse" : "forward"));
  {
    std::lock_guard<std::mutex> lk(g_out_mu);
    if (do_reverse) reverse_alignment_candidates += sample_size;
    else forward_alignment_candidates += sample_size;
  }
  if (sample_size <= 0) return;
  const int n = sample_size;
  const size_t slots = total_genome_array_size;
  const int lane = do_reverse ? 1 : 0;
  saru_batch b{};
  b.genome = genome_sequences_on_host;
  b.reads = read_sequences_on_host;
  b.genome_offsets = genome_offsets;
  b.read_offsets = read_offsets;
  b.dirs = reinterpret_cast<const int8_t *>(direction_array);
  b.n = n;
  b.k = error;
  b.match = match;
  b.mismatch = mismatch;
  b.first_of_call = 1;
  b.genome_bytes = genome_offsets[n - 1];
  b.total_slots = (int64_t)slots;
  float ms = 0.f;
  int rc;
  PinnedBuf *hb = g_legacy_out[lane];
  {
    std::lock_guard<std::mutex> lk(g_lanes[lane].mu);
    // the lane's pinned result arrays, reused call after call; 64 zero bytes
    // past the slots (the writer's scans may look past the last slot)
    rc = hb[0].ensure(4 * (size_t)n);
    if (!rc) rc = hb[1].ensure(slots + 64);
    if (!rc) rc = hb[2].ensure(slots + 64);
    if (!rc) {
      memset(hb[1].as<char>() + slots, 0, 64);
      memset(hb[2].as<char>() + slots, 0, 64);
      saru_result r{hb[0].as<int32_t>(), hb[1].as<char>(), hb[2].as<char>(), nullptr};
      rc = align_host_impl(&b, &r, g_lanes[lane], &ms);
    }
    if (rc == SARU_OK) legacy_write(b, hb, read_id_array, genome_pos_array, direction_array,
                                    error, lane, ms);
  }
  if (rc != SARU_OK)
    fprintf(stderr, "ERROR: saruman_b200 alignment failed: %s\n", g_last_error.c_str());
}

}  // extern "C"
