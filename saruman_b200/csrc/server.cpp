// server.cpp -- request loop with continuous batching on one GPU.
//
// A request is a set of reference-style calls (host arrays in, host arrays
// out), typically one per read-length bin.  The scheduler thread admits
// requests in arrival order while the device arena has room for their
// inputs and outputs; the requests admitted together form a launch group
// whose calls all go to one multi-call request of the banded kernel (one
// persistent launch per read-length class, classes concurrent).  Three
// streams overlap the work: the inputs of group i+1 are copied in while
// group i computes, and the completion thread copies group i's results out
// while group i+1 computes.  Requests that arrive while groups are on the GPU
// join the next group as arena space and launch slots free up.
//
// Plain mode (pipeline = 0) processes one request at a time, one launch per
// call and a full round trip before the next request: the per-request loop
// the batched mode is measured against.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/saruman_b200.h"
#include "kernels.cuh"
#include "saru_core.cuh"
#include "server_internal.h"

namespace {

int64_t now_us() {
  return std::chrono::duration_cast<std::chrono::microseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// How long the filter thread waits for room in the pinned result pool
// before it gives a request pageable memory instead (a client that keeps
// its results does not stall the server for longer).
constexpr int kPoolWaitMs = 200;

// First-fit allocator over one device allocation (the admission budget).
class Arena {
 public:
  bool init(size_t bytes) {
    if (cudaMalloc(&base_, bytes) != cudaSuccess) {
      base_ = nullptr;
      return false;
    }
    size_ = bytes;
    free_[0] = bytes;
    return true;
  }
  void release() {
    if (base_) cudaFree(base_);
    base_ = nullptr;
  }
  long alloc(size_t bytes) {  // offset, or -1 when no free range is large enough
    bytes = up256(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      return (long)off;
    }
    return -1;
  }
  void free(size_t off, size_t bytes) {
    bytes = up256(bytes);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  uint8_t *ptr(size_t off) const { return static_cast<uint8_t *>(base_) + off; }
  size_t size() const { return size_; }

 private:
  void *base_ = nullptr;
  size_t size_ = 0;
  std::map<size_t, size_t> free_;  // offset -> length
};

// Results of one read set of a reads-only request, owned by the server:
// the filter's calls (both strands), their gather descriptors and outputs.
// First-fit allocator over one pinned host allocation (reads-only requests'
// results: copies out of pinned memory run at full bus speed and take no
// page faults).  Thread-safe.
class HostPool {
 public:
  ~HostPool() {
    if (base_) cudaFreeHost(base_);
  }
  long alloc(size_t bytes, size_t want_total) {
    std::lock_guard<std::mutex> lk(mu_);
    return alloc_locked(bytes, want_total);
  }
  // As alloc, but when the pool has no room for `bytes` now (and could hold
  // them), waits up to wait_ms for results to be freed.  The filter thread
  // runs ahead of the aligner; without this it fills the pool with results
  // of requests far ahead and the rest go to pageable memory.
  long alloc_wait(size_t bytes, size_t want_total, int wait_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(wait_ms);
    for (;;) {
      const long off = alloc_locked(bytes, want_total);
      if (off >= 0 || !base_ || up256(bytes) > size_) return off;
      if (freed_.wait_until(lk, until) == std::cv_status::timeout)
        return alloc_locked(bytes, want_total);
    }
  }

 private:
  long alloc_locked(size_t bytes, size_t want_total) {
    if (!base_ && !tried_) {  // on first use
      tried_ = true;
      if (cudaMallocHost(&base_, want_total) != cudaSuccess) {
        cudaGetLastError();
        base_ = nullptr;
      } else {
        size_ = want_total;
        free_[0] = want_total;
      }
    }
    if (!base_) return -1;
    bytes = up256(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      return (long)off;
    }
    return -1;
  }

 public:
  void free(size_t off, size_t bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    freed_.notify_all();
    bytes = up256(bytes);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  char *ptr(size_t off) const { return static_cast<char *>(base_) + off; }

 private:
  std::mutex mu_;
  std::condition_variable freed_;
  void *base_ = nullptr;
  size_t size_ = 0;
  bool tried_ = false;
  std::map<size_t, size_t> free_;
};

struct ReadSetOut {
  saru_read_set set{};
  std::vector<int64_t> call_begin{0}, slot_begin{0};
  std::vector<int8_t> call_strand;
  std::vector<int32_t> ids, pos, goff, rindex, scores;
  std::vector<int8_t> dirs;
  // outputs, written whole by the copies out (not zero-filled first): in
  // the server's pinned pool when it has room (pool offset >= 0), else in
  // pageable memory the set owns
  char *ra = nullptr, *ga = nullptr;
  uint8_t *records = nullptr;
  long pool_off = -1;
  size_t pool_bytes = 0;
  std::unique_ptr<char[]> owned;
  int64_t rec_bytes = 0;
  std::vector<int32_t> perfect_ids, perfect_pos;
  std::vector<int8_t> perfect_strand;
  std::vector<saru_gather_call> gcalls;  // this set's calls
  std::vector<saru_result> results;
  int rc = SARU_OK;
};

struct Request {
  int64_t ticket = 0;
  bool gather = false;                  // calls given as saru_gather_call (resident genome)
  bool compact = false;                 // compact records instead of slot strings
  std::vector<saru_gather_call> gcalls; // host views (caller's arrays), when gather
  std::vector<saru_batch> calls;     // host views (caller's arrays); shapes only when gather
  std::vector<saru_result> results;  // host outputs (caller's arrays)
  std::vector<saru_batch> dcalls;    // device views inside the arena
  std::vector<saru_result> dres;
  std::vector<saru::CompactOut> dcmp;  // device records per call (compact requests)
  std::vector<int32_t> call_status;  // kernel status bits per call, read back
  size_t dev_bytes = 0;
  long dev_off = -1;
  int32_t *dstatus = nullptr;  // one device word per call, inside the arena
  int64_t t_submit = 0, t_admit = 0, t_done = 0;
  int32_t group = -1, redone = 0;
  int rc = SARU_OK;
  bool done = false;
  size_t pooled = 0;  // pinned pool bytes of its results (reads-only requests)
  std::vector<ReadSetOut> rsets;  // reads-only request: its sets and results
};

// Read bytes of call i (the gathered reads of a gather call).
size_t read_bytes(const Request &r, size_t i) {
  const saru_batch &b = r.calls[i];
  if (r.gather) return (size_t)b.n * (size_t)b.max_read_length;
  return b.n ? (size_t)b.read_offsets[b.n - 1] : 0;
}

size_t record_bytes(const saru_batch &b) {
  return (size_t)saru_compact_record_bytes(b.max_read_length, b.k);
}

// Device bytes of a call's results: two slot arrays, or its records.
size_t output_bytes(const Request &r, const saru_batch &b) {
  return r.compact ? up256((size_t)b.n * record_bytes(b) + 64)
                   : 2 * up256((size_t)b.total_slots + 64);
}

// Arena bytes one request takes: every device array up256-aligned.
size_t request_bytes(const Request &r) {
  size_t t = up256(4 * r.calls.size());  // status words
  for (size_t i = 0; i < r.calls.size(); ++i) {
    const saru_batch &b = r.calls[i];
    const size_t n = (size_t)b.n;
    t += up256((size_t)b.genome_bytes + 64);
    t += up256(read_bytes(r, i) + 64);
    t += 3 * up256(4 * n + 64);  // genome_offsets, read_offsets, scores
    t += up256(n + 64);          // dirs
    t += output_bytes(r, b);
    if (r.gather)  // read table, read_index, positions
      t += up256((size_t)r.gcalls[i].nreads * (size_t)b.max_read_length + 64) +
           2 * up256(4 * n + 64);
  }
  return t;
}

// The saru_batch shape of a gather call (pointers unset).
saru_batch shape_of(const saru_gather_call &g) {
  return saru_batch{nullptr, nullptr, g.genome_offsets, nullptr, g.dirs, g.n, g.k,
                    g.match, g.mismatch, g.first_of_call, g.read_length, g.genome_bytes,
                    g.total_slots};
}

}  // namespace

struct saru_server {
  saru_server_config cfg{};
  Arena arena;
  cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  // resident genome of gather requests: 2 bits a base, non-ACGT bytes as
  // exceptions (device memory: one quarter of the bytes plus the exceptions)
  uint8_t *genome = nullptr;
  int64_t *exc_pos = nullptr;
  uint8_t *exc_byte = nullptr;
  saru::PackedGenome pg;
  int64_t genome_len = 0;
  std::vector<char> genome_host;  // the same genome, for the filters' q-gram indexes
  HostPool host_pool;             // pinned memory for reads-only requests' results
  // filters per worker and (read length, k): the filter stage runs
  // kFilterWorkers requests at once in pipeline mode (one request's host
  // call assembly overlaps another's kernel and copies), one in plain mode
  static constexpr int kFilterWorkers = 2;
  std::map<std::pair<int, int>, saru_filter *> filters[kFilterWorkers];

  struct Group {
    std::vector<std::shared_ptr<Request>> reqs;
    cudaEvent_t done_ev = nullptr;  // recorded on s_comp after the launch
    int rc = SARU_OK;
  };

  std::mutex mu;
  std::condition_variable cv_pending, cv_inflight, cv_freed, cv_done;
  std::deque<std::shared_ptr<Request>> pending;
  std::deque<Group> inflight;
  std::unordered_map<int64_t, std::shared_ptr<Request>> tickets;
  std::unordered_map<int64_t, std::shared_ptr<Request>> read_done;  // until released
  std::deque<std::shared_ptr<Request>> filter_q;  // reads-only requests to filter
  std::condition_variable cv_filter;
  // filtered requests wait here until those that arrived before them have
  // gone on (to the pending queue, or done): arrival order is kept
  std::map<int64_t, std::shared_ptr<Request>> filtered;
  int64_t filter_taken = 0, filter_next = 0;  // sequence numbers
  // pinned pool bytes held by filtered requests that are not done yet; in
  // pipeline mode a filter worker takes no new request while they exceed
  // ahead_limit (half the pool), so the filter cannot fill the pool with
  // results of requests far ahead of the aligner
  size_t ahead_bytes = 0, ahead_limit = 0;
  int64_t next_ticket = 1, groups = 0, launches = 0, free_gen = 0;
  bool stop = false, sched_done = false, filter_stop = false;
  std::thread sched_thr, done_thr;
  std::vector<std::thread> filter_thrs;

  void free_genome() {
    if (genome) cudaFree(genome);
    if (exc_pos) cudaFree(exc_pos);
    if (exc_byte) cudaFree(exc_byte);
    genome = nullptr;
    exc_pos = nullptr;
    exc_byte = nullptr;
    pg = saru::PackedGenome{};
    genome_len = 0;
  }

  // Returns a reads-only request's pooled result ranges to the pool.
  void free_outputs(Request &r) {
    for (auto &o : r.rsets)
      if (o.pool_off >= 0) {
        host_pool.free((size_t)o.pool_off, o.pool_bytes);
        o.pool_off = -1;
        o.ra = o.ga = nullptr;
        o.records = nullptr;
      }
  }

  size_t pool_bytes() const {
    return (size_t)(cfg.host_pool_bytes > 0 ? cfg.host_pool_bytes : (int64_t)4 << 30);
  }

  // The filter of (m, k) for worker w.  The first use of (m, k) by any
  // worker builds it for every worker: a worker that built its own on its
  // first request of that length would stall that request (and, through
  // the in-order hand-off, every one behind it) for the index build.
  std::mutex filters_mu;
  saru_filter *filter_for(int m, int k, int w) {
    std::lock_guard<std::mutex> lk(filters_mu);
    auto it = filters[w].find({m, k});
    if (it != filters[w].end()) return it->second;
    for (auto &fv : filters) {
      if (fv.count({m, k})) continue;
      saru_filter *f = saru_filter_create(genome_host.data(), (int64_t)genome_host.size(), m,
                                          k, cfg.device);
      if (!f) return nullptr;
      fv[{m, k}] = f;
    }
    return filters[w][{m, k}];
  }
  void destroy_filters() {
    for (auto &fw : filters) {
      for (auto &kv : fw) saru_filter_destroy(kv.second);
      fw.clear();
    }
  }

  // One read set through the filter on both strands: its calls as gather
  // calls over the set's own read table, outputs in the set's arrays.
  int filter_set(Request &r, ReadSetOut &o, int w) {
    const saru_read_set &rs = o.set;
    const int m = rs.read_length, k = rs.k;
    saru_filter *f = filter_for(m, k, w);
    if (!f) return SARU_E_INVALID;
    const uint32_t cv = rs.chunk_value
                            ? rs.chunk_value
                            : (uint32_t)(0.92 * 2147483648.0 / ((m + 1.0) * (m + 2.0 * k + 1.0)) /
                                         1000.0) * 1000u;
    for (int dr : {0, 4}) {
      int64_t cnt[3] = {0, 0, 0};
      int rc = saru_filter_run(f, rs.reads, rs.nreads, dr, cv, cnt);
      if (rc) return rc;
      const size_t nc = (size_t)cnt[0], na = (size_t)cnt[1], np = (size_t)cnt[2];
      std::vector<int64_t> cb(nc + 1);
      const size_t a0 = o.ids.size(), p0 = o.perfect_ids.size();
      o.ids.resize(a0 + na);
      o.pos.resize(a0 + na);
      o.dirs.resize(a0 + na);
      o.perfect_ids.resize(p0 + np);
      o.perfect_pos.resize(p0 + np);
      o.perfect_strand.resize(p0 + np, (int8_t)dr);
      if ((rc = saru_filter_results(f, cb.data(), o.ids.data() + a0, o.pos.data() + a0,
                                    o.dirs.data() + a0, o.perfect_ids.data() + p0,
                                    o.perfect_pos.data() + p0)))
        return rc;
      for (size_t c = 0; c < nc; ++c) {
        o.call_begin.push_back((int64_t)a0 + cb[c + 1]);
        o.call_strand.push_back((int8_t)dr);
      }
    }
    const size_t n = o.ids.size(), ncalls = o.call_strand.size();
    o.goff.resize(n);
    o.rindex.resize(n);
    o.scores.assign(n, 0);
    int64_t slots = 0;
    for (size_t c = 0; c < ncalls; ++c) {
      const int64_t a = o.call_begin[c], b = o.call_begin[c + 1];
      int64_t acc = 0;
      int32_t lo = INT32_MAX, hi = -1;
      for (int64_t t = a; t < b; ++t) {
        int so = 0, eo = 0;
        saru::flank_of(o.dirs[(size_t)t], k, so, eo);
        acc += m + so + eo;
        o.goff[(size_t)t] = (int32_t)acc;
        lo = std::min(lo, o.ids[(size_t)t]);
        hi = std::max(hi, o.ids[(size_t)t]);
      }
      for (int64_t t = a; t < b; ++t) o.rindex[(size_t)t] = o.ids[(size_t)t] - lo;
      slots += acc + (int64_t)k * (b - a);
      o.slot_begin.push_back(slots);
      saru_gather_call g{};
      g.read_table = rs.reads + (size_t)lo * (size_t)m;
      g.read_index = o.rindex.data() + a;
      g.positions = o.pos.data() + a;
      g.dirs = o.dirs.data() + a;
      g.genome_offsets = o.goff.data() + a;
      g.n = (int32_t)(b - a);
      g.nreads = hi - lo + 1;
      g.k = k;
      g.match = 0;
      g.mismatch = 1;
      g.first_of_call = 1;
      g.read_length = m;
      g.genome_bytes = acc;
      g.total_slots = acc + (int64_t)k * (b - a);
      o.gcalls.push_back(g);
    }
    if (r.compact) o.rec_bytes = saru_compact_record_bytes(m, k);
    const size_t half = r.compact ? n * (size_t)o.rec_bytes + 64 : (size_t)slots + 64;
    const size_t total = r.compact ? half : 2 * up256(half);
    o.pool_off = host_pool.alloc_wait(total, pool_bytes(), kPoolWaitMs);
    char *base;
    if (o.pool_off >= 0) {
      o.pool_bytes = total;
      base = host_pool.ptr((size_t)o.pool_off);
    } else {  // the pool is full or unavailable: pageable memory of the set's own
      o.owned.reset(new char[total]);
      base = o.owned.get();
    }
    if (r.compact) {
      o.records = reinterpret_cast<uint8_t *>(base);
    } else {
      o.ra = base;
      o.ga = base + up256(half);
      memset(o.ra + slots, 0, 64);
      memset(o.ga + slots, 0, 64);
    }
    for (size_t c = 0; c < ncalls; ++c) {
      const int64_t a = o.call_begin[c];
      saru_result res{o.scores.data() + a, nullptr, nullptr, nullptr};
      if (r.compact) {
        res.read_aln = reinterpret_cast<char *>(o.records + a * o.rec_bytes);
      } else {
        res.read_aln = o.ra + o.slot_begin[c];
        res.genome_aln = o.ga + o.slot_begin[c];
      }
      o.results.push_back(res);
    }
    return SARU_OK;
  }

  // Filter workers: reads-only requests become gather requests on the
  // pending queue (or finish here with an error or nothing to align), while
  // the scheduler and completer work on earlier ones.  In pipeline mode
  // kFilterWorkers requests are filtered at once, each worker with its own
  // filters; a filtered request goes on only after every request that
  // arrived before it, so the pending queue keeps arrival order.  Plain mode
  // has one worker, and the next request's filter waits for this one.
  void filterer(int w) {
    cudaSetDevice(cfg.device);
    for (;;) {
      std::shared_ptr<Request> r;
      int64_t seq = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_filter.wait(lk, [&] {
          return filter_stop ||
                 (!filter_q.empty() && (!cfg.pipeline || ahead_bytes < ahead_limit));
        });
        if (filter_q.empty()) return;
        r = filter_q.front();
        filter_q.pop_front();
        seq = filter_taken++;
      }
      int rc = SARU_OK;
      // the sets' filters (one per read length and k) run at once, each on
      // its own stream; sets sharing a filter run one after the other
      std::vector<std::pair<int, int>> keys;
      for (auto &o : r->rsets) {
        const std::pair<int, int> key(o.set.read_length, o.set.k);
        if (!filter_for(key.first, key.second, w)) rc = SARU_E_INVALID;
        if (std::find(keys.begin(), keys.end(), key) == keys.end()) keys.push_back(key);
      }
      if (!rc) {
        std::vector<std::thread> th;
        for (const auto &key : keys)
          th.emplace_back([this, &r, key, w] {
            cudaSetDevice(cfg.device);
            for (auto &o : r->rsets)
              if (o.set.read_length == key.first && o.set.k == key.second && !o.rc)
                o.rc = filter_set(*r, o, w);
          });
        for (auto &t : th) t.join();
        for (auto &o : r->rsets)
          if (!rc && o.rc) rc = o.rc;
      }
      for (auto &o : r->rsets) {
        r->gcalls.insert(r->gcalls.end(), o.gcalls.begin(), o.gcalls.end());
        r->results.insert(r->results.end(), o.results.begin(), o.results.end());
      }
      if (!rc && r->gcalls.size() > (size_t)SARU_MAX_CALLS) {
        saru::set_last_error("reads-only request: more than SARU_MAX_CALLS calls");
        rc = SARU_E_INVALID;
      }
      if (!rc) {
        for (const auto &g : r->gcalls) r->calls.push_back(shape_of(g));
        r->dev_bytes = request_bytes(*r);
        if (r->dev_bytes > arena.size()) {
          saru::set_last_error("reads-only request larger than the device budget");
          rc = SARU_E_NOMEM;
        }
      }
      r->rc = rc;
      for (auto &o : r->rsets)
        if (o.pool_off >= 0) r->pooled += o.pool_bytes;
      std::unique_lock<std::mutex> lk(mu);
      filtered[seq] = r;
      ahead_bytes += r->pooled;
      // hand on, in arrival order, every request whose predecessors have gone
      for (auto it = filtered.find(filter_next); it != filtered.end();
           it = filtered.find(filter_next)) {
        std::shared_ptr<Request> q = it->second;
        filtered.erase(it);
        ++filter_next;
        if (q->rc || q->calls.empty()) {
          q->t_done = now_us();
          q->done = true;
          ahead_bytes -= q->pooled;
          cv_done.notify_all();
          cv_filter.notify_all();
        } else {
          pending.push_back(q);
          cv_pending.notify_all();
        }
      }
      if (!cfg.pipeline) cv_done.wait(lk, [&] { return r->done; });
    }
  }

  // Carves a request's device arrays out of its arena range and copies its
  // inputs in on s_in.
  void stage(Request &r) {
    uint8_t *p = arena.ptr((size_t)r.dev_off);
    auto take = [&](size_t bytes) {
      uint8_t *q = p;
      p += up256(bytes);
      return q;
    };
    const size_t nc = r.calls.size();
    r.dstatus = reinterpret_cast<int32_t *>(take(4 * nc));
    cudaMemsetAsync(r.dstatus, 0, 4 * nc, s_in);
    r.dcalls.resize(nc);
    r.dres.resize(nc);
    r.dcmp.assign(nc, saru::CompactOut{nullptr, 0});
    for (size_t i = 0; i < nc; ++i) {
      const saru_batch &h = r.calls[i];
      const size_t n = (size_t)h.n;
      const size_t rbytes = read_bytes(r, i);
      uint8_t *g = take((size_t)h.genome_bytes + 64), *rd = take(rbytes + 64);
      uint8_t *go = take(4 * n + 64), *ro = take(4 * n + 64), *sc = take(4 * n + 64);
      uint8_t *dr = take(n + 64);
      uint8_t *ra = nullptr, *ga = nullptr;
      if (r.compact) {
        ra = take(n * record_bytes(h) + 64);
        r.dcmp[i] = saru::CompactOut{ra, (long)record_bytes(h)};
      } else {
        ra = take((size_t)h.total_slots + 64);
        ga = take((size_t)h.total_slots + 64);
      }
      saru_batch &d = r.dcalls[i];
      d = h;
      d.genome = reinterpret_cast<const char *>(g);
      d.reads = reinterpret_cast<const char *>(rd);
      d.genome_offsets = reinterpret_cast<const int32_t *>(go);
      d.read_offsets = reinterpret_cast<const int32_t *>(ro);
      d.dirs = reinterpret_cast<const int8_t *>(dr);
      r.dres[i] = saru_result{reinterpret_cast<int32_t *>(sc), reinterpret_cast<char *>(ra),
                              reinterpret_cast<char *>(ga), r.dstatus + i};
      if (!n) continue;
      cudaMemcpyAsync(go, h.genome_offsets, 4 * n, cudaMemcpyHostToDevice, s_in);
      cudaMemcpyAsync(dr, h.dirs, n, cudaMemcpyHostToDevice, s_in);
      if (!r.gather) {
        cudaMemcpyAsync(g, h.genome, (size_t)h.genome_bytes, cudaMemcpyHostToDevice, s_in);
        cudaMemcpyAsync(rd, h.reads, rbytes, cudaMemcpyHostToDevice, s_in);
        cudaMemcpyAsync(ro, h.read_offsets, 4 * n, cudaMemcpyHostToDevice, s_in);
        continue;
      }
      // filter output in, windows and reads gathered from the resident genome
      const saru_gather_call &hg = r.gcalls[i];
      const size_t tbytes = (size_t)hg.nreads * (size_t)hg.read_length;
      uint8_t *tab = take(tbytes + 64), *ri = take(4 * n + 64), *ps = take(4 * n + 64);
      cudaMemcpyAsync(tab, hg.read_table, tbytes, cudaMemcpyHostToDevice, s_in);
      cudaMemcpyAsync(ri, hg.read_index, 4 * n, cudaMemcpyHostToDevice, s_in);
      cudaMemcpyAsync(ps, hg.positions, 4 * n, cudaMemcpyHostToDevice, s_in);
      saru_gather_call dg = hg;
      dg.read_table = reinterpret_cast<const char *>(tab);
      dg.read_index = reinterpret_cast<const int32_t *>(ri);
      dg.positions = reinterpret_cast<const int32_t *>(ps);
      dg.dirs = d.dirs;
      dg.genome_offsets = d.genome_offsets;
      saru_batch gathered;
      if (saru::gather_packed(&dg, pg, reinterpret_cast<char *>(g), reinterpret_cast<char *>(rd),
                              reinterpret_cast<int32_t *>(ro), r.dstatus + i, &gathered,
                              s_in) != SARU_OK)
        r.rc = SARU_E_CUDA;
    }
  }

  // A flagged call, redone on the exact path as saru_align_host does.  A
  // gather call's windows and reads come back from the arena first; a
  // compact request gets the exact path's slot strings as records.
  int redo_call(Request &r, size_t i) {
    saru_batch h = r.calls[i];
    const size_t n = (size_t)h.n;
    std::vector<char> win, rd;
    std::vector<int32_t> ro;
    if (r.gather) {
      const saru_batch &d = r.dcalls[i];
      win.resize((size_t)d.genome_bytes);
      rd.resize(read_bytes(r, i));
      ro.resize(n);
      if (cudaMemcpy(win.data(), d.genome, win.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(rd.data(), d.reads, rd.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        saru::set_last_error(cudaGetErrorString(cudaGetLastError()));
        return SARU_E_CUDA;
      }
      for (size_t t = 0; t < n; ++t) ro[t] = (int32_t)((t + 1) * (size_t)d.max_read_length);
      h.genome = win.data();
      h.reads = rd.data();
      h.read_offsets = ro.data();
    }
    if (!r.compact) return saru::redo_on_host_path(&h, &r.results[i]);
    std::vector<char> sr((size_t)h.total_slots + 64), sg((size_t)h.total_slots + 64);
    saru_result tmp{r.results[i].scores, sr.data(), sg.data(), nullptr};
    const int rc = saru::redo_on_host_path(&h, &tmp);
    if (rc) return rc;
    return saru::records_from_slots(&h, tmp.scores, sr.data(), sg.data(),
                                    reinterpret_cast<uint8_t *>(r.results[i].read_aln),
                                    (long)record_bytes(h));
  }

  int ensure_scratch(size_t bytes) {
    if (bytes <= scratch_bytes) return SARU_OK;
    // stream-ordered on s_comp: the old scratch is freed after the launches
    // already enqueued there, and nothing waits (a plain cudaFree would
    // synchronize the whole device, the filters' work and copies included)
    if (scratch) cudaFreeAsync(scratch, s_comp);
    scratch = nullptr;
    scratch_bytes = 0;
    if (cudaMallocAsync(&scratch, bytes, s_comp) != cudaSuccess) {
      scratch = nullptr;
      cudaGetLastError();
      saru::set_last_error("request server: scratch allocation failed");
      return SARU_E_NOMEM;
    }
    scratch_bytes = bytes;
    return SARU_OK;
  }

  // Next launch group: requests in arrival order while arena space, call
  // slots and the group cap last.  Empty only when stopping.
  std::vector<std::shared_ptr<Request>> admit() {
    std::unique_lock<std::mutex> lk(mu);
    std::vector<std::shared_ptr<Request>> grp;
    const size_t cap = cfg.pipeline ? (size_t)cfg.max_requests_per_launch : 1;
    const size_t max_inflight = cfg.pipeline ? (size_t)cfg.max_inflight : 1;
    for (;;) {
      cv_pending.wait(lk, [&] { return stop || !pending.empty(); });
      if (pending.empty()) return grp;  // stopping, queue drained
      cv_inflight.wait(lk, [&] { return inflight.size() < max_inflight; });
      size_t ncalls = 0;
      while (!pending.empty() && grp.size() < cap) {
        auto &r = pending.front();
        if (ncalls + r->calls.size() > (size_t)SARU_MAX_CALLS) break;
        const long off = arena.alloc(r->dev_bytes);
        if (off < 0) break;
        r->dev_off = off;
        r->t_admit = now_us();
        r->group = (int32_t)groups;
        ncalls += r->calls.size();
        grp.push_back(r);
        pending.pop_front();
      }
      if (!grp.empty()) {
        groups += 1;
        return grp;
      }
      // The head request waits for completed groups to free arena space.
      // Something is in flight here: a request alone always fits the empty
      // arena (submit checks it), and admitted requests hold arena space
      // until the completion thread frees it.
      const int64_t gen = free_gen;
      cv_freed.wait(lk, [&] { return free_gen != gen; });
    }
  }

  void scheduler() {
    cudaSetDevice(cfg.device);
    for (;;) {
      std::vector<std::shared_ptr<Request>> grp = admit();
      if (grp.empty()) break;
      for (auto &r : grp) stage(*r);
      cudaEvent_t in_ev = nullptr, done_ev = nullptr;
      cudaEventCreateWithFlags(&in_ev, cudaEventDisableTiming);
      cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming);
      cudaEventRecord(in_ev, s_in);
      cudaStreamWaitEvent(s_comp, in_ev, 0);
      std::vector<saru_batch> calls;
      std::vector<saru_result> res;
      std::vector<saru::CompactOut> cmp;
      for (auto &r : grp)
        for (size_t i = 0; i < r->dcalls.size(); ++i)
          if (r->dcalls[i].n > 0) {
            calls.push_back(r->dcalls[i]);
            res.push_back(r->dres[i]);
            cmp.push_back(r->dcmp[i]);
          }
      int rc = SARU_OK;
      const uint64_t l0 = saru::thread_launches();
      if (!calls.empty() && cfg.pipeline) {
        rc = ensure_scratch(saru_multi_scratch_bytes(calls.data(), (int)calls.size()));
        if (!rc)  // every call has its own status word; res[0]'s is the unused fallback
          rc = saru::align_multi_mixed(calls.data(), res.data(), cmp.data(), (int)calls.size(),
                                       res[0].status, scratch, scratch_bytes, s_comp);
      } else {
        for (size_t i = 0; i < calls.size() && !rc; ++i) {
          rc = ensure_scratch(saru_scratch_bytes(calls[i].n, calls[i].max_read_length,
                                                 calls[i].k, calls[i].k > 7));
          if (rc) break;
          rc = cmp[i].records
                   ? saru_align_device_compact(&calls[i], res[i].scores, cmp[i].records,
                                               cmp[i].rec_bytes, res[i].status, scratch,
                                               scratch_bytes, s_comp)
                   : saru_align_device(&calls[i], &res[i], scratch, scratch_bytes, s_comp);
        }
      }
      cudaEventRecord(done_ev, s_comp);
      cudaEventDestroy(in_ev);
      {
        std::lock_guard<std::mutex> lk(mu);
        launches += (int64_t)(saru::thread_launches() - l0);
        inflight.push_back(Group{grp, done_ev, rc});
      }
      cv_inflight.notify_all();
      if (!cfg.pipeline) {  // plain mode: one request's round trip at a time
        std::unique_lock<std::mutex> lk(mu);
        cv_done.wait(lk, [&] { return grp.back()->done; });
      }
    }
  }

  // Copies a group's results out, redoes flagged calls on the exact path,
  // frees its arena ranges and completes its requests.
  void completer() {
    cudaSetDevice(cfg.device);
    for (;;) {
      Group g;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_inflight.wait(lk, [&] { return !inflight.empty() || sched_done; });
        if (inflight.empty()) break;
        g = inflight.front();
      }
      cudaStreamWaitEvent(s_out, g.done_ev, 0);
      for (auto &r : g.reqs) {
        r->call_status.assign(r->calls.size(), 0);
        for (size_t i = 0; i < r->calls.size(); ++i) {
          const saru_batch &h = r->calls[i];
          if (h.n == 0) continue;
          const saru_result &d = r->dres[i], &o = r->results[i];
          cudaMemcpyAsync(o.scores, d.scores, 4 * (size_t)h.n, cudaMemcpyDeviceToHost, s_out);
          if (r->compact) {
            cudaMemcpyAsync(o.read_aln, d.read_aln, (size_t)h.n * record_bytes(h),
                            cudaMemcpyDeviceToHost, s_out);
            continue;
          }
          cudaMemcpyAsync(o.read_aln, d.read_aln, (size_t)h.total_slots, cudaMemcpyDeviceToHost,
                          s_out);
          cudaMemcpyAsync(o.genome_aln, d.genome_aln, (size_t)h.total_slots,
                          cudaMemcpyDeviceToHost, s_out);
        }
        cudaMemcpyAsync(r->call_status.data(), r->dstatus, 4 * r->calls.size(),
                        cudaMemcpyDeviceToHost, s_out);
      }
      int rc = g.rc;
      if (cudaStreamSynchronize(s_out) != cudaSuccess && rc == SARU_OK) {
        saru::set_last_error(cudaGetErrorString(cudaGetLastError()));
        rc = SARU_E_CUDA;
      }
      cudaEventDestroy(g.done_ev);
      for (auto &r : g.reqs) {
        if (r->rc == SARU_OK) r->rc = rc;
        for (size_t i = 0; i < r->calls.size() && r->rc == SARU_OK; ++i) {
          const int st = r->call_status[i];
          if (st & saru::kStatusGather) {
            saru::set_last_error("a gathered candidate lies outside the genome or read table, "
                                 "or its window length does not match its flag");
            r->rc = SARU_E_INVALID;
          } else if (st & (saru::kStatusAlphabet | saru::kStatusIrregular)) {
            // as saru_align_host does: the whole call again on the exact path
            r->rc = redo_call(*r, i);
            r->redone += 1;
          } else if (st & saru::kStatusOverflow) {
            saru::set_last_error("banded traceback left its band");
            r->rc = SARU_E_OVERFLOW;
          }
        }
      }
      const int64_t t = now_us();
      {
        std::lock_guard<std::mutex> lk(mu);
        inflight.pop_front();
        for (auto &r : g.reqs) {
          arena.free((size_t)r->dev_off, r->dev_bytes);
          r->t_done = t;
          r->done = true;
          ahead_bytes -= r->pooled;
        }
        free_gen += 1;
      }
      cv_inflight.notify_all();
      cv_freed.notify_all();
      cv_done.notify_all();
      cv_filter.notify_all();
    }
  }
};

extern "C" {

saru_server *saru_server_create(const saru_server_config *cfg) {
  if (!cfg || cfg->max_inflight < 1 || cfg->max_requests_per_launch < 1 ||
      cfg->device_budget_bytes < (1 << 20)) {
    saru::set_last_error("saru_server_create: max_inflight >= 1, max_requests_per_launch >= 1 "
                         "and device_budget_bytes >= 1 MiB");
    return nullptr;
  }
  auto *s = new saru_server();
  s->cfg = *cfg;
  s->ahead_limit = s->pool_bytes() / 2;
  if (cudaSetDevice(cfg->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->s_in, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->s_comp, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->s_out, cudaStreamNonBlocking) != cudaSuccess ||
      !s->arena.init((size_t)cfg->device_budget_bytes)) {
    saru::set_last_error(cudaGetErrorString(cudaGetLastError()));
    if (s->s_in) cudaStreamDestroy(s->s_in);
    if (s->s_comp) cudaStreamDestroy(s->s_comp);
    if (s->s_out) cudaStreamDestroy(s->s_out);
    delete s;
    return nullptr;
  }
  s->sched_thr = std::thread([s] { s->scheduler(); });
  s->done_thr = std::thread([s] { s->completer(); });
  const int nf = cfg->pipeline ? saru_server::kFilterWorkers : 1;
  for (int w = 0; w < nf; ++w) s->filter_thrs.emplace_back([s, w] { s->filterer(w); });
  return s;
}

int saru_server_submit_reads(saru_server *s, const saru_read_set *sets, int32_t nsets,
                             int32_t compact, int64_t *ticket) {
  if (!s || !sets || !ticket || nsets < 1 || nsets > 16) {
    saru::set_last_error("saru_server_submit_reads: 1..16 read sets and a ticket");
    return SARU_E_INVALID;
  }
  for (int i = 0; i < nsets; ++i) {
    const saru_read_set &rs = sets[i];
    if (rs.nreads < 0 || (rs.nreads > 0 && !rs.reads) || rs.k < 0 || rs.k > 15 ||
        rs.read_length < 2 || rs.read_length > saru::kMaxBandM) {
      saru::set_last_error("saru_server_submit_reads: every set needs reads, k <= 15 and "
                           "2 <= read_length <= 512");
      return SARU_E_INVALID;
    }
  }
  auto r = std::make_shared<Request>();
  r->gather = true;
  r->compact = compact != 0;
  r->rsets.resize((size_t)nsets);
  for (int i = 0; i < nsets; ++i) r->rsets[(size_t)i].set = sets[i];
  r->t_submit = now_us();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->genome) {
      saru::set_last_error("saru_server_submit_reads: no genome (saru_server_set_genome)");
      return SARU_E_INVALID;
    }
    if (s->stop || s->filter_stop) {
      saru::set_last_error("saru_server_submit_reads: server is shutting down");
      return SARU_E_INVALID;
    }
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->read_done[r->ticket] = r;
    s->filter_q.push_back(r);
  }
  *ticket = r->ticket;
  s->cv_filter.notify_all();
  return SARU_OK;
}

int saru_server_read_results(saru_server *s, int64_t ticket, int32_t set,
                             saru_read_results *out) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->read_done.find(ticket);
  if (it == s->read_done.end() || !it->second->done || it->second->rc != SARU_OK || set < 0 ||
      (size_t)set >= it->second->rsets.size() || !out) {
    saru::set_last_error("saru_server_read_results: not a finished reads-only request, or no "
                         "such set");
    return SARU_E_INVALID;
  }
  const ReadSetOut &o = it->second->rsets[(size_t)set];
  *out = saru_read_results{};
  out->ncalls = (int32_t)o.call_strand.size();
  out->nperfect = (int32_t)o.perfect_ids.size();
  out->n = (int64_t)o.ids.size();
  out->call_begin = o.call_begin.data();
  out->slot_begin = o.slot_begin.data();
  out->call_strand = o.call_strand.data();
  out->ids = o.ids.data();
  out->pos = o.pos.data();
  out->dirs = o.dirs.data();
  out->scores = o.scores.data();
  out->read_aln = o.ra;
  out->genome_aln = o.ga;
  out->records = o.records;
  out->record_bytes = o.rec_bytes;
  out->perfect_ids = o.perfect_ids.data();
  out->perfect_pos = o.perfect_pos.data();
  out->perfect_strand = o.perfect_strand.data();
  return SARU_OK;
}

void saru_server_release(saru_server *s, int64_t ticket) {
  if (!s) return;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->read_done.find(ticket);
  if (it != s->read_done.end() && it->second->done) {
    s->free_outputs(*it->second);
    s->read_done.erase(it);
  }
}

int saru_server_submit(saru_server *s, const saru_request *req, int64_t *ticket) {
  if (!s || !req || !ticket || req->ncalls < 1 || req->ncalls > SARU_MAX_CALLS) {
    saru::set_last_error("saru_server_submit: 1..SARU_MAX_CALLS calls and a ticket");
    return SARU_E_INVALID;
  }
  auto r = std::make_shared<Request>();
  r->compact = req->compact != 0;
  r->results.assign(req->results, req->results + req->ncalls);
  if (req->gather) {
    r->gather = true;
    r->gcalls.assign(req->gather, req->gather + req->ncalls);
    for (const auto &g : r->gcalls) r->calls.push_back(shape_of(g));
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->genome) {
      saru::set_last_error("saru_server_submit: gather request before saru_server_set_genome");
      return SARU_E_INVALID;
    }
    for (const auto &g : r->gcalls)
      if (g.nreads < 0 || g.total_slots != g.genome_bytes + (int64_t)g.k * g.n) {
        saru::set_last_error("saru_server_submit: gather call with nreads < 0 or total_slots "
                             "!= genome_bytes + k * n");
        return SARU_E_INVALID;
      }
  } else {
    r->calls.assign(req->calls, req->calls + req->ncalls);
  }
  for (const auto &b : r->calls) {
    if (b.n < 0 || b.k < 0 || b.k > 15 || b.match != 0 || b.mismatch != 1 ||
        b.max_read_length < 2 || b.max_read_length > saru::kMaxBandM) {
      saru::set_last_error("saru_server_submit: calls need unit costs, k <= 15 and "
                           "2 <= max_read_length <= 512");
      return SARU_E_INVALID;
    }
  }
  r->dev_bytes = request_bytes(*r);
  if (r->dev_bytes > s->arena.size()) {
    saru::set_last_error("saru_server_submit: request larger than the device budget");
    return SARU_E_NOMEM;
  }
  r->t_submit = now_us();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      saru::set_last_error("saru_server_submit: server is shutting down");
      return SARU_E_INVALID;
    }
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->pending.push_back(r);
  }
  *ticket = r->ticket;
  s->cv_pending.notify_all();
  return SARU_OK;
}

int saru_server_wait(saru_server *s, int64_t ticket, int32_t timeout_ms,
                     saru_request_stats *stats) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    saru::set_last_error("saru_server_wait: unknown ticket");
    return SARU_E_INVALID;
  }
  std::shared_ptr<Request> r = it->second;
  if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                           [&] { return r->done; }))
    return SARU_E_TIMEOUT;
  if (stats) {
    stats->submit_us = r->t_submit;
    stats->admit_us = r->t_admit;
    stats->done_us = r->t_done;
    stats->group = r->group;
    stats->redone_calls = r->redone;
  }
  s->tickets.erase(it);
  return r->rc;
}

int saru_server_set_genome(saru_server *s, const char *genome, int64_t genome_len) {
  if (!s || !genome || genome_len < 1) {
    saru::set_last_error("saru_server_set_genome: a genome of at least one byte");
    return SARU_E_INVALID;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->tickets.empty()) {
    saru::set_last_error("saru_server_set_genome: requests are unfinished");
    return SARU_E_INVALID;
  }
  cudaSetDevice(s->cfg.device);
  s->free_genome();
  // 2 bits a base; bytes other than A/C/G/T kept as (position, byte)
  const size_t nb = ((size_t)genome_len + 3) / 4;
  std::vector<uint8_t> packed(nb, 0);
  std::vector<int64_t> epos;
  std::vector<uint8_t> ebyte;
  for (int64_t p = 0; p < genome_len; ++p) {
    const uint8_t c = (uint8_t)genome[p];
    const int code = saru::base_code(c);
    if (code < 0) {
      epos.push_back(p);
      ebyte.push_back(c);
      continue;
    }
    packed[(size_t)(p >> 2)] |= (uint8_t)(code << (2 * (p & 3)));
  }
  const size_t ne = epos.size();
  if (cudaMalloc(&s->genome, nb + 64) != cudaSuccess ||
      (ne && (cudaMalloc(&s->exc_pos, 8 * ne) != cudaSuccess ||
              cudaMalloc(&s->exc_byte, ne) != cudaSuccess))) {
    cudaGetLastError();
    s->free_genome();
    saru::set_last_error("saru_server_set_genome: device allocation failed");
    return SARU_E_NOMEM;
  }
  if (cudaMemcpy(s->genome, packed.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      (ne && (cudaMemcpy(s->exc_pos, epos.data(), 8 * ne, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemcpy(s->exc_byte, ebyte.data(), ne, cudaMemcpyHostToDevice) != cudaSuccess))) {
    saru::set_last_error(cudaGetErrorString(cudaGetLastError()));
    s->free_genome();
    return SARU_E_CUDA;
  }
  s->pg = saru::PackedGenome{s->genome, s->exc_pos, s->exc_byte, genome_len, (int64_t)ne};
  s->genome_len = genome_len;
  s->genome_host.assign(genome, genome + genome_len);
  s->destroy_filters();  // indexes of the old genome
  cudaSetDevice(s->cfg.device);
  return SARU_OK;
}

void saru_server_counters(saru_server *s, int64_t *groups, int64_t *launches) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (groups) *groups = s->groups;
  if (launches) *launches = s->launches;
}

void saru_server_destroy(saru_server *s) {
  if (!s) return;
  {  // the filter thread first: what it has queued goes to the scheduler
    std::lock_guard<std::mutex> lk(s->mu);
    s->filter_stop = true;
  }
  s->cv_filter.notify_all();
  for (auto &t : s->filter_thrs)
    if (t.joinable()) t.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_pending.notify_all();
  if (s->sched_thr.joinable()) s->sched_thr.join();  // drains the pending queue first
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->sched_done = true;
  }
  s->cv_inflight.notify_all();
  if (s->done_thr.joinable()) s->done_thr.join();
  cudaSetDevice(s->cfg.device);
  if (s->scratch) cudaFreeAsync(s->scratch, s->s_comp);
  cudaStreamSynchronize(s->s_comp);
  s->free_genome();
  s->destroy_filters();
  cudaSetDevice(s->cfg.device);
  s->arena.release();
  cudaStreamDestroy(s->s_in);
  cudaStreamDestroy(s->s_comp);
  cudaStreamDestroy(s->s_out);
  delete s;
}

}  // extern "C"
