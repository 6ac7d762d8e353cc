// Host run of the q-gram pair filter (saruman_b200/csrc/filter_core.cuh)
// with the reference's own data layout: a q-gram index built with a plain
// map, the data array of each read chunk built literally (lists in q-gram
// order per read, each ended by a 0), then the call assembly of
// filter_calls.h.  Compared with the calls the reference program itself
// submits (tests/test_filter_host.py).  Test infrastructure only.
#include <stdint.h>
#include <string.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../saruman_b200/csrc/filter_calls.h"

using namespace saru;

static uint8_t comp(uint8_t c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return c;
  }
}

// The genome may be a chunk of a larger one: `offset` is the genome
// position of its first byte, `limit` the position windows must end by.
extern "C" int filter_host_calls_chunk(const uint8_t *genome, long glen, long offset, long limit,
                                       const uint8_t *reads, int nreads, int m, int k, int dr,
                                       int chunksize, unsigned chunk_value, int cap,
                                       int64_t *call_begin, int64_t cb_cap, int32_t *ids,
                                       int32_t *pos, int8_t *dirs, int64_t cand_cap,
                                       int32_t *pids, int32_t *ppos, int64_t pcap,
                                       int64_t *counts) {
  FilterShape S;
  if (!filter_shape(m, k, &S)) return -1;
  std::unordered_map<std::string, std::vector<uint32_t>> index;
  for (long p = 0; p + S.q <= glen; ++p)
    index[std::string((const char *)genome + p, (size_t)S.q)].push_back((uint32_t)(p + offset));
  CallAssembler asmb(m, k, limit, chunk_value);
  std::vector<int32_t> hp((size_t)cap);
  std::vector<int8_t> hf((size_t)cap);
  int overflow = 0;
  for (int run = 0; run * chunksize < nreads; ++run) {
    const int r0 = run * chunksize, r1 = std::min(nreads, r0 + chunksize);
    std::vector<uint32_t> data;
    std::vector<size_t> offs((size_t)(r1 - r0) * S.P), lens((size_t)(r1 - r0) * S.P);
    std::vector<std::string> strand((size_t)(r1 - r0));
    for (int r = r0; r < r1; ++r) {
      std::string rd((const char *)reads + (size_t)r * m, (size_t)m);
      if (dr == 4) {
        std::string rc(rd.rbegin(), rd.rend());
        for (auto &c : rc) c = (char)comp((uint8_t)c);
        rd = rc;
      }
      strand[(size_t)(r - r0)] = rd;
      for (int x = 0; x < S.P; ++x) {
        offs[(size_t)(r - r0) * S.P + x] = data.size();
        auto it = index.find(rd.substr((size_t)S.qpos[x], (size_t)S.q));
        if (it != index.end()) data.insert(data.end(), it->second.begin(), it->second.end());
        lens[(size_t)(r - r0) * S.P + x] = it != index.end() ? it->second.size() : 0;
        data.push_back(0);
      }
    }
    for (int r = r0; r < r1; ++r) {
      const size_t base = (size_t)(r - r0) * S.P;
      struct Lists {
        const std::vector<uint32_t> *data;
        const size_t *offs, *lens;
        uint32_t len(int x) const { return (uint32_t)lens[x]; }
        uint32_t at(int x, uint32_t i) const {
          const size_t j = offs[x] + i;
          return j < data->size() ? (*data)[j] : 0u;
        }
        int find(int x, uint32_t lo, uint32_t want) const {
          for (uint32_t i = lo; i < lens[x]; ++i)  // literal scan: the checker
            if ((*data)[offs[x] + i] == want) return (int)i;
          return -1;
        }
      } lists{&data, &offs[base], &lens[base]};
      const std::string &rd = strand[(size_t)(r - r0)];
      auto perfect = [&](int g1) {
        const long l1 = (long)g1 - offset;
        return l1 + m <= glen && memcmp(genome + l1, rd.data(), (size_t)m) == 0;
      };
      ReadHits h{hp.data(), hf.data(), cap, 0, 0, 0};
      filter_read(S, dr, lists, perfect, h, (int)offset);
      overflow |= h.overflow;
      asmb.add_read(r, h.pos, h.flag, h.n, h.queue);
    }
  }
  asmb.finish();
  const FilterCalls &o = asmb.out;
  counts[0] = (int64_t)o.call_begin.size() - 1;
  counts[1] = (int64_t)o.ids.size();
  counts[2] = (int64_t)o.perfect_ids.size();
  if ((int64_t)o.call_begin.size() > cb_cap || (int64_t)o.ids.size() > cand_cap ||
      (int64_t)o.perfect_ids.size() > pcap)
    return -2;
  memcpy(call_begin, o.call_begin.data(), o.call_begin.size() * 8);
  memcpy(ids, o.ids.data(), o.ids.size() * 4);
  memcpy(pos, o.pos.data(), o.pos.size() * 4);
  memcpy(dirs, o.dirs.data(), o.dirs.size());
  memcpy(pids, o.perfect_ids.data(), o.perfect_ids.size() * 4);
  memcpy(ppos, o.perfect_pos.data(), o.perfect_pos.size() * 4);
  return overflow ? 1 : 0;
}

extern "C" int filter_host_calls(const uint8_t *genome, long glen, const uint8_t *reads,
                                 int nreads, int m, int k, int dr, int chunksize,
                                 unsigned chunk_value, int cap, int64_t *call_begin,
                                 int64_t cb_cap, int32_t *ids, int32_t *pos, int8_t *dirs,
                                 int64_t cand_cap, int32_t *pids, int32_t *ppos, int64_t pcap,
                                 int64_t *counts) {
  return filter_host_calls_chunk(genome, glen, 0, glen, reads, nreads, m, k, dr, chunksize,
                                 chunk_value, cap, call_begin, cb_cap, ids, pos, dirs, cand_cap,
                                 pids, ppos, pcap, counts);
}
