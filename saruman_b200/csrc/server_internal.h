// Hooks abi.cu gives the request server.
#pragma once
#include <stdint.h>

#include "../../include/saruman_b200.h"

namespace saru {
// Compact records of a call instead of its slot strings (records == nullptr:
// slot strings).
struct CompactOut {
  uint8_t *records;
  long rec_bytes;
};
// saru_align_multi_device with, per call, compact records or slot strings
// (the same checks are the caller's)
int align_multi_mixed(const saru_batch *calls, const saru_result *results,
                      const CompactOut *cmp, int32_t ncalls, int32_t *status, void *scratch,
                      size_t scratch_bytes, void *stream);
// kernel launches enqueued by the calling thread so far
uint64_t thread_launches();
// counts a kernel launch made outside abi.cu
void count_launch();
void set_last_error(const char *msg);
// aligns a host call as saru_align_host does, on the server's own lane
int redo_on_host_path(const saru_batch *b, saru_result *r);
// A genome resident on the device 2 bits a base, with its non-ACGT bytes as
// exceptions (gather.cu).
struct PackedGenome {
  const uint8_t *packed = nullptr;     // (len + 3) / 4 bytes
  const int64_t *exc_pos = nullptr;    // ascending genome positions
  const uint8_t *exc_byte = nullptr;
  int64_t len = 0, nexc = 0;
};
// saru_gather_device over a packed resident genome
int gather_packed(const saru_gather_call *c, const PackedGenome &g, char *windows, char *reads,
                  int32_t *read_offsets, int32_t *status, saru_batch *batch, void *stream);
// compact records of a host call from its slot strings (compact.cpp)
int records_from_slots(const saru_batch *b, const int32_t *scores, const char *read_aln,
                       const char *genome_aln, uint8_t *records, long record_bytes);
}  // namespace saru
