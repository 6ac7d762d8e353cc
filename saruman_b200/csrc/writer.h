// writer.h -- the reference's TSV writer over host result arrays.
#pragma once
#include <stdint.h>

#include <string>

namespace saru {

// One aligned call, host memory.
struct WriterCall {
  const int32_t *scores;
  const char *read_aln;
  const char *genome_aln;
  int64_t total_slots;
  const int32_t *goff;
  const int32_t *pos;
  const int8_t *dirs;
  const int32_t *ids;
  int32_t k;
  int32_t read_length;
  const char *(*name_of)(void *ctx, int32_t id);
  void *name_ctx;
  // read_aln/genome_aln hold slot bytes [window_lo, window_hi) of the call
  // (window_hi < 0: the whole call, [0, total_slots)); the writer's scans
  // never leave the window when it covers the slots they reach
  int64_t window_lo = 0;
  int64_t window_hi = -1;
};

struct LineFields {
  const char *name;
  int64_t name_len;
  int start, stop, score;
  int64_t from, len_read, len_genome;
  bool reverse;
  int64_t bytes;  // upper bound of the line length
};

bool line_fields(const WriterCall &w, int64_t v, LineFields *f);
int64_t line_write(const WriterCall &w, const LineFields &f, char *out);
// Appends the lines of candidates [begin, end) to `out`.
void format_range(const WriterCall &w, int64_t begin, int64_t end, std::string *out,
                  int32_t *done_fwd, int32_t *done_rev);

}  // namespace saru
