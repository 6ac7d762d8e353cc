// input.cpp -- the reference's input readers (host code): reads from a
// FASTA or FASTQ file in batches, the genome from a FASTA file in chunks
// with an overhang.
//
// What the alignment stage sees is decided here: which reads exist (short
// reads and reads with more Ns than the error count are dropped), their
// names and ids, the genome bytes of each chunk and the limit that windows
// must end by.  Both readers follow the reference's steps, quirks included,
// because the reference's output depends on them:
//
//  reads (src/util.c:294-452): records of two lines (FASTA) or four
//    (FASTQ), each line read with fgets into a buffer of fixed size: the
//    name line into 60 bytes, the sequence and quality lines into
//    read_length + 2; a longer line is split, and its rest read as the next
//    line, exactly as fgets does.  A sequence is cut at read_length and
//    upper-cased; shorter than read_length: dropped; more than max_n Ns:
//    dropped; otherwise kept, its name being the name line without its
//    first byte (the '>' or '@') and its last byte (the newline).  A batch
//    is up to max_entries records (kept or dropped); read ids restart at 0
//    in each batch.
//  genome (src/saruman.c:139-271): a chunk is chunk_value bases followed by
//    an overhang of read_length bases, taken from the file read through a
//    buffer of chunk_value + read_length bytes: newlines are dropped, every
//    other byte is kept upper-cased (a later '>' header line or a '\r'
//    included); the first chunk skips the first line.  Bases the buffer
//    does not hold are read one byte at a time; a one-byte read that fails
//    at the end of the file still keeps the byte left at the buffer's start
//    (unless it is a newline), so a genome that ends inside a chunk gains
//    one trailing byte.  The next chunk starts where the chunk's own bases
//    ended in the file (before the overhang), first taking what is left of
//    the buffer.  Chunks continue while the last one filled its chunk_value
//    bases.
#include <ctype.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/saruman_b200.h"
#include "server_internal.h"

namespace {

constexpr int kNameLine = 60;  // the reference's name buffer (and name slot) size

// fgets into a buffer of `size` bytes: up to size - 1 bytes, through the
// first newline; false (buffer untouched) at the end of the file.
bool get_line(FILE *f, char *buf, int size) {
  int n = 0;
  while (n < size - 1) {
    const int c = fgetc(f);
    if (c == EOF) break;
    buf[n++] = (char)c;
    if (c == '\n') break;
  }
  if (n == 0) return false;
  buf[n] = '\0';
  return true;
}

}  // namespace

struct saru_reads {
  FILE *f = nullptr;
  int fastq = 0, m = 0, max_n = 0;
  std::vector<char> name, seq, qname, qual;
  bool done = false;
};

struct saru_genome_reader {
  FILE *f = nullptr;
  long chunk = 0;
  int m = 0;
  std::vector<char> buffer;  // chunk + m bytes, as the reference's read buffer
  size_t buffer_read = 0;    // bytes the last whole-buffer read returned
  size_t buffer_pos = 0;     // where the last chunk stopped taking from the buffer
  long file_pos = 0;         // where the next chunk continues in the file
  bool first = true, done = false;
  int64_t total = 0;         // bases read so far, overhangs excluded
  int run = 0;
};

extern "C" {

saru_reads *saru_reads_open(const char *path, int32_t fastq, int32_t read_length, int32_t max_n) {
  saru::set_last_error("");
  if (!path || read_length < 1 || max_n < 0) {
    saru::set_last_error("saru_reads_open: a path, read_length >= 1, max_n >= 0");
    return nullptr;
  }
  FILE *f = fopen(path, "rb");
  if (!f) {
    saru::set_last_error((std::string("saru_reads_open: cannot open ") + path).c_str());
    return nullptr;
  }
  auto *r = new saru_reads();
  r->f = f;
  r->fastq = fastq ? 1 : 0;
  r->m = read_length;
  r->max_n = max_n;
  r->name.assign(kNameLine, '\0');
  r->seq.assign((size_t)read_length + 2, '\0');
  r->qname.assign(kNameLine, '\0');
  r->qual.assign((size_t)read_length + 2, '\0');
  return r;
}

int32_t saru_reads_next(saru_reads *r, int32_t max_entries, char *reads, char *names,
                        int32_t *skipped) {
  saru::set_last_error("");
  if (!r || max_entries < 1 || !reads || !names) {
    saru::set_last_error("saru_reads_next: a reader, max_entries >= 1 and output buffers");
    return -1;
  }
  const int m = r->m;
  int kept = 0, dropped = 0, records = 0;
  while (!r->done && records < max_entries) {
    if (!get_line(r->f, r->name.data(), kNameLine)) {
      r->done = true;
      break;
    }
    // a missing line leaves its buffer as it was, as fgets does
    get_line(r->f, r->seq.data(), m + 2);
    if (r->fastq) {
      get_line(r->f, r->qname.data(), kNameLine);
      get_line(r->f, r->qual.data(), m + 2);
    }
    ++records;
    char *seq = r->seq.data();
    seq[m] = '\0';
    char *nm = r->name.data();
    const size_t len = strlen(nm);
    if (len > 0) nm[len - 1] = '\0';  // the last byte (the newline) goes
    int ns = 0;
    for (int i = 0; i < m; ++i) {
      seq[i] = (char)toupper((unsigned char)seq[i]);
      if (seq[i] == 'N') ++ns;
    }
    if ((int)strlen(seq) < m || ns > r->max_n) {
      ++dropped;
      continue;
    }
    memcpy(reads + (size_t)kept * m, seq, (size_t)m);
    char *slot = names + (size_t)kept * kNameLine;
    memset(slot, 0, kNameLine);
    if (len > 1) memcpy(slot, nm + 1, strlen(nm + 1));  // at most 58 bytes
    ++kept;
  }
  if (skipped) *skipped = dropped;
  return kept;
}

void saru_reads_close(saru_reads *r) {
  if (!r) return;
  if (r->f) fclose(r->f);
  delete r;
}

saru_genome_reader *saru_genome_open(const char *path, int64_t chunk_value, int32_t read_length) {
  saru::set_last_error("");
  if (!path || chunk_value < 1 || read_length < 1 || chunk_value > (1LL << 31)) {
    saru::set_last_error("saru_genome_open: a path, 1 <= chunk_value <= 2^31, read_length >= 1");
    return nullptr;
  }
  FILE *f = fopen(path, "rb");
  if (!f) {
    saru::set_last_error((std::string("saru_genome_open: cannot open ") + path).c_str());
    return nullptr;
  }
  auto *g = new saru_genome_reader();
  g->f = f;
  g->chunk = (long)chunk_value;
  g->m = read_length;
  g->buffer.assign((size_t)(chunk_value + read_length), '\0');
  return g;
}

int32_t saru_genome_next(saru_genome_reader *g, char *out, int64_t *len, int64_t *bases,
                         int64_t *total) {
  saru::set_last_error("");
  if (!g || !out || !len) {
    saru::set_last_error("saru_genome_next: a reader and an output of chunk + read_length bytes");
    return -1;
  }
  if (g->done) return 0;
  const size_t cap = g->buffer.size();
  char *buf = g->buffer.data();
  long n = 0;  // bytes of this chunk
  auto keep = [&](char c) {
    if (c != '\n') out[n++] = (char)toupper((unsigned char)c);
    return c != '\n';
  };
  if (!g->first) {
    fseek(g->f, g->file_pos, SEEK_SET);
    // what the last chunk left of the buffer comes first
    if (g->buffer_pos < cap)
      for (size_t p = g->buffer_pos; n < g->chunk && p < g->buffer_read; ++p) keep(buf[p]);
  }
  g->buffer_read = fread(buf, 1, cap, g->f);
  size_t p = 0;
  if (g->first)  // the first line is the header (up to a newline or a 0 byte)
    while (p < g->buffer_read && buf[p] != '\n' && buf[p] != '\0') ++p;
  for (; n < g->chunk && p < g->buffer_read; ++p) keep(buf[p]);
  g->buffer_pos = p;
  g->first = false;
  bool more = true;
  while (n < g->chunk && more) {  // the chunk's rest, a byte at a time
    more = fread(buf, 1, 1, g->f) == 1;
    keep(buf[0]);  // at the end of the file: the byte left there
  }
  const long own = n;
  g->total += own;
  g->file_pos = ftell(g->f);
  for (int over = 0; over < g->m && more;) {  // the overhang
    more = fread(buf, 1, 1, g->f) == 1;
    if (keep(buf[0])) ++over;
  }
  out[n] = '\0';
  *len = n;
  if (bases) *bases = own;
  if (total) *total = g->total;
  ++g->run;
  if (own < g->chunk) g->done = true;  // the reference's loop: while the chunk filled
  return 1;
}

void saru_genome_close(saru_genome_reader *g) {
  if (!g) return;
  if (g->f) fclose(g->f);
  delete g;
}

}  // extern "C"
