// sam.cpp -- SAM records from the reference writer's TSV lines.
//
// The reference prints one line per alignment (src/cuda-functions.cu:987):
// name, start, stop, strand (">>" forward, "<<" reverse), the aligned read
// string, the aligned genome string (gaps as '_'), the edit distance;
// perfect hits come from the filter in the same layout (src/hash.c:580),
// unmapped reads as name, '*', '*', strand, read, '*', length
// (src/hash.c:821).  The reference's README points to an external script
// for SAM (README.md:32); this converter writes, per line:
//   QNAME  the name up to the first blank ('*' if none)
//   FLAG   16 for '<<', 0 for '>>', 4 for an unmapped line
//   RNAME  the reference name given to the converter
//   POS    start (1-based, as printed)
//   MAPQ   255 (not computed)
//   CIGAR  run-length of the columns: M (bytes in both strings), I ('_' in
//          the genome string), D ('_' in the read string)
//   SEQ    the read string without gaps ('*' if empty)
//   QUAL   '*'
//   NM:i   the printed edit distance
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/saruman_b200.h"
#include "server_internal.h"

namespace {

struct Field {
  const char *p;
  size_t n;
};

// Splits a line (without its newline) at tabs into up to `max` fields.
size_t split_tabs(const char *p, size_t n, Field *f, size_t max) {
  size_t k = 0, start = 0;
  for (size_t i = 0; i <= n && k < max; ++i) {
    if (i == n || p[i] == '\t') {
      f[k++] = Field{p + start, i - start};
      start = i + 1;
    }
  }
  return k;
}

void put(std::string &o, const Field &f) { o.append(f.p, f.n); }

// The whitespace Python's str.split() and str.strip() drop, in ASCII.
bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f' ||
         (c >= '\x1c' && c <= '\x1f');
}

// One SAM record for a TSV line; false if the line has fewer than 7 fields.
bool record(const char *p, size_t n, const char *rname, std::string &o) {
  Field f[8];
  if (split_tabs(p, n, f, 8) < 7) return false;
  // QNAME: the name up to the first blank (Python's str.split semantics:
  // leading blanks skipped, '*' if nothing is left)
  size_t a = 0;
  while (a < f[0].n && is_space(f[0].p[a])) ++a;
  size_t b = a;
  while (b < f[0].n && !is_space(f[0].p[b])) ++b;
  if (b > a) o.append(f[0].p + a, b - a);
  else o.push_back('*');
  if (f[1].n == 1 && f[1].p[0] == '*') {  // unmapped read
    o.append("\t4\t*\t0\t0\t*\t*\t0\t0\t");
    put(o, f[4]);
    o.append("\t*\n");
    return true;
  }
  const bool rev = f[3].n == 2 && f[3].p[0] == '<' && f[3].p[1] == '<';
  o.append(rev ? "\t16\t" : "\t0\t");
  o.append(rname);
  o.push_back('\t');
  put(o, f[1]);
  o.append("\t255\t");
  const Field &ra = f[4], &ga = f[5];
  const size_t cols = ra.n < ga.n ? ra.n : ga.n;
  char prev = 0;
  size_t run = 0;
  auto flush = [&] {
    if (run) {
      o.append(std::to_string(run));
      o.push_back(prev);
    }
  };
  for (size_t i = 0; i < cols; ++i) {
    const char op = ra.p[i] == '_' ? 'D' : (ga.p[i] == '_' ? 'I' : 'M');
    if (op != prev) {
      flush();
      prev = op;
      run = 0;
    }
    ++run;
  }
  flush();
  o.append("\t*\t0\t0\t");
  const size_t before = o.size();
  for (size_t i = 0; i < ra.n; ++i)
    if (ra.p[i] != '_') o.push_back(ra.p[i]);
  if (o.size() == before) o.push_back('*');
  o.append("\t*\tNM:i:");
  put(o, f[6]);
  o.push_back('\n');
  return true;
}

}  // namespace

extern "C" {

int64_t saru_tsv_to_sam(const char *tsv, int64_t len, const char *rname, int64_t rlen,
                        char *out, int64_t cap) {
  if (!tsv || len < 0 || !rname || rlen < 0 || cap < 0 || (cap > 0 && !out)) {
    saru::set_last_error("saru_tsv_to_sam: TSV bytes, a reference name and length, an output");
    return -1;
  }
  std::string o;
  o.reserve((size_t)len + 256);
  o.append("@HD\tVN:1.6\tSO:unsorted\n@SQ\tSN:");
  o.append(rname);
  o.append("\tLN:" + std::to_string(rlen) + "\n@PG\tID:saruman_b200\tPN:saruman_b200\n");
  size_t i = 0;
  const size_t n = (size_t)len;
  while (i < n) {
    size_t e = i;
    while (e < n && tsv[e] != '\n') ++e;
    bool blank = true;  // lines of whitespace only are skipped
    for (size_t j = i; j < e && blank; ++j) blank = is_space(tsv[j]);
    if (!blank && !record(tsv + i, e - i, rname, o)) {
      saru::set_last_error("saru_tsv_to_sam: a line with fewer than 7 tab-separated fields");
      return -1;
    }
    i = e + 1;
  }
  if (out && cap > 0) memcpy(out, o.data(), o.size() < (size_t)cap ? o.size() : (size_t)cap);
  return (int64_t)o.size();
}

}  // extern "C"
