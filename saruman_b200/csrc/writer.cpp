// writer.cpp -- the reference's TSV output for one aligned call.
//
// Reproduces src/cuda-functions.cu:827-1006 byte for byte from the scores
// and the two alignment-slot arrays: for each candidate whose score is <= k
//   start  = genome position + number of leading '_' in the read string
//   stop_correction = number of '_' in the run of '_'/NUL that ends the slot
//   a forward scan from the first non-gap byte counts '_' in the read
//     (deletions) and in the window string (insertions) until a NUL, its
//     bound growing by one per gap (z in the reference)
//   chars  = (scan position of the NUL) - stop_correction, or
//            read_length + deletions when no NUL was met
//   line   = name, start, chars - insertions + start - 1, ">>" or "<<",
//            both strings cut at chars bytes (or their NUL), score
// with the reference's integer types (unsigned short counters, short chars,
// unsigned positions printed with %d).  Bytes past the end of the arrays
// read as 0; callers allocate the arrays with zeroed slack.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "writer.h"

namespace saru {

static inline char *put_int(char *p, int v) {
  char tmp[12];
  int n = 0;
  unsigned int u = v < 0 ? 0u - (unsigned int)v : (unsigned int)v;
  do {
    tmp[n++] = char('0' + u % 10u);
    u /= 10u;
  } while (u);
  if (v < 0) *p++ = '-';
  while (n) *p++ = tmp[--n];
  return p;
}

// Byte i of a slot array: 0 outside the call (the reference's memset
// arena), a[i - lo] inside the window the caller holds.
struct ByteView {
  const char *a;  // byte lo
  int64_t lo;
  uint64_t len;   // the window clipped to the call: [lo, lo + len)
  inline char operator[](int64_t i) const {
    return (uint64_t)(i - lo) < len ? a[i - lo] : 0;
  }
  // Bytes from i up to (not including) the first 0 byte, at most `limit`
  // (limit < 0: no limit); bytes outside the window read as 0.
  inline int64_t run_to_nul(int64_t i, int64_t limit) const {
    const uint64_t off = (uint64_t)(i - lo);
    if (off >= len) return 0;
    uint64_t room = len - off;
    if (limit >= 0 && (uint64_t)limit < room) room = (uint64_t)limit;
    const void *z = memchr(a + off, 0, (size_t)room);
    return z ? (int64_t)(static_cast<const char *>(z) - (a + off)) : (int64_t)room;
  }
  // Byte i's address; valid for bytes inside the window (run_to_nul
  // counted them there).
  inline const char *ptr(int64_t i) const { return a + (i - lo); }
  // Copies bytes [i, i + n) to out; the caller has checked they are
  // inside the window (run_to_nul counted them there).
  inline char *copy(char *out, int64_t i, int64_t n) const {
    memcpy(out, a + (i - lo), (size_t)n);
    return out + n;
  }
};

static inline ByteView view(const WriterCall &w, const char *a) {
  int64_t lo = w.window_lo, hi = w.window_hi < 0 ? w.total_slots : w.window_hi;
  if (hi > w.total_slots) hi = w.total_slots;
  const char *base = a;
  if (lo < 0) {  // the call starts at 0: bytes before it read as 0
    base -= lo;
    lo = 0;
  }
  return ByteView{base, lo, (uint64_t)(hi > lo ? hi - lo : 0)};
}

// Computes the fields of candidate v's line.  Returns false if the
// candidate prints nothing (score > k).
bool line_fields(const WriterCall &w, int64_t v, LineFields *f) {
  if (w.scores[v] > w.k) return false;
  const ByteView ra = view(w, w.read_aln), ga = view(w, w.genome_aln);
  unsigned short L;
  int64_t gs, eb = 0;
  if (v > 0) {
    L = (unsigned short)(w.goff[v] - w.goff[v - 1]);
    gs = w.goff[v - 1];
    eb = (int64_t)w.k * v;
  } else {
    L = (unsigned short)w.goff[0];
    gs = 0;
  }
  const int64_t slot = gs + eb;
  unsigned int start = (unsigned int)w.pos[v];
  unsigned short start_corr = 0, stop_corr = 0, deletion = 0, insertion = 0;
  for (int64_t i = 0; ra[slot + i] == '_'; ++i) {
    start++;
    start_corr++;
  }
  for (int64_t i = slot + L + w.k - 1; i >= -1; --i) {
    const char ch = ra[i];
    if (ch != '_' && ch != 0) break;
    if (ch == '_') stop_corr++;
  }
  // The forward scan reads position i (from the first non-gap byte) while
  // i < L - stop_corr - start_corr + z, z being the gaps met so far, and
  // stops at a 0 byte (end_of_read).  z only grows, so every position below
  // the bound known when a stretch starts is read: a stretch is counted at
  // once and the bound moves by the gaps it held.
  const int64_t p0 = slot + start_corr, base = (int64_t)L - stop_corr - start_corr;
  int64_t i = 0, z = 0;
  short end_of_read = 0;
  while (i < base + z) {
    const int64_t want = base + z - i;
    const int64_t run = ra.run_to_nul(p0 + i, want);  // bytes before a 0 (or the window's end)
    unsigned int dl = 0, in = 0;
    if (run > 0) {
      const char *rp = ra.ptr(p0 + i), *gp = ga.ptr(p0 + i);
      for (int64_t q = 0; q < run; ++q) {
        const unsigned int gr = rp[q] == '_';
        dl += gr;
        in += (gr ^ 1u) & (unsigned int)(gp[q] == '_');
      }
    }
    deletion = (unsigned short)(deletion + dl);
    insertion = (unsigned short)(insertion + in);
    z += dl + in;
    i += run;
    if (run < want) {  // a 0 byte at position i
      end_of_read = (short)i;
      break;
    }
  }
  const short chars =
      end_of_read > 0 ? (short)(end_of_read - stop_corr) : (short)(w.read_length + deletion);
  const char *name = w.name_of ? w.name_of(w.name_ctx, w.ids[v]) : "";
  if (!name) name = "";
  f->name = name;
  f->name_len = (int64_t)strlen(name);
  f->start = (int)start;
  f->stop = (int)((unsigned int)(chars - insertion) + start - 1u);
  f->from = slot + start_corr;
  // "%.*s": up to chars bytes, or to the NUL (a negative precision is no limit)
  const int64_t la = ra.run_to_nul(f->from, chars), lb = ga.run_to_nul(f->from, chars);
  f->len_read = la;
  f->len_genome = lb;
  f->reverse = w.dirs[v] > 3;
  f->score = w.scores[v];
  f->bytes = f->name_len + la + lb + 3 * 12 + 8;
  return true;
}

// Writes a line computed by line_fields; `out` has f.bytes of room.
// Returns the bytes written.
int64_t line_write(const WriterCall &w, const LineFields &f, char *out) {
  const ByteView ra = view(w, w.read_aln), ga = view(w, w.genome_aln);
  char *p = out;
  memcpy(p, f.name, (size_t)f.name_len);
  p += f.name_len;
  *p++ = '\t';
  p = put_int(p, f.start);
  *p++ = '\t';
  p = put_int(p, f.stop);
  memcpy(p, f.reverse ? "\t<<\t" : "\t>>\t", 4);
  p += 4;
  p = ra.copy(p, f.from, f.len_read);
  *p++ = '\t';
  p = ga.copy(p, f.from, f.len_genome);
  *p++ = '\t';
  p = put_int(p, f.score);
  *p++ = '\n';
  return p - out;
}

void format_range(const WriterCall &w, int64_t begin, int64_t end, std::string *out,
                  int32_t *done_fwd, int32_t *done_rev) {
  LineFields f;
  std::vector<char> line;
  for (int64_t v = begin; v < end; ++v) {
    if (!line_fields(w, v, &f)) continue;
    if ((int64_t)line.size() < f.bytes) line.resize((size_t)f.bytes * 2);
    const int64_t n = line_write(w, f, line.data());
    out->append(line.data(), (size_t)n);
    if (f.reverse) {
      if (done_rev) ++*done_rev;
    } else if (done_fwd) {
      ++*done_fwd;
    }
  }
}

}  // namespace saru
