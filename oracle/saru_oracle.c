/*
 * saru_oracle.c -- host C restatement of SARUMAN's alignment stage.
 *
 * TEST INFRASTRUCTURE, NOT THE PRODUCT (see saru_oracle.h).  Written from
 * the recurrences of the reference, with each rule citing where the
 * reference states it.
 *
 * Notation: candidate t has read r (m bytes), window g (L bytes), flank
 * offsets so/eo in {0,k} chosen by its direction flag, and an (L+1) x (m+1)
 * matrix D of int16 stored row-major (row = window position, column = read
 * position) at absolute cell index eoff[t] of a virtual arena that holds all
 * matrices of the call back to back, as the reference's arena does.
 */
#define _POSIX_C_SOURCE 200809L
#include "saru_oracle.h"

#include <limits.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int match, mis, k, n;
  const char *g, *r;
  long glen, rlen;
  const int *go, *ro, *eo;
  const signed char *dirs;
  long total_slots;
  long total_cells;
  int *scores;
  char *ra, *ga;
} batch_t;

static inline long gstart(const batch_t *b, long t) { return t ? b->go[t - 1] : 0; }
static inline long rstart(const batch_t *b, long t) { return t ? b->ro[t - 1] : 0; }
static inline long glen_of(const batch_t *b, long t) { return b->go[t] - gstart(b, t); }
static inline long rlen_of(const batch_t *b, long t) { return b->ro[t] - rstart(b, t); }
static inline long cells_of(const batch_t *b, long t) {
  return (rlen_of(b, t) + 1) * (glen_of(b, t) + 1);
}

/* Flank offsets of a direction flag (src/cuda-functions.cu:380-410):
 * 1/5 free end gap, 2/6 free start gap, 3/7 both; 0/4 (perfect hits) none. */
static void flank(int dir, int k, int *so, int *eo) {
  *so = 0;
  *eo = 0;
  switch (dir) {
    case 1: case 5: *eo = k; break;
    case 2: case 6: *so = k; break;
    case 3: case 7: *so = k; *eo = k; break;
    default: break;
  }
}

static inline short min3s(short a, short b, short c) {
  short x = a;
  if (x > b) x = b;
  if (x > c) x = c;
  return x;
}

/* The full-rectangle fill, int16 arithmetic as in the reference.
 *  row 0:    D[0][j] = j                                   (:413-416)
 *  column 0: D[i][0] = D[i-1][0] (+1 once i >= 2*so+1)     (:419-439)
 *  interior: D[i+1][j+1] = min(D[i][j] + (g[i]!=r[j] ? mis : mat),
 *                               D[i+1][j] + mis,
 *                               D[i][j+1] + mis - corr)    (:444-491)
 *  with corr = mis on the last read column for rows i >= L - 2*eo (free
 *  trailing gaps, :449-455). */
static void fill(const batch_t *b, long t, short *M) {
  long m = rlen_of(b, t), L = glen_of(b, t), W = m + 1;
  const char *g = b->g + gstart(b, t), *r = b->r + rstart(b, t);
  int so, eo;
  flank(b->dirs[t], b->k, &so, &eo);
  for (long j = 0; j <= m; ++j) M[j] = (short)j;
  for (long i = 1; i <= L; ++i)
    M[i * W] = (short)(i < 2 * so + 1 ? M[(i - 1) * W] : M[(i - 1) * W] + 1);
  for (long i = 0; i < L; ++i) {
    const short *up = M + i * W;
    short *cur = M + (i + 1) * W;
    for (long j = 0; j < m; ++j) {
      int corr = (j == m - 1 && i >= L - 2 * eo) ? b->mis : 0;
      short d = (short)(up[j] + (g[i] != r[j] ? b->mis : b->match));
      short l = (short)(cur[j] + b->mis);
      short u = (short)(up[j + 1] + b->mis - corr);
      cur[j + 1] = min3s(d, l, u);
    }
  }
}

/* A small cache of filled matrices; tracebacks only ever move to lower
 * absolute cells, so round-robin reuse is safe. */
#define NCACHE 4
typedef struct {
  long t[NCACHE];
  short *M[NCACHE];
  long cap[NCACHE];
  int next;
} cache_t;

static void cache_init(cache_t *c) {
  for (int i = 0; i < NCACHE; ++i) {
    c->t[i] = -1;
    c->M[i] = NULL;
    c->cap[i] = 0;
  }
  c->next = 0;
}

static void cache_free(cache_t *c) {
  for (int i = 0; i < NCACHE; ++i) free(c->M[i]);
}

static short *matrix(const batch_t *b, cache_t *c, long t) {
  for (int i = 0; i < NCACHE; ++i)
    if (c->t[i] == t) return c->M[i];
  int s = c->next;
  c->next = (c->next + 1) % NCACHE;
  long need = cells_of(b, t);
  if (c->cap[s] < need) {
    free(c->M[s]);
    c->M[s] = (short *)malloc(sizeof(short) * (size_t)need);
    if (!c->M[s]) {
      fprintf(stderr, "saru_oracle: out of memory\n");
      abort();
    }
    c->cap[s] = need;
  }
  fill(b, t, c->M[s]);
  c->t[s] = t;
  return c->M[s];
}

/* value of absolute arena cell P */
static short cell(const batch_t *b, cache_t *c, long P) {
  long lo = 0, hi = b->n - 1;
  while (lo < hi) {
    long mid = (lo + hi + 1) / 2;
    if (b->eo[mid] <= P) lo = mid;
    else hi = mid - 1;
  }
  return matrix(b, c, lo)[P - b->eo[lo]];
}

/* Traceback of candidate t, as src/cuda-functions.cu:108-315 states it.
 * P is an absolute arena index and the loop runs while P >= m+1, so the
 * first candidate of a call stops on row 0 while later ones keep walking
 * (on row 0 their diagonal/top neighbours are the previous matrix's last
 * row).  Tests in order: (1) diag+mis == v, (2) diag+mat == v with equal
 * bytes, (3) top+mis-corr == v, (4) left+mis == v; else stop.  corr = mis on
 * the last read column below row L-2eo, and, for so != 0, on the first read
 * column (width 0) for heights <= 2so+2.  Characters go to the slot starting
 * at sum_{i<t}(L_i+k) and are reversed in place at the end. */
static int traceback(const batch_t *b, cache_t *c, long t, long *out_len) {
  int st = 0;
  long m = rlen_of(b, t), L = glen_of(b, t), W = m + 1;
  long base = b->eo[t];
  long gs = gstart(b, t), rs = rstart(b, t);
  long slot = gs + (long)b->k * t;
  int so, eo;
  flank(b->dirs[t], b->k, &so, &eo);
  long P = base + (L + 1) * W - 1;
  long ap = slot;
  while (P >= W) {
    short v = cell(b, c, P), dg, lf, tp;
    if (P % W != 0) {
      dg = cell(b, c, P - W - 1);
      lf = cell(b, c, P - 1);
    } else {
      dg = 999;
      lf = 999;
    }
    tp = P != 0 ? cell(b, c, P - W) : 999;
    short width = 0, width_tmp = (short)((P % W) - 1);
    if (width_tmp > 0) width = width_tmp;
    short h_tmp = (short)(((P - base - width) / W) - 1);
    short height = h_tmp > 0 ? h_tmp : 0;
    int corr = ((width == m - 1 && height >= L - 2 * eo) ||
                (so && width == 0 && height <= (so + 1) * 2))
                   ? b->mis
                   : 0;
    long gi = gs + height, ri = rs + width;
    char gch = 0, rch = 0;
    if (gi >= 0 && gi < b->glen) gch = b->g[gi];
    else st |= SARU_ORACLE_UNDEFINED;
    if (ri >= 0 && ri < b->rlen) rch = b->r[ri];
    else st |= SARU_ORACLE_UNDEFINED;
    char oa, ob;
    long step;
    if (dg + b->mis == v) {
      oa = rch; ob = gch; step = W + 1;
    } else if (dg + b->match == v && gch == rch) {
      oa = rch; ob = gch; step = W + 1;
    } else if (tp + b->mis - corr == v) {
      oa = '_'; ob = gch; step = W;
    } else if (lf + b->mis == v) {
      oa = rch; ob = '_'; step = 1;
    } else {
      break;
    }
    if (ap >= b->total_slots) {
      st |= SARU_ORACLE_UNDEFINED;
      break;
    }
    b->ra[ap] = oa;
    b->ga[ap] = ob;
    ++ap;
    P -= step;
  }
  long len = ap - slot;
  for (long i = slot, j = ap - 1; i < j; ++i, --j) {
    char x = b->ra[i]; b->ra[i] = b->ra[j]; b->ra[j] = x;
    x = b->ga[i]; b->ga[i] = b->ga[j]; b->ga[j] = x;
  }
  if (len > L + b->k) st |= SARU_ORACLE_SLOT_OVERFLOW;
  *out_len = len;
  return st;
}

/* One candidate: fill, score D[L][m], traceback iff score <= k
 * (src/cuda-functions.cu:495-534). */
static int align_one(const batch_t *b, cache_t *c, long t) {
  short *M = matrix(b, c, t);
  long m = rlen_of(b, t), L = glen_of(b, t);
  int score = M[(m + 1) * (L + 1) - 1];
  b->scores[t] = score;
  if (score <= b->k) {
    long len;
    return traceback(b, c, t, &len);
  }
  return 0;
}

typedef struct {
  const batch_t *b;
  long chunk, nchunks;
  long *next;
  pthread_mutex_t *mu;
  int status;
} work_t;

static void *worker(void *arg) {
  work_t *w = (work_t *)arg;
  cache_t c;
  cache_init(&c);
  for (;;) {
    pthread_mutex_lock(w->mu);
    long ci = (*w->next)++;
    pthread_mutex_unlock(w->mu);
    if (ci >= w->nchunks) break;
    long s = ci * w->chunk, e = s + w->chunk < w->b->n ? s + w->chunk : w->b->n;
    for (long t = s; t < e; ++t) w->status |= align_one(w->b, &c, t);
  }
  cache_free(&c);
  return NULL;
}

static int validate(const batch_t *b) {
  long esum = 0;
  for (long t = 0; t < b->n; ++t) {
    long m = rlen_of(b, t), L = glen_of(b, t);
    if (m <= 0 || L <= 0 || m > 32000 || L > 32000) return SARU_ORACLE_BAD_INPUT;
    if (b->eo[t] != esum) return SARU_ORACLE_BAD_INPUT;
    esum += (m + 1) * (L + 1);
    if (esum > INT_MAX) return SARU_ORACLE_BAD_INPUT;
  }
  if (b->n > 0 && (b->go[b->n - 1] > b->glen || b->ro[b->n - 1] > b->rlen))
    return SARU_ORACLE_BAD_INPUT;
  return 0;
}

int saru_oracle_align(int match, int mismatch, const char *genome, long genome_len,
                      const char *reads, long reads_len, const int *genome_offsets,
                      const int *read_offsets, const int *edit_offsets, int n,
                      const signed char *dirs, int k, int nthreads, int *scores, char *read_aln,
                      char *genome_aln) {
  batch_t b = {match, mismatch, k, n, genome, reads, genome_len, reads_len,
               genome_offsets, read_offsets, edit_offsets, dirs, 0, 0, scores, read_aln,
               genome_aln};
  if (n <= 0) return 0;
  int bad = validate(&b);
  if (bad) return bad;
  b.total_slots = genome_offsets[n - 1] + (long)k * n;
  for (int attempt = 0; attempt < 2; ++attempt) {
    int threads = attempt == 0 ? nthreads : 1;
    if (threads < 1) threads = 1;
    memset(read_aln, 0, (size_t)b.total_slots);
    memset(genome_aln, 0, (size_t)b.total_slots);
    long chunk = 256, next = 0;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    long nchunks = (n + chunk - 1) / chunk;
    if (threads == 1) chunk = n, nchunks = 1;
    work_t *ws = (work_t *)calloc((size_t)threads, sizeof(work_t));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int i = 0; i < threads; ++i) {
      ws[i] = (work_t){&b, chunk, nchunks, &next, &mu, 0};
      if (threads > 1) pthread_create(&th[i], NULL, worker, &ws[i]);
    }
    int st = 0;
    if (threads == 1) worker(&ws[0]);
    for (int i = 0; i < threads; ++i) {
      if (threads > 1) pthread_join(th[i], NULL);
      st |= ws[i].status;
    }
    free(ws);
    free(th);
    /* a slot overflow makes the bytes depend on the order tracebacks ran;
     * the settled order is the serial one */
    if ((st & SARU_ORACLE_SLOT_OVERFLOW) && threads > 1) continue;
    return st;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* The writer (src/cuda-functions.cu:827-1006).                              */

typedef struct {
  char *out;
  long cap, len;
} sbuf_t;

static void sb_put(sbuf_t *s, const char *p, long n) {
  if (n <= 0) return;
  if (s->len < s->cap) {
    long room = s->cap - s->len;
    memcpy(s->out + s->len, p, (size_t)(n < room ? n : room));
  }
  s->len += n;
}

static void sb_int(sbuf_t *s, int v) {
  char tmp[16];
  int n = snprintf(tmp, sizeof(tmp), "%d", v);
  sb_put(s, tmp, n);
}

/* bytes of the slot arrays; positions outside them are undefined in the
 * reference (it reads past its host buffers) and flagged here */
static inline char at(const char *a, long total, long i, int *st) {
  if (i < 0 || i >= total) {
    *st |= SARU_ORACLE_UNDEFINED;
    return 0;
  }
  return a[i];
}

/* "%.*s": up to prec bytes, stopping at NUL; a negative precision prints
 * up to the NUL */
static void sb_prec(sbuf_t *s, const char *a, long total, long from, int prec, int *st) {
  for (long i = 0; prec < 0 || i < prec; ++i) {
    char ch = at(a, total, from + i, st);
    if (!ch) break;
    sb_put(s, &ch, 1);
  }
}

long saru_oracle_write_tsv(const int *scores, const char *read_aln, const char *genome_aln,
                           long total_slots, const int *genome_offsets, const int *pos,
                           const signed char *dirs, const int *ids, int n, int k,
                           int read_length, const char *names, int name_stride, int n_names,
                           char *out, long cap, int *status, int *done_fwd, int *done_rev) {
  sbuf_t s = {out, cap, 0};
  int st = 0, df = 0, dr = 0;
  for (long v = 0; v < n; ++v) {
    int reverse = dirs[v] > 3;
    if (scores[v] > k) continue;
    unsigned short L;
    long gs, eb = 0;
    if (v > 0) {
      L = (unsigned short)(genome_offsets[v] - genome_offsets[v - 1]);
      gs = genome_offsets[v - 1];
      eb = (long)k * v;
    } else {
      L = (unsigned short)genome_offsets[0];
      gs = 0;
    }
    long slot = gs + eb;
    unsigned int start = (unsigned int)pos[v];
    unsigned short start_corr = 0, stop_corr = 0, deletion = 0, insertion = 0;
    /* leading gaps of the read shift the start (:877-886) */
    for (long i = 0; at(read_aln, total_slots, slot + i, &st) == '_'; ++i) {
      start++;
      start_corr++;
    }
    /* trailing run of '_' or NUL scanned back from the slot's last byte;
     * its '_' count is the stop correction (:897-907) */
    for (long i = 0;; --i) {
      char ch = at(read_aln, total_slots, slot + L + i + k - 1, &st);
      if (ch != '_' && ch != 0) break;
      if (ch == '_') stop_corr++;
      if (st & SARU_ORACLE_UNDEFINED) break;
    }
    /* forward scan counting gaps in read (deletions) and window
     * (insertions) until a NUL (:910-959) */
    long i = 0, z = 0;
    short end_of_read = 0;
    while (i < (long)L - stop_corr - start_corr + z) {
      char rc = at(read_aln, total_slots, slot + start_corr + i, &st);
      if (rc == 0) {
        end_of_read = (short)i;
        break;
      }
      if (rc == '_') {
        deletion++;
        z++;
        i++;
        continue;
      }
      if (at(genome_aln, total_slots, slot + start_corr + i, &st) == '_') {
        insertion++;
        z++;
        i++;
        continue;
      }
      i++;
    }
    short chars = end_of_read > 0 ? (short)(end_of_read - stop_corr)
                                  : (short)(read_length + deletion);
    const char *name = "";
    if (ids[v] >= 0 && ids[v] < n_names) name = names + (long)ids[v] * name_stride;
    else st |= SARU_ORACLE_UNDEFINED;
    long nl = (long)strnlen(name, (size_t)name_stride);
    sb_put(&s, name, nl);
    sb_put(&s, "\t", 1);
    sb_int(&s, (int)start);
    sb_put(&s, "\t", 1);
    sb_int(&s, (int)((unsigned int)(chars - insertion) + start - 1u));
    sb_put(&s, reverse ? "\t<<\t" : "\t>>\t", 4);
    sb_prec(&s, read_aln, total_slots, slot + start_corr, chars, &st);
    sb_put(&s, "\t", 1);
    sb_prec(&s, genome_aln, total_slots, slot + start_corr, chars, &st);
    sb_put(&s, "\t", 1);
    sb_int(&s, scores[v]);
    sb_put(&s, "\n", 1);
    if (reverse) dr++;
    else df++;
  }
  if (status) *status = st;
  if (done_fwd) *done_fwd = df;
  if (done_rev) *done_rev = dr;
  return s.len;
}

/* ------------------------------------------------------------------------ */
/* Whole-call check in sub-calls (saru_oracle_check).                        */
/* ------------------------------------------------------------------------ */

typedef struct {
  int match, mis, k;
  const char *g, *r;
  const long *go, *ro;
  long n;
  const signed char *dirs;
  const int *scores;
  const char *ra, *ga;
  long chunk, nchunks;
  long *next;
  pthread_mutex_t *mu;
  long bad, first_bad;
  int status;
} check_t;

static void *check_worker(void *arg) {
  check_t *w = (check_t *)arg;
  const long cap = w->chunk + 1;
  int *go = (int *)malloc(sizeof(int) * (size_t)cap);
  int *ro = (int *)malloc(sizeof(int) * (size_t)cap);
  int *eo = (int *)malloc(sizeof(int) * (size_t)cap);
  int *sc = (int *)malloc(sizeof(int) * (size_t)cap);
  char *ra = NULL, *ga = NULL;
  long slots_cap = 0;
  cache_t c;
  cache_init(&c);
  for (;;) {
    pthread_mutex_lock(w->mu);
    long ci = (*w->next)++;
    pthread_mutex_unlock(w->mu);
    if (ci >= w->nchunks) break;
    const long s = ci * w->chunk, e = s + w->chunk < w->n ? s + w->chunk : w->n;
    const long a = s > 0 ? s - 1 : 0; /* the lead: the candidate before the chunk */
    const long g0 = a ? w->go[a - 1] : 0, r0 = a ? w->ro[a - 1] : 0;
    const long nn = e - a;
    long esum = 0, bad_input = 0;
    for (long i = 0; i < nn; ++i) {
      const long t = a + i;
      go[i] = (int)(w->go[t] - g0);
      ro[i] = (int)(w->ro[t] - r0);
      eo[i] = (int)esum;
      const long m = w->ro[t] - (t ? w->ro[t - 1] : 0), L = w->go[t] - (t ? w->go[t - 1] : 0);
      if (m <= 3 * w->k || m > 32000 || L <= 0 || L > 32000) bad_input = 1;
      esum += (m + 1) * (L + 1);
    }
    if (bad_input || esum > INT_MAX) {
      w->status |= SARU_ORACLE_BAD_INPUT;
      continue;
    }
    const long slots = go[nn - 1] + (long)w->k * nn;
    if (slots > slots_cap) {
      free(ra);
      free(ga);
      ra = (char *)malloc((size_t)slots);
      ga = (char *)malloc((size_t)slots);
      slots_cap = slots;
    }
    memset(ra, 0, (size_t)slots);
    memset(ga, 0, (size_t)slots);
    batch_t b = {w->match, w->mis, w->k, (int)nn, w->g + g0, w->r + r0, go[nn - 1], ro[nn - 1],
                 go, ro, eo, w->dirs + a, slots, esum, sc, ra, ga};
    for (int i = 0; i < NCACHE; ++i) c.t[i] = -1; /* matrices of the previous chunk */
    for (long i = s - a; i < nn; ++i) w->status |= align_one(&b, &c, i);
    for (long i = s - a; i < nn; ++i) {
      const long t = a + i;
      const long L = go[i] - (i ? go[i - 1] : 0);
      const long sub = (i ? go[i - 1] : 0) + (long)w->k * i;
      const long full = (t ? w->go[t - 1] : 0) + (long)w->k * t;
      const int x = sc[i] < w->k + 1 ? sc[i] : w->k + 1;
      const int y = w->scores[t] < w->k + 1 ? w->scores[t] : w->k + 1;
      if (x != y || memcmp(ra + sub, w->ra + full, (size_t)(L + w->k)) != 0 ||
          memcmp(ga + sub, w->ga + full, (size_t)(L + w->k)) != 0) {
        if (w->bad == 0 || t < w->first_bad) w->first_bad = t;
        w->bad++;
      }
    }
  }
  cache_free(&c);
  free(go);
  free(ro);
  free(eo);
  free(sc);
  free(ra);
  free(ga);
  return NULL;
}

long saru_oracle_check(int match, int mismatch, const char *genome, const char *reads,
                       const long *genome_offsets, const long *read_offsets, long n,
                       const signed char *dirs, int k, int nthreads, const int *scores,
                       const char *read_aln, const char *genome_aln, long *first_bad,
                       int *status) {
  *first_bad = -1;
  *status = 0;
  if (n <= 0) return 0;
  if (nthreads < 1) nthreads = 1;
  long next = 0;
  pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
  const long chunk = 2048;
  const long nchunks = (n + chunk - 1) / chunk;
  check_t *ws = (check_t *)calloc((size_t)nthreads, sizeof(check_t));
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int i = 0; i < nthreads; ++i) {
    ws[i] = (check_t){match, mismatch, k, genome, reads, genome_offsets, read_offsets, n, dirs,
                      scores, read_aln, genome_aln, chunk, nchunks, &next, &mu, 0, -1, 0};
    pthread_create(&th[i], NULL, check_worker, &ws[i]);
  }
  long bad = 0;
  for (int i = 0; i < nthreads; ++i) {
    pthread_join(th[i], NULL);
    bad += ws[i].bad;
    *status |= ws[i].status;
    if (ws[i].bad && (*first_bad < 0 || ws[i].first_bad < *first_bad)) *first_bad = ws[i].first_bad;
  }
  free(ws);
  free(th);
  return bad;
}
