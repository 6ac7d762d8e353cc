/*
 * C-side glue for the oracle build of the reference (oracle/_ref).  TEST
 * INFRASTRUCTURE ONLY.  Compiled as C with the reference's own headers
 * (-fcommon, so their tentative definitions merge), it lets a test harness
 *  - fill the caller-owned globals the reference CUDA module reads
 *    (read_names, read_length_value, output-control arrays), and
 *  - capture each cuda_needleman_wunsch() batch to a file (".nwb").
 *
 * .nwb layout (little endian): char magic[8]="SARUNWB1"; int32 match,
 * mismatch, n, k, do_reverse, read_length; int64 total_genome, total_read,
 * total_edit; then genome bytes (total_genome - n*k), read bytes
 * (total_read), int32 genome_offsets[n], read_offsets[n], edit_offsets[n],
 * read_ids[n], genome_pos[n], int8 directions[n], and char names[n][60]
 * (the read name of each candidate, NUL padded).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "util.h"
#include "saruman.h"
#include "hash.h"
#include "cuda-functions.h" /* tentative definitions of the arena pointers */

void ref_set_read_length(int m) { read_length_value = (unsigned short)m; }
void ref_set_verbose(int v) { be_verbose_value = (unsigned short)v; }

/* names: n entries of `stride` bytes each; entry i becomes read number i. */
void ref_set_read_names(int n, const char *names, int stride) {
  struct read_name_hash *cur, *tmp;
  HASH_ITER(hh, read_names, cur, tmp) {
    HASH_DEL(read_names, cur);
    free(cur);
  }
  read_names = NULL;
  for (int i = 0; i < n; i++) {
    struct read_name_hash *e = (struct read_name_hash *)calloc(1, sizeof(*e));
    e->read_number = i;
    strncpy(e->name, names + (size_t)i * stride, MAX_READ_DESCRIPTION_LENGTH - 1);
    HASH_ADD_INT(read_names, read_number, e);
  }
}

void ref_alloc_output_control(int n) {
  free(forward_output_control);
  free(reverse_output_control);
  forward_output_control = (char *)calloc(n > 0 ? n : 1, 1);
  reverse_output_control = (char *)calloc(n > 0 ? n : 1, 1);
}

void ref_set_memory_per_thread(unsigned long bytes) { cuda_memory_per_thread = bytes; }

unsigned int ref_alignments_done(int reverse) {
  return reverse ? reverse_alignments_done : forward_alignments_done;
}

static void wr(FILE *f, const void *p, size_t n) {
  if (n && fwrite(p, 1, n, f) != n) {
    fprintf(stderr, "capture: short write\n");
    exit(3);
  }
}

void ref_capture_batch(const char *dir, int match, int mismatch, const char *genome,
                       const char *reads, const int *genome_offsets, const int *read_offsets,
                       const int *edit_offsets, int n, const int *ids, const int *pos,
                       const char *dirs, int k, size_t total_genome, size_t total_read,
                       size_t total_edit, int do_reverse) {
  static int seq[2];
  int which = do_reverse ? 1 : 0;
  char path[4096];
  snprintf(path, sizeof(path), "%s/batch_%s_%04d.nwb", dir, which ? "rev" : "fwd", seq[which]++);
  FILE *f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "capture: cannot open %s\n", path);
    exit(3);
  }
  int32_t hdr[6] = {match, mismatch, n, k, do_reverse, (int32_t)read_length_value};
  int64_t sz[3] = {(int64_t)total_genome, (int64_t)total_read, (int64_t)total_edit};
  wr(f, "SARUNWB1", 8);
  wr(f, hdr, sizeof(hdr));
  wr(f, sz, sizeof(sz));
  wr(f, genome, total_genome - (size_t)n * k);
  wr(f, reads, total_read);
  wr(f, genome_offsets, sizeof(int) * (size_t)n);
  wr(f, read_offsets, sizeof(int) * (size_t)n);
  wr(f, edit_offsets, sizeof(int) * (size_t)n);
  wr(f, ids, sizeof(int) * (size_t)n);
  wr(f, pos, sizeof(int) * (size_t)n);
  wr(f, dirs, (size_t)n);
  char name[MAX_READ_DESCRIPTION_LENGTH];
  for (int i = 0; i < n; i++) {
    struct read_name_hash *e = NULL;
    int id = ids[i];
    HASH_FIND_INT(read_names, &id, e);
    memset(name, 0, sizeof(name));
    if (e) strncpy(name, e->name, sizeof(name) - 1);
    wr(f, name, sizeof(name));
  }
  fclose(f);
}
