/*
 * saru_oracle -- host C restatement of SARUMAN's alignment stage.
 *
 * TEST INFRASTRUCTURE, NOT THE PRODUCT.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it, and only as the checker.  The product
 * (the saruman_b200 library) never links or calls it.
 *
 * It restates, from the mathematics of the reference and not from its code:
 *   the full-rectangle semiglobal fill   src/cuda-functions.cu:340-497
 *   the traceback with its tie order     src/cuda-functions.cu:108-315
 *   the TSV writer                       src/cuda-functions.cu:827-1006
 * over a batch in the call layout of cuda_needleman_wunsch
 * (src/cuda-functions.h:55-63, built by src/hash.c:898-1111).  Semantics are
 * the "settled" ones: every traceback sees complete matrices of the earlier
 * candidates of the call, as a serial ascending run of the reference does.
 */
#ifndef SARU_ORACLE_H
#define SARU_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* status bits returned by saru_oracle_align / saru_oracle_write_tsv */
#define SARU_ORACLE_SLOT_OVERFLOW 1  /* a traceback wrote past its own slot */
#define SARU_ORACLE_UNDEFINED 2      /* the reference would touch memory outside its arrays */
#define SARU_ORACLE_BAD_INPUT 4      /* offsets not in the reference's own layout */

/* Aligns candidates [0, n) of one call.  Output arrays must hold
 * total_slots = sum(L_t + k) bytes; they are zero-filled first.  nthreads<=1
 * runs serially; more threads give the same bytes.  Returns status bits. */
int saru_oracle_align(int match, int mismatch, const char *genome, long genome_len,
                      const char *reads, long reads_len, const int *genome_offsets,
                      const int *read_offsets, const int *edit_offsets, int n,
                      const signed char *dirs, int k, int nthreads, int *scores, char *read_aln,
                      char *genome_aln);

/* Formats the TSV lines the reference prints for one call into `out`
 * (capacity `cap`).  names: table of read names, `name_stride` bytes each,
 * indexed by read id (n_names entries).  Returns the number of bytes the
 * text needs (it is truncated if that exceeds cap); *status gets status
 * bits; done_fwd and done_rev get the alignments counted per strand. */
long saru_oracle_write_tsv(const int *scores, const char *read_aln, const char *genome_aln,
                           long total_slots, const int *genome_offsets, const int *pos,
                           const signed char *dirs, const int *ids, int n, int k,
                           int read_length, const char *names, int name_stride, int n_names,
                           char *out, long cap, int *status, int *done_fwd, int *done_rev);

/* Checks another implementation's outputs for one whole call (candidate 0
 * opens it) of any size against this restatement.  The call is aligned in
 * sub-calls of a few thousand candidates, each led by the candidate before
 * it: a traceback only reads the previous matrix's last row when m > 3k,
 * so every candidate after the lead gets the whole call's bytes (the lead's
 * own result is discarded).  Compares min(score, k + 1) and the candidate's
 * L + k slot bytes of both strings.  Offsets are int64 so a call may hold
 * more than 2^31 window bytes.  Returns the number of candidates that
 * differ; *first_bad gets the lowest such index (-1 if none) and *status
 * the OR of the oracle's status bits (SARU_ORACLE_BAD_INPUT if some
 * candidate has m <= 3k, where the lead would not suffice). */
long saru_oracle_check(int match, int mismatch, const char *genome, const char *reads,
                       const long *genome_offsets, const long *read_offsets, long n,
                       const signed char *dirs, int k, int nthreads, const int *scores,
                       const char *read_aln, const char *genome_aln, long *first_bad,
                       int *status);

#ifdef __cplusplus
}
#endif
#endif
