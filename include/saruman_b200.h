/*
 * saruman_b200.h -- C ABI of libsaruman_b200.so, a B200 (sm_100a) drop-in
 * for the alignment stage of SARUMAN.
 *
 * Part 1 is the reference's own interface, unchanged, so the reference's
 * host C (q-gram filter, candidate collection, src/hash.c:898-1111) links
 * against this library instead of its src/cuda-functions.cu.
 * Part 2 adds entry points with explicit arguments and return codes for
 * callers that hold their batches in host or device memory themselves.
 *
 * Plain C types only; no CUDA or torch types appear in the signatures
 * (streams are passed as void*).
 */
#ifndef SARUMAN_B200_H
#define SARUMAN_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Part 1: the reference interface (src/cuda-functions.h:55-78).
 * ---------------------------------------------------------------------- */

/* Replaces cuda_needleman_wunsch (src/cuda-functions.h:55-63, implemented
 * at src/cuda-functions.cu:584-1049).  Aligns sample_size candidates laid
 * out as src/hash.c:1055-1059 builds them: windows back to back with
 * genome_offsets their inclusive prefix sums, reads at read_offsets, one
 * direction/flank flag each; error = k.  Prints one TSV line per candidate
 * whose edit distance is <= k, in candidate order, exactly as the reference
 * writer does (src/cuda-functions.cu:827-1006), updates the same counters
 * and output-control arrays, and returns when the lines are written.  Safe
 * to call from the forward (do_reverse = 0) and reverse (4) threads at once.
 * Errors are reported on stderr and in saru_last_error(); the process is not
 * terminated. */
void cuda_needleman_wunsch(int match, int mismatch, char *genome_sequences_on_host,
                           char *read_sequences_on_host, int *genome_offsets, int *read_offsets,
                           int *edit_offsets, int sample_size, int *read_id_array,
                           int *genome_pos_array, char *direction_array, int error,
                           size_t total_genome_array_size, size_t total_read_sequence_array_size,
                           size_t total_edit_matrix_size, int do_reverse);

/* Replaces cuda_allocate_memory (src/cuda-functions.h:65-67,
 * src/cuda-functions.cu:541-562): selects GPU use_gpu_value and prepares the
 * stream and buffers of the forward (do_reverse != 4) or reverse (4) caller.
 * Device memory grows on demand instead of taking cuda_memory_per_thread up
 * front. */
void cuda_allocate_memory(int do_reverse);

/* Replaces cuda_free_memory (src/cuda-functions.h:69-71,
 * src/cuda-functions.cu:564-575): releases the reverse caller's resources if
 * do_reverse != 0, else the forward caller's. */
void cuda_free_memory(int do_reverse);

/* Replaces get_cuda_infos (src/cuda-functions.h:77-78,
 * src/cuda-functions.cu:1051-1120): lists the GPUs on stderr, selects the
 * one with the most free memory unless use_gpu_value names one, and returns
 * that free memory in bytes.  Exits(1) like the reference when no GPU has
 * 128 MB free. */
unsigned long int get_cuda_infos(void);

/* Defined by the reference's CUDA module (src/cuda-functions.cu:61) and read
 * by its driver (src/saruman.c:321-397): milliseconds spent aligning, per
 * strand (0 forward, 1 reverse).  This library accumulates into it. */
extern float alignment_time[2];

/* ------------------------------------------------------------------------
 * Part 2: batch entry points (no counterpart in the reference; they take the
 * same call layout with explicit arguments and return 0 or a SARU_E* code).
 * ---------------------------------------------------------------------- */

#define SARU_OK 0
#define SARU_E_INVALID 1     /* malformed batch (offsets, lengths, sizes) */
#define SARU_E_CUDA 2        /* CUDA runtime error */
#define SARU_E_NOMEM 3       /* device or host allocation failed */
#define SARU_E_OVERFLOW 4    /* a traceback left its slot (order-dependent in the reference) */
#define SARU_E_TIMEOUT 5     /* saru_server_wait: the request is not done yet */
#define SARU_MAX_CALLS 192   /* calls in one saru_align_multi_device request */

/* One call's candidates in the reference layout.  All pointers are either
 * all host or all device pointers, depending on the entry point. */
typedef struct {
  const char *genome;           /* windows back to back, genome_offsets[n-1] bytes */
  const char *reads;            /* read bytes, read_offsets[n-1] bytes */
  const int32_t *genome_offsets;/* inclusive prefix sums of the window lengths */
  const int32_t *read_offsets;  /* inclusive prefix sums of the read lengths */
  const int8_t *dirs;           /* direction/flank flags */
  int32_t n;                    /* candidates */
  int32_t k;                    /* error threshold */
  int32_t match, mismatch;      /* DP costs */
  int32_t first_of_call;        /* 1 if candidate 0 opens a reference call (its
                                   traceback stops on row 0); 0 if the batch
                                   continues an earlier one */
  int32_t max_read_length;      /* upper bound of the read lengths (device entry
                                   point; the host entry point computes it) */
  int64_t genome_bytes;         /* genome_offsets[n-1] */
  int64_t total_slots;          /* sum(L_t + k): size of each alignment array */
} saru_batch;

typedef struct {
  int32_t *scores;              /* n: D[L][m] when <= k; above k, k + 1 from the
                                   banded kernel or the exact D[L][m] from the
                                   full-rectangle path (never printed either way) */
  char *read_aln;               /* total_slots bytes, reference slot layout */
  char *genome_aln;             /* total_slots bytes */
  int32_t *status;              /* optional (device entry point): OR of SARU_S_* */
} saru_result;

/* Status bits the device entry point ORs into result->status. */
#define SARU_S_IRREGULAR 1  /* a window is not m + so + eo long, or m <= 3k */
#define SARU_S_ALPHABET 2   /* a read holds more than 2 distinct non-ACGT bytes */
#define SARU_S_OVERFLOW 4   /* a traceback left its band */
#define SARU_S_GATHER 16    /* saru_gather_device: a candidate outside the genome or read
                               table, a bad flag, or a window length that does not match */

/* One call given as the reference's filter output instead of its windows:
 * per candidate the read's row in a read table, the window's start in the
 * genome and the flag; the windows and reads of the call are then gathered
 * on the device (saru_gather_device, or the request server's resident
 * genome) exactly as src/hash.c:986-1059 builds them on the host.  No
 * counterpart in the reference, whose calls always ship the windows. */
typedef struct {
  const char *read_table;       /* nreads rows of read_length bytes, as sequenced */
  const int32_t *read_index;    /* n: row of each candidate's read */
  const int32_t *positions;     /* n: window start in the genome */
  const int8_t *dirs;           /* n: flags 0..7 (4..7: reverse-complemented read) */
  const int32_t *genome_offsets;/* n: inclusive prefix sums of the window lengths
                                   m + so + eo, as in saru_batch */
  int32_t n, nreads, k, match, mismatch, first_of_call, read_length;
  int64_t genome_bytes;         /* genome_offsets[n-1] */
  int64_t total_slots;          /* genome_bytes + k * n */
} saru_gather_call;

/* Device arrays in, enqueued on `stream`: writes the call's windows
 * (genome_bytes bytes), reads (n * read_length bytes) and read offsets (n)
 * into the caller's device buffers and fills *batch with the saru_batch
 * that views them (for saru_align_device).  Candidates it cannot gather
 * set SARU_S_GATHER in *status (device) and leave their bytes unwritten. */
int saru_gather_device(const saru_gather_call *call, const char *genome, int64_t genome_len,
                       char *windows, char *reads, int32_t *read_offsets, int32_t *status,
                       saru_batch *batch, void *stream);

/* Host buffers in, host buffers out: copies the batch to the GPU, aligns it
 * and copies back the scores and both alignment-slot arrays exactly as the
 * reference leaves them after its device-to-host copies
 * (src/cuda-functions.cu:807-824).  Prints nothing.  `lane` (0 or 1)
 * selects one of two independent streams/buffer sets. */
int saru_align_host(const saru_batch *batch, saru_result *result, int lane);
/* saru_align_host with compact result records (see saru_align_device_compact)
 * in place of the two slot strings: scores (n) and records (n x record_bytes,
 * at least saru_compact_record_bytes(read length, k), a multiple of 16) in
 * host memory.  Calls the exact path takes come back as records too.  No
 * counterpart in the reference: its output is the slot strings; the records
 * cut the bytes copied back 4x (saru_expand_compact rebuilds the slots,
 * saru_format_tsv_compact the reference's TSV). */
int saru_align_host_compact(const saru_batch *batch, int32_t *scores, uint8_t *records,
                            int64_t record_bytes, int32_t lane);

/* Device buffers in and out, enqueued on `stream` (a cudaStream_t, may be
 * NULL for the legacy stream).  Returns after enqueueing; completion is
 * ordered on the stream.  Runs the banded kernel only (unit costs, k <= 15,
 * one read length m > 3k with m <= max_read_length <= 512); candidates it
 * cannot take are reported in result->status, with score k + 1.  `scratch`
 * must be 16-byte aligned and hold saru_scratch_bytes(n, max_read_length,
 * k, k > 7) bytes of device memory.  Enqueues no allocation, so it can be captured in a CUDA
 * graph. */
int saru_align_device(const saru_batch *batch, saru_result *result, void *scratch,
                      size_t scratch_bytes, void *stream);

/* saru_align_device without any allocation, for callers that cannot call
 * cudaMalloc: a host program whose own allocator owns the device budget and
 * forbids other allocations, or a code path that must not add an
 * allocation's synchronisation and latency.  No counterpart in the
 * reference.  Same batch, result and stream arguments and the same outputs
 * as saru_align_device; the banded kernel's scratch comes from a device
 * array inside the library of SARU_STATIC_SCRATCH_BYTES (32 MiB), present on
 * every GPU that loads the library until the process exits.  Fewer thread
 * blocks run when the planes of a full grid do not fit in the array.  A batch outside the banded kernel's domain
 * is refused with SARU_E_INVALID and a message; so would be one that cannot
 * get a single block, which with reads of at most 512 bases (about 0.5 MB
 * of planes a block) cannot happen at this array size.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress, with
 * that device current), so make that first call before any stream capture;
 * the address is kept for the life of the process, so a cudaDeviceReset
 * after that first call is not supported.  All calls share the array: each
 * call clears the work counter at its start and writes every other byte it
 * reads, so nothing from an earlier call is used, but calls that overlap on
 * the GPU race. */
#define SARU_STATIC_SCRATCH_BYTES (32u << 20)
int saru_align_device_static(const saru_batch *batch, saru_result *result, void *stream);

/* Launch shape of the banded kernel for calls of one (read length, k):
 * the autotuner (saruman_b200.autotune) times the shapes on a sample and
 * installs the fastest here; every entry point that launches the banded
 * kernel for that class (saru_scratch_bytes included) then uses it.  0 in
 * a field keeps the default: as many warps per CTA (up to 4) and CTAs per
 * SM as fit, 32-bit band words when k <= 7 and 64-bit ones above.  A
 * multi-call launch looks up its class by (longest read, largest k).
 * Results do not depend on the shape.  Not in the reference. */
typedef struct {
  int32_t warps_per_cta; /* 1..4: alignments per CTA = 32 x warps */
  int32_t ctas_per_sm;   /* cap on resident CTAs per SM */
  int32_t word_bits;     /* 64: 64-bit band words for k <= 7 too; 32 only for k <= 7 */
} saru_tuning;
int saru_tuning_set(int32_t read_length, int32_t k, const saru_tuning *t); /* NULL: remove */
int saru_tuning_get(int32_t read_length, int32_t k, saru_tuning *t);       /* 1 if set */
void saru_tuning_clear(void);

/* ---- cost model of the autotuner (costmodel.cu) -----------------------------
 * A fully connected network, dims[0] inputs -> ... -> dims[nlayers] = 1
 * output, tanh hidden layers, fp32, that predicts the banded kernel's log
 * time per candidate from a bin's features and a launch shape; the
 * autotuner times only the shapes it ranks best.  Parameters: per layer
 * W (fan_out x fan_in, row-major) then the bias.  x: n rows of dims[0]
 * features.  All arrays are device arrays; `work` holds
 * saru_mlp_work_floats(dims, nlayers, n) floats.  Gradients are exact
 * (fixed-order sums) for the mean squared error over the n rows.  Not in the
 * reference. */
int64_t saru_mlp_param_count(const int32_t *dims, int32_t nlayers);
int64_t saru_mlp_work_floats(const int32_t *dims, int32_t nlayers, int32_t n);
int saru_mlp_forward(const int32_t *dims, int32_t nlayers, const float *params, const float *x,
                     int32_t n, float *y, float *work, void *stream);
int saru_mlp_loss_grad(const int32_t *dims, int32_t nlayers, const float *params, const float *x,
                       const float *y, int32_t n, float *loss, float *grad, float *work,
                       void *stream);
int saru_mlp_adam_step(float *params, const float *grad, float *m, float *v, int64_t count,
                       float lr, float beta1, float beta2, float eps, int32_t step, void *stream);

/* ---- compact results (no counterpart in the reference) ---------------------
 * The banded kernel can return, instead of the two slot strings of each
 * candidate (2(L + k) bytes), a fixed-size record of its traceback steps,
 * 2 bits each: record_bytes = saru_compact_record_bytes(m, k), 48 bytes for
 * m = 100, k = 5 against ~230 for the slots.  Word 0 of a record: the step
 * count n (bits 0-15) and an overflow flag (bit 16); words 1..: the steps
 * in traceback order, 16 per word (1 DIAG, 2 UP = gap in the read, 3 LEFT =
 * gap in the window).  saru_expand_compact rebuilds on the host, from the
 * records and the call's own reads and windows, exactly the slot strings the
 * slot mode writes (the reference's layout).  Same conditions as
 * saru_align_device; `records` holds n * record_bytes bytes (device). */
int64_t saru_compact_record_bytes(int32_t max_read_length, int32_t k);
int saru_align_device_compact(const saru_batch *batch, int32_t *scores, uint8_t *records,
                              int64_t record_bytes, int32_t *status, void *scratch,
                              size_t scratch_bytes, void *stream);
/* Host arrays: the call (host batch), its scores and records -> both slot
 * arrays (total_slots bytes each).  nthreads <= 0: all hardware threads. */
int saru_expand_compact(const saru_batch *batch, const int32_t *scores, const uint8_t *records,
                        int64_t record_bytes, char *read_aln, char *genome_aln,
                        int32_t nthreads);

/* The reference writer's TSV lines (as saru_format_tsv) straight from host
 * compact records, without the call's slot arrays: each thread expands only
 * the slots its lines and the writer's scans reach.  Returns the bytes
 * needed (-1 on invalid input) and writes min(needed, cap) bytes to out.
 * nthreads <= 0: all hardware threads. */
int64_t saru_format_tsv_compact(const saru_batch *batch, const int32_t *scores,
                                const uint8_t *records, int64_t record_bytes,
                                const int32_t *read_ids, const int32_t *genome_pos,
                                int32_t read_length, const char *names, int32_t name_stride,
                                int32_t n_names, char *out, int64_t cap, int32_t *done_fwd,
                                int32_t *done_rev, int32_t nthreads);

/* ---- candidate generation on the device (no counterpart in the reference,
 * whose filter runs on the host: src/hash.c:348-839) ---------------------------
 * The reference's q-gram pair filter for one strand and one batch of reads
 * (the reads it loads at a time, its -c option; read ids count from 0 in
 * each batch), one warp per read, against a q-gram index of the genome
 * held on the device (device < 0: the calling thread's current device).
 * The kept positions are assembled into exactly the
 * calls the reference would submit: read ids, positions, flags and call
 * boundaries, set by chunk_value (its -s option: the queue threshold, which
 * is also the number of reads per chunk of its data array).  Perfect hits,
 * which the reference prints from the filter, come back as (read id,
 * 0-based start).  A genome read in chunks (-G) takes one filter per chunk
 * (saru_filter_set_chunk).  The filter's device buffers grow with the
 * largest batch it has run, stream-ordered on its own stream
 * (cudaMallocAsync from the device's current memory pool), so a growth
 * does not wait for other work on the device. */
typedef struct saru_filter saru_filter;
saru_filter *saru_filter_create(const char *genome, int64_t genome_len, int32_t read_length,
                                int32_t k, int32_t device);
/* reads: nreads x read_length bytes (host), as the reference reads them.
 * counts[0..2] = calls, candidates, perfect hits.  SARU_E_OVERFLOW if a read
 * keeps more than 4096 positions on one strand. */
int saru_filter_run(saru_filter *f, const char *reads, int32_t nreads, int32_t do_reverse,
                    uint32_t chunk_value, int64_t *counts);
/* The last run's calls: call_begin (calls + 1 entries), ids, pos, dirs
 * (candidates), perfect_ids, perfect_pos (perfect hits); NULL skips one. */
int saru_filter_results(const saru_filter *f, int64_t *call_begin, int32_t *ids, int32_t *pos,
                        int8_t *dirs, int32_t *perfect_ids, int32_t *perfect_pos);
/* Device time of the last run's filter (ms), and the resident genome (device). */
double saru_filter_last_ms(const saru_filter *f);
const char *saru_filter_genome(const saru_filter *f);
/* The filter's genome as chunk of a larger genome (the reference's -G loop,
 * src/saruman.c:181-415): `offset` is the genome position of its first
 * byte, `limit` the position windows must end by (the reference's
 * total_bases_read, src/hash.c:982).  The q-gram lists then hold positions
 * in the whole genome (src/util.c:481), starts at or before the chunk's
 * first byte are not taken (src/hash.c:545), and the calls' positions are
 * whole-genome positions (windows at position - offset in the chunk).
 * Default: offset 0, limit = the genome's length. */
int saru_filter_set_chunk(saru_filter *f, int64_t offset, int64_t limit);
void saru_filter_destroy(saru_filter *f);

/* ---- input readers (host): the reference's read and genome readers -------
 * Reads of a FASTA (fastq = 0) or FASTQ file in the reference's batches
 * (replaces read_multiple_fasta_file, src/util.c:294-452): records of 2 or
 * 4 lines read as fgets reads them (names into 60 bytes, sequence lines
 * into read_length + 2), sequences cut at read_length and upper-cased;
 * shorter reads and reads with more than max_n Ns are dropped.
 * saru_reads_next takes up to max_entries records: the kept ones go to
 * reads (read_length bytes each) and names (60-byte NUL-padded slots: the
 * name line without its first and last byte), *skipped gets the dropped
 * count; returns the kept count (read ids 0.. of this batch), 0 with
 * *skipped == 0 at the end of the file, -1 on bad arguments. */
typedef struct saru_reads saru_reads;
saru_reads *saru_reads_open(const char *path, int32_t fastq, int32_t read_length, int32_t max_n);
int32_t saru_reads_next(saru_reads *r, int32_t max_entries, char *reads, char *names,
                        int32_t *skipped);
void saru_reads_close(saru_reads *r);

/* The genome of a FASTA file in the reference's chunks (replaces the chunk
 * loop of src/saruman.c:139-271, -G): each chunk is chunk_value bases and
 * an overhang of read_length bases, newlines dropped, upper-cased, the
 * first line skipped.  saru_genome_next writes the chunk (out: at least
 * chunk_value + read_length + 1 bytes, NUL-terminated), *len its bytes,
 * *bases its own bases (without the overhang), *total the bases of all
 * chunks so far (the limit windows must end by); returns 1 for a chunk, 0
 * after the last one (the first that did not fill chunk_value bases), -1 on
 * bad arguments.  Chunk i's bytes start at genome position i * chunk_value. */
typedef struct saru_genome_reader saru_genome_reader;
saru_genome_reader *saru_genome_open(const char *path, int64_t chunk_value, int32_t read_length);
int32_t saru_genome_next(saru_genome_reader *g, char *out, int64_t *len, int64_t *bases,
                         int64_t *total);
void saru_genome_close(saru_genome_reader *g);

/* Device scratch the banded kernel needs for a batch (bytes). */
size_t saru_scratch_bytes(int32_t n, int32_t read_length, int32_t k, int wide);

/* Several calls at once: each saru_batch is one reference-style call (its
 * own read length, k, band width, first-of-call flag and output arrays, all
 * device pointers).  Calls of similar read length and band width share one
 * persistent launch whose warps take 32-candidate tiles of all its calls
 * from one work counter, heaviest first; the launches of different length
 * classes run concurrently on streams forked from `stream` and joined back
 * to it.  Up to 192 calls (SARU_MAX_CALLS); conditions per call as for
 * saru_align_device.  Each call's status bits are ORed into its
 * results[i].status when that is non-NULL, else into *status (device
 * words the caller zeroes).  `scratch` must hold
 * saru_multi_scratch_bytes(calls, ncalls) bytes of device memory. */
int saru_align_multi_device(const saru_batch *calls, saru_result *results, int32_t ncalls,
                            int32_t *status, void *scratch, size_t scratch_bytes, void *stream);
size_t saru_multi_scratch_bytes(const saru_batch *calls, int32_t ncalls);
/* The same request with compact records instead of slot strings: call i's
 * records (n x saru_compact_record_bytes(max_read_length, k) bytes, device
 * memory) go to results[i].read_aln; results[i].genome_aln is unused.  Same
 * scratch as saru_align_multi_device. */
int saru_align_multi_device_compact(const saru_batch *calls, saru_result *results,
                                    int32_t ncalls, int32_t *status, void *scratch,
                                    size_t scratch_bytes, void *stream);

/* ---- request server (continuous batching on one GPU) ----------------------
 * Not in the reference, whose alignment calls are synchronous
 * (src/cuda-functions.cu:77-239).  A server owns one GPU, a device arena of
 * device_budget_bytes for the inputs and outputs of admitted requests, and
 * three streams (copy in, compute, copy out).  A request is a set of
 * reference-style calls with HOST arrays (pinned memory lets the copies
 * overlap; pageable memory works but serialises them) and host outputs.
 * Requests are admitted in arrival order while the arena has room; all
 * requests admitted together form one launch group, aligned by one
 * saru_align_multi_device request, while the next group's inputs are copied
 * in and the previous group's results are copied out.  Each request's
 * results are those saru_align_host gives for each of its calls: calls the
 * banded kernel flags (rare bytes, irregular windows, m <= 3k) are redone on
 * the exact path before the request completes.
 * pipeline = 0 processes one request at a time, one launch per call and no
 * overlap: the plain per-request loop, for comparison.
 * The caller keeps a request's host arrays alive until saru_server_wait
 * returns something other than SARU_E_TIMEOUT for its ticket. */
typedef struct saru_server saru_server;
typedef struct {
  int32_t device;
  int32_t pipeline;                /* 1: continuous batching; 0: one request at a time */
  int32_t max_requests_per_launch; /* cap on a launch group (>= 1) */
  int32_t max_inflight;            /* launch groups queued on the GPU at once (>= 1) */
  int64_t device_budget_bytes;     /* arena for request inputs and outputs */
  int64_t host_pool_bytes;         /* pinned host memory for reads-only requests' results,
                                      allocated on first use (0: 4 GiB); results that do not
                                      fit go to pageable memory */
} saru_server_config;
typedef struct {
  const saru_batch *calls;        /* host pointers */
  saru_result *results;           /* host outputs; status unused */
  int32_t ncalls;
  const saru_gather_call *gather; /* if not NULL: the ncalls calls are these (host arrays),
                                     gathered from the resident genome; `calls` is unused */
  int32_t compact;                /* 1: results[i].read_aln receives the call's compact
                                     records (n x saru_compact_record_bytes(m, k) bytes;
                                     genome_aln unused) instead of the slot strings */
} saru_request;
typedef struct {
  int64_t submit_us, admit_us, done_us; /* steady clock, microseconds */
  int32_t group;                        /* launch group the request ran in */
  int32_t redone_calls;                 /* calls redone on the exact path */
} saru_request_stats;

/* NULL on failure (saru_last_error() says why). */
saru_server *saru_server_create(const saru_server_config *cfg);
/* Copies the genome that gather requests index to the server's GPU, where
 * it stays (outside the device budget) until replaced or the server is
 * destroyed.  Refused (SARU_E_INVALID) while requests are unfinished. */
int saru_server_set_genome(saru_server *s, const char *genome, int64_t genome_len);
/* Queues a request; *ticket identifies it.  SARU_E_INVALID for calls the
 * banded kernel cannot take at all (costs, k, read length), SARU_E_NOMEM if
 * it can never fit the arena. */
int saru_server_submit(saru_server *s, const saru_request *req, int64_t *ticket);
/* Waits up to timeout_ms for a request: SARU_OK (results written),
 * SARU_E_TIMEOUT (still running; wait again), or the error the request
 * ended with.  A ticket is forgotten once a wait returns anything else
 * than SARU_E_TIMEOUT. */
int saru_server_wait(saru_server *s, int64_t ticket, int32_t timeout_ms, saru_request_stats *stats);
/* Requests of reads only: the server does the reference's whole per-strand
 * daemon work (src/hash.c:295-470, 841-851, 898-1111) for them.  For each
 * read set it runs the q-gram pair filter against the resident genome
 * (saru_server_set_genome) on both strands, cuts the calls at the queue
 * threshold, gathers every call's windows and reads on the device, aligns
 * and keeps the results for saru_server_read_results.  A filter thread
 * works on the next request while earlier ones align, as the reference's
 * strand daemons filter while the GPU aligns.  Not in the reference's ABI
 * (its filter is host code calling cuda_needleman_wunsch per call). */
typedef struct {
  const char *reads;     /* nreads x read_length bytes, as sequenced; read ids 0..nreads-1;
                            must stay valid until the request is waited for */
  int32_t nreads, read_length, k;
  uint32_t chunk_value;  /* the queue threshold (-s), candidates per call; 0: one that keeps
                            each call under 2^31 matrix cells */
} saru_read_set;
/* Queues a reads-only request (1..16 sets, compact: records instead of slot
 * strings).  Needs saru_server_set_genome first. */
int saru_server_submit_reads(saru_server *s, const saru_read_set *sets, int32_t nsets,
                             int32_t compact, int64_t *ticket);
/* The results of set `set` of a reads-only request, after saru_server_wait
 * returned SARU_OK for it: pointers into the server's memory, valid until
 * saru_server_release.  Call c (strand call_strand[c], 0 or 4) holds
 * candidates call_begin[c] .. call_begin[c+1]; its slot strings start at
 * slot_begin[c] of read_aln / genome_aln (slot mode), its records at
 * candidate call_begin[c] of records (compact mode).  Perfect hits are the
 * filter's own output lines (never aligned). */
typedef struct {
  int32_t ncalls, nperfect;
  int64_t n;                   /* candidates */
  const int64_t *call_begin;   /* ncalls + 1 */
  const int64_t *slot_begin;   /* ncalls + 1 */
  const int8_t *call_strand;   /* ncalls */
  const int32_t *ids, *pos;    /* n: read id, window start */
  const int8_t *dirs;          /* n */
  const int32_t *scores;       /* n */
  const char *read_aln, *genome_aln;  /* slot mode, slot_begin[ncalls] bytes each */
  const uint8_t *records;      /* compact mode, n x record_bytes */
  int64_t record_bytes;
  const int32_t *perfect_ids, *perfect_pos;  /* nperfect; pos = 0-based start */
  const int8_t *perfect_strand;              /* nperfect */
} saru_read_results;
int saru_server_read_results(saru_server *s, int64_t ticket, int32_t set, saru_read_results *out);
/* Frees a waited-for reads-only request's results. */
void saru_server_release(saru_server *s, int64_t ticket);

/* Launch groups formed and kernel launches enqueued so far. */
void saru_server_counters(saru_server *s, int64_t *groups, int64_t *launches);
/* Finishes queued requests, then frees everything. */
void saru_server_destroy(saru_server *s);

/* Formats the reference's TSV lines for one aligned call into `out`
 * (capacity cap) and returns the bytes needed (ordered ranges of candidates
 * on the host cores).  names: n_names entries of name_stride bytes, indexed
 * by read id. */
int64_t saru_format_tsv(const saru_batch *batch, const saru_result *result,
                        const int32_t *read_ids, const int32_t *genome_pos, int32_t read_length,
                        const char *names, int32_t name_stride, int32_t n_names, char *out,
                        int64_t cap, int32_t *done_fwd, int32_t *done_rev);

/* SAM records for the reference writer's TSV lines (tsv: len bytes, lines
 * separated by '\n'; blank lines skipped): a header (@HD, @SQ with rname and
 * rlen, @PG), then per line QNAME (the name up to its first blank), FLAG (16
 * for "<<", 0 for ">>", 4 for an unmapped line), RNAME, POS (the printed
 * 1-based start), MAPQ 255, CIGAR (M, I for '_' in the genome string, D for
 * '_' in the read string), '*', 0, 0, SEQ (the read string without gaps),
 * '*', NM:i:<edit distance>.  Writes up to cap bytes to out and returns the
 * bytes the text needs, or -1 for a line of fewer than 7 tab-separated
 * fields.  The reference leaves SAM to an external script (README.md:32);
 * no counterpart in its code. */
int64_t saru_tsv_to_sam(const char *tsv, int64_t len, const char *rname, int64_t rlen,
                        char *out, int64_t cap);

/* Message of the last error on the calling thread ("" if none). */
const char *saru_last_error(void);

/* Number of kernels this library has launched (for accounting). */
uint64_t saru_kernel_launches(void);

/* Diagnostics: 32-bit integer operations per second the current GPU
 * sustains on independent logic/add/shift chains at full occupancy (the
 * denominator of the banded kernel's roofline); -1 on error. */
double saru_int32_issue_probe(int iters);

#ifdef __cplusplus
}
#endif
#endif
