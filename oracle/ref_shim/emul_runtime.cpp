/*
 * Host emulation of the CUDA runtime for the oracle build of the reference
 * (oracle/_ref).  TEST INFRASTRUCTURE ONLY: nothing here is on the product
 * path, and only tests/ and bench.py's CPU legs load what it builds.
 *
 * It provides
 *  - the few runtime/driver calls src/cuda-functions.cu makes, over host
 *    memory ("device" pointers are host pointers);
 *  - emul_launch_compute_score(): the reference launch
 *    `compute_score<<<blocks, 8>>>` (src/cuda-functions.cu:783-796) run as a
 *    serial loop over ascending thread ids.  With blockDim left at the
 *    reference's own const default (1,1,1) (src/cuda-functions.cu:51), the
 *    kernel's thread id is blockIdx.x, so each emulated thread sets it;
 *  - cuda_needleman_wunsch(): an optional batch capture (env SARU_CAPTURE_DIR)
 *    followed by the reference's own host function, renamed by the recipe;
 *  - ref_align_batch(): a driver that runs the reference kernel code over one
 *    batch laid out exactly like the reference arena, either strictly serial
 *    (the settled semantics: every predecessor matrix complete before a
 *    traceback reads it) or on a pool of host threads (the CPU baseline).
 */
#include "cuda.h"

#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <thread>
#include <vector>

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;

/* --------------------------- emulated runtime ---------------------------- */

static size_t emul_free_bytes() {
  const char *e = getenv("SARU_EMUL_FREE_MB");
  size_t mb = e ? strtoull(e, NULL, 10) : 1024;
  return mb << 20;
}

cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaMalloc(void **p, size_t n) {
  *p = aligned_alloc(256, (n + 255) & ~size_t(255));
  return *p ? cudaSuccess : 2;
}
cudaError_t cudaFree(void *p) {
  free(p);
  return cudaSuccess;
}
cudaError_t cudaMemset(void *p, int v, size_t n) {
  memset(p, v, n);
  return cudaSuccess;
}
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) {
  memcpy(d, s, n);
  return cudaSuccess;
}
cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int) {
  snprintf(p->name, sizeof(p->name), "host emulation");
  return cudaSuccess;
}
CUresult cuInit(unsigned int) { return CUDA_SUCCESS; }
CUresult cuDeviceGetCount(int *n) {
  *n = 1;
  return CUDA_SUCCESS;
}
CUresult cuDeviceGet(CUdevice *d, int i) {
  *d = i;
  return CUDA_SUCCESS;
}
CUresult cuCtxCreate(CUcontext *c, unsigned int, CUdevice) {
  *c = NULL;
  return CUDA_SUCCESS;
}
CUresult cuMemGetInfo(size_t *f, size_t *t) {
  *f = emul_free_bytes();
  *t = *f;
  return CUDA_SUCCESS;
}
CUresult cuCtxDetach(CUcontext) { return CUDA_SUCCESS; }

/* ------------------------------ launches --------------------------------- */

/* Defined by the reference TU (src/cuda-functions.cu:317). */
void compute_score(int match, int mismatch, char *read_sequences, char *genome_sequences,
                   int *read_offsets, int *genome_offsets, char *read_alignments,
                   char *genome_alignments, int sample_size, short int *edit_matrices_on_device_gpu,
                   int *edit_offsets, int *device_score_array, char *direction_array, int error);

void emul_launch_compute_score(int blocks, int threads, int match, int mismatch,
                               char *read_sequences, char *genome_sequences, int *read_offsets,
                               int *genome_offsets, char *read_alignments,
                               char *genome_alignments, int sample_size, short int *edit_matrices,
                               int *edit_offsets, int *device_score_array, char *direction_array,
                               int error) {
  long total = (long)blocks * threads;
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  blockIdx.y = blockIdx.z = 0;
  for (long id = 0; id < total; ++id) {
    blockIdx.x = (unsigned)id;
    compute_score(match, mismatch, read_sequences, genome_sequences, read_offsets, genome_offsets,
                  read_alignments, genome_alignments, sample_size, edit_matrices, edit_offsets,
                  device_score_array, direction_array, error);
  }
}

/* ------------------------- module entry + capture ------------------------ */

extern "C" void ref_emul_cuda_needleman_wunsch(int match, int mismatch, char *genome, char *reads,
                                               int *genome_offsets, int *read_offsets,
                                               int *edit_offsets, int sample_size,
                                               int *read_id_array, int *genome_pos_array,
                                               char *direction_array, int error,
                                               size_t total_genome, size_t total_read,
                                               size_t total_edit, int do_reverse);
extern "C" void ref_capture_batch(const char *dir, int match, int mismatch, const char *genome,
                                  const char *reads, const int *genome_offsets,
                                  const int *read_offsets, const int *edit_offsets,
                                  int sample_size, const int *read_id_array,
                                  const int *genome_pos_array, const char *direction_array,
                                  int error, size_t total_genome, size_t total_read,
                                  size_t total_edit, int do_reverse);

extern "C" void cuda_needleman_wunsch(int match, int mismatch, char *genome, char *reads,
                                      int *genome_offsets, int *read_offsets, int *edit_offsets,
                                      int sample_size, int *read_id_array, int *genome_pos_array,
                                      char *direction_array, int error, size_t total_genome,
                                      size_t total_read, size_t total_edit, int do_reverse) {
  const char *cap = getenv("SARU_CAPTURE_DIR");
  if (cap && *cap)
    ref_capture_batch(cap, match, mismatch, genome, reads, genome_offsets, read_offsets,
                      edit_offsets, sample_size, read_id_array, genome_pos_array, direction_array,
                      error, total_genome, total_read, total_edit, do_reverse);
  ref_emul_cuda_needleman_wunsch(match, mismatch, genome, reads, genome_offsets, read_offsets,
                                 edit_offsets, sample_size, read_id_array, genome_pos_array,
                                 direction_array, error, total_genome, total_read, total_edit,
                                 do_reverse);
}

/* ------------------------------ batch driver ----------------------------- */

namespace {

struct Batch {
  int match, mismatch, n, k;
  const char *genome, *reads;
  const int *goff, *roff;
  const char *dirs;
  int *scores;
  char *read_aln, *genome_aln;
};

inline long gstart(const Batch &b, long t) { return t ? b.goff[t - 1] : 0; }
inline long rstart(const Batch &b, long t) { return t ? b.roff[t - 1] : 0; }
inline long glen(const Batch &b, long t) { return b.goff[t] - gstart(b, t); }
inline long rlen(const Batch &b, long t) { return b.roff[t] - rstart(b, t); }

/* Runs candidates [s, e) of the batch.  When s > 0 the predecessor s-1 is
 * recomputed first as the local thread 0 of a private arena (so its own
 * traceback stops at row 0 and its outputs go to scratch); this gives every
 * traceback in [s, e) a complete predecessor matrix, exactly as a serial run
 * does, without sharing matrices between host threads. */
void run_range(const Batch &b, long s, long e, std::vector<short> &arena,
               std::vector<char> &scratch) {
  long p = s > 0 ? s - 1 : 0;
  long cnt = e - p;
  std::vector<int> ro(cnt), go(cnt), eo(cnt);
  long rb = rstart(b, p), gb = gstart(b, p);
  long esum = 0;
  for (long i = 0; i < cnt; ++i) {
    long t = p + i;
    ro[i] = (int)(b.roff[t] - rb);
    go[i] = (int)(b.goff[t] - gb);
    eo[i] = (int)esum;
    esum += (rlen(b, t) + 1) * (glen(b, t) + 1);
  }
  if ((long)arena.size() < esum) arena.resize(esum);
  char *reads = const_cast<char *>(b.reads) + rb;
  char *genome = const_cast<char *>(b.genome) + gb;
  char *dirs = const_cast<char *>(b.dirs) + p;
  long out_base = gb + (long)b.k * p; /* slot of candidate p */
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  blockIdx.y = blockIdx.z = 0;
  for (long i = 0; i < cnt; ++i) {
    long t = p + i;
    char *ra = b.read_aln + out_base;
    char *ga = b.genome_aln + out_base;
    int *sc = b.scores + p;
    if (s > 0 && i == 0) {
      /* predecessor recompute: outputs to scratch */
      long need = 2 * (glen(b, t) + b.k) + 64;
      if ((long)scratch.size() < need) scratch.resize(need);
      memset(scratch.data(), 0, need);
      ra = scratch.data();
      ga = scratch.data() + need / 2;
      static thread_local int dummy;
      sc = &dummy;
    }
    blockIdx.x = (unsigned)i;
    compute_score(b.match, b.mismatch, reads, genome, ro.data(), go.data(), ra, ga, (int)cnt,
                  arena.data(), eo.data(), sc, dirs, b.k);
  }
}

}  // namespace

/* Aligns one batch with the reference kernel code.
 *   strict=1: one arena holding every matrix at the reference's own
 *             edit_offsets, threads run serially in ascending order.
 *   strict=0: nthreads host threads, each over contiguous sub-ranges of
 *             `chunk` candidates (see run_range).
 * Output arrays are zero-filled first (the reference memsets its arena,
 * src/cuda-functions.cu:680).  Returns 0, or -1 on allocation failure. */
extern "C" int ref_align_batch(int match, int mismatch, const char *genome, const char *reads,
                               const int *genome_offsets, const int *read_offsets,
                               const int *edit_offsets, int n, const char *dirs, int k,
                               size_t total_genome, int strict, int nthreads, int chunk,
                               int *scores, char *read_aln, char *genome_aln) {
  Batch b{match, mismatch, n, k, genome, reads, genome_offsets, read_offsets,
          dirs, scores, read_aln, genome_aln};
  if (n <= 0) return 0;
  if (strict) {
    memset(read_aln, 0, total_genome);
    memset(genome_aln, 0, total_genome);
    memset(scores, 0, sizeof(int) * (size_t)n);
    long last = n - 1;
    size_t cells = (size_t)edit_offsets[last] + (size_t)(rlen(b, last) + 1) * (glen(b, last) + 1);
    short *arena = (short *)calloc(cells, sizeof(short));
    if (!arena) return -1;
    emul_launch_compute_score(n, 1, match, mismatch, const_cast<char *>(reads),
                              const_cast<char *>(genome), const_cast<int *>(read_offsets),
                              const_cast<int *>(genome_offsets), read_aln, genome_aln, n, arena,
                              const_cast<int *>(edit_offsets), scores, const_cast<char *>(dirs),
                              k);
    free(arena);
    return 0;
  }
  if (nthreads < 1) nthreads = (int)std::thread::hardware_concurrency();
  if (chunk < 1) chunk = 512;
  std::atomic<long> next(0);
  long nchunks = (n + chunk - 1) / chunk;
  auto worker = [&]() {
    std::vector<short> arena;
    std::vector<char> scratch;
    for (;;) {
      long c = next.fetch_add(1);
      if (c >= nchunks) break;
      long s = c * chunk, e = s + chunk < n ? s + chunk : n;
      long zs = gstart(b, s) + (long)k * s, ze = gstart(b, e - 1) + glen(b, e - 1) + (long)k * e;
      memset(read_aln + zs, 0, ze - zs);
      memset(genome_aln + zs, 0, ze - zs);
      run_range(b, s, e, arena, scratch);
    }
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < nthreads; ++i) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
  return 0;
}
