// kernels.cuh -- launch interface of the alignment kernels (host <-> device).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace saru {

// status bits written by the kernels
constexpr int kStatusIrregular = 1;  // window length != m + so + eo, or m <= 3k
constexpr int kStatusAlphabet = 2;   // a read with more distinct non-ACGT bytes than supported
constexpr int kStatusOverflow = 4;   // a traceback left its slot / band
constexpr int kStatusUndefined = 8;  // the reference would read outside its arrays
constexpr int kStatusGather = 16;    // a gathered candidate lies outside the genome or read table

constexpr int kMaxBandM = 512;  // longest read of the banded kernel
constexpr int kMaxOpWords = (kMaxBandM + 3 * 15 + 15) / 16 + 1;

// One reference-style call inside a launch: its own read length, k, band
// width and output arrays; offsets are relative to its own arrays.
struct Segment {
  const uint8_t *genome;
  const uint8_t *reads;
  const int32_t *goff;
  const int32_t *roff;
  const int8_t *dirs;
  int32_t *scores;
  uint8_t *read_aln;
  uint8_t *genome_aln;
  int *status;      // this call's status word (device)
  uint8_t *records;  // compact result records instead of slot strings (nullptr: slots)
  long rec_bytes;
  long n;           // candidates t0 .. n - 1 of the call's arrays are this segment's
  long t0;          // (t0 > 0, a multiple of 32: a later slice of a call)
  long tile_begin;  // first 32-candidate tile of this segment in the launch
  int k, max_m, first_of_call, wide;
};

constexpr int kMaxSegs = 192;         // segments per launch (kernel parameter space)
constexpr size_t kCounterBytes = 256;  // tile counter at the start of the scratch

struct KernelArgs {
  Segment segs[kMaxSegs];  // by value in the parameter space
  int nseg;
  long total_tiles;
  int *counter;  // zeroed before the launch: next tile to take
  void *planes;  // decision planes: plane_units(max_m, wide_any) x lanes units (band_tile.cuh)
  long grid;
  int max_m, max_k, wide_any;
  int warps_req;                       // requested warps per CTA (0: as many as fit)
  long rs_bytes, ws_bytes, warp_smem;  // shared-memory slice layout (set by the launcher)
};

// Launch shape of the banded kernel for one (read length, k) class; 0 keeps
// the default (as many warps per CTA and CTAs per SM as fit; 32-bit band
// words when k <= 7).
struct Tuning {
  int warps = 0;        // warps per CTA, 1..4
  int ctas_per_sm = 0;  // cap on resident CTAs per SM
  int word_bits = 0;    // 64: 64-bit band words even when k <= 7
};

struct BandLayout {
  long rs_bytes = 0, ws_bytes = 0, region_bytes = 0, warp_smem = 0, cta_smem = 0;
  int warps = 0;  // warps per CTA (0: a warp slice does not fit)
};

struct FullArgs {
  const uint8_t *genome;
  const uint8_t *reads;
  const int32_t *goff;
  const int32_t *roff;
  const int8_t *dirs;
  const int64_t *eoff;  // cell offset of each matrix in the arena
  long n;
  int k, match, mismatch, first_of_call;
  long genome_bytes, read_bytes;
  short *arena;
  int32_t *scores;
  uint8_t *read_aln;
  uint8_t *genome_aln;
  int *status;
};

// Windows and reads of one call gathered from a resident genome (gather.cu).
struct GatherArgs {
  const uint8_t *genome;  // resident genome, one byte a base (nullptr: packed)
  long genome_len;
  // or 2 bits a base (A 0, C 1, G 2, T 3; base p in bits 2(p & 3) of byte
  // p >> 2) with the bytes that are not A/C/G/T as exceptions, their genome
  // positions ascending
  const uint8_t *packed;
  const int64_t *exc_pos;
  const uint8_t *exc_byte;
  long nexc;
  const uint8_t *table;  // read table: nreads rows of m bytes, as sequenced
  long nreads;
  const int32_t *read_index, *positions, *goff;
  const int8_t *dirs;
  long n, genome_bytes;
  int m, k;
  uint8_t *windows, *reads;  // outputs in the reference call layout
  int32_t *read_offsets;
  int *status;
};

cudaError_t launch_gather(const GatherArgs &a, int sms, cudaStream_t s);

BandLayout band_layout(int max_m, int k, int warps_req = 0, bool wide = true);
long band_grid(int sms, long n, const BandLayout &L, int smem_per_sm, int ctas_cap = 0);
size_t band_scratch_bytes(long grid, int max_m, int k, bool wide,
                          int warps_req = 0);  // counter + planes
cudaError_t launch_band_kernel(KernelArgs &a, cudaStream_t s);
cudaError_t launch_full_kernels(const FullArgs &a, cudaStream_t s);

}  // namespace saru
