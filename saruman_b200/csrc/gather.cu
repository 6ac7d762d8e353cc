// gather.cu -- builds a call's windows and reads on the device from a
// resident genome and a read table, as the reference's host collection loop
// builds them (src/hash.c:986-1059): the window of candidate t is the
// m + so + eo genome bytes from its position (strncpy of
// genome_sequence[pos], :997-998 and :1017-1018); its read is the table row
// as sequenced for flags 0-3 and its reverse complement for flags 4-7
// (src/util.c:35-57: A<->T, C<->G, other bytes kept, then reversed).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/saruman_b200.h"
#include "kernels.cuh"
#include "saru_core.cuh"
#include "server_internal.h"

namespace saru {

__device__ __forceinline__ uint8_t complement_byte(uint8_t c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return c;
  }
}

// One warp per candidate; lanes copy consecutive bytes (coalesced).
__global__ void __launch_bounds__(256) saru_gather_kernel(GatherArgs a) {
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  int status = 0;
  for (long t = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < a.n; t += warps) {
    const int8_t dir = a.dirs[t];
    const long gend = a.goff[t];
    const long gbeg = t ? (long)a.goff[t - 1] : 0;
    const long pos = a.positions[t];
    const long ri = a.read_index[t];
    int so = 0, eo = 0;
    flank_of(dir, a.k, so, eo);
    const long L = (long)a.m + so + eo;
    // the reference's filter never emits these; report instead of reading
    // outside the genome or the read table
    if (dir < 0 || dir > 7 || gend - gbeg != L || gend > a.genome_bytes || pos < 0 ||
        pos + L > a.genome_len || ri < 0 || ri >= a.nreads) {
      status |= kStatusGather;
      continue;
    }
    uint8_t *dst = a.windows + gbeg;
    if (a.genome) {
      const uint8_t *src = a.genome + pos;
      for (long j = lane; j < L; j += 32) dst[j] = src[j];
    } else {
      for (long j = lane; j < L; j += 32) {
        const long p = pos + j;
        dst[j] = (uint8_t)(0x54474341u >> (8 * ((a.packed[p >> 2] >> (2 * (p & 3))) & 3u)));
      }
      if (a.nexc > 0) {  // the window's exceptions: first one at or after pos
        long lo = 0, hi = a.nexc;
        while (lo < hi) {
          const long mid = (lo + hi) >> 1;
          if (a.exc_pos[mid] < pos) lo = mid + 1;
          else hi = mid;
        }
        __syncwarp();
        for (long e = lo + lane; e < a.nexc && a.exc_pos[e] < pos + L; e += 32)
          dst[a.exc_pos[e] - pos] = a.exc_byte[e];
      }
    }
    const uint8_t *row = a.table + ri * a.m;
    uint8_t *rd = a.reads + t * a.m;
    if (dir < 4) {
      for (int j = lane; j < a.m; j += 32) rd[j] = row[j];
    } else {
      for (int j = lane; j < a.m; j += 32) rd[j] = complement_byte(row[a.m - 1 - j]);
    }
    if (lane == 0) a.read_offsets[t] = (int32_t)((t + 1) * a.m);
  }
  status = __reduce_or_sync(0xffffffffu, status);
  if (status && lane == 0) atomicOr(a.status, status);
}

cudaError_t launch_gather(const GatherArgs &a, int sms, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const long warps_needed = a.n;
  long blocks = (warps_needed + 7) / 8;
  const long cap = (long)sms * 8;  // 8 blocks of 256 threads per SM
  if (blocks > cap) blocks = cap;
  saru_gather_kernel<<<(unsigned)blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace saru

namespace saru {

int gather_packed(const saru_gather_call *c, const PackedGenome &g, char *windows, char *reads,
                  int32_t *read_offsets, int32_t *status, saru_batch *batch, void *stream) {
  set_last_error("");
  if (!c || !batch || !status || c->n < 0 || c->k < 0 || c->read_length < 1 || c->nreads < 0 ||
      (c->n > 0 && (!g.packed || !windows || !reads || !read_offsets || !c->read_table ||
                    !c->read_index || !c->positions || !c->dirs || !c->genome_offsets))) {
    set_last_error("gather: invalid call");
    return SARU_E_INVALID;
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    set_last_error(cudaGetErrorString(cudaGetLastError()));
    return SARU_E_CUDA;
  }
  GatherArgs a{};
  a.genome = nullptr;
  a.genome_len = g.len;
  a.packed = g.packed;
  a.exc_pos = g.exc_pos;
  a.exc_byte = g.exc_byte;
  a.nexc = g.nexc;
  a.table = reinterpret_cast<const uint8_t *>(c->read_table);
  a.nreads = c->nreads;
  a.read_index = c->read_index;
  a.positions = c->positions;
  a.goff = c->genome_offsets;
  a.dirs = c->dirs;
  a.n = c->n;
  a.genome_bytes = c->genome_bytes;
  a.m = c->read_length;
  a.k = c->k;
  a.windows = reinterpret_cast<uint8_t *>(windows);
  a.reads = reinterpret_cast<uint8_t *>(reads);
  a.read_offsets = read_offsets;
  a.status = status;
  const cudaError_t e = launch_gather(a, sms, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    return SARU_E_CUDA;
  }
  count_launch();
  *batch = saru_batch{windows, reads, c->genome_offsets, read_offsets, c->dirs, c->n, c->k,
                      c->match, c->mismatch, c->first_of_call, c->read_length, c->genome_bytes,
                      c->total_slots};
  return SARU_OK;
}

}  // namespace saru

extern "C" int saru_gather_device(const saru_gather_call *c, const char *genome,
                                  int64_t genome_len, char *windows, char *reads,
                                  int32_t *read_offsets, int32_t *status, saru_batch *batch,
                                  void *stream) {
  saru::set_last_error("");
  if (!c || !batch || !status || c->n < 0 || c->k < 0 || c->read_length < 1 || c->nreads < 0 ||
      (c->n > 0 && (!genome || !windows || !reads || !read_offsets || !c->read_table ||
                    !c->read_index || !c->positions || !c->dirs || !c->genome_offsets))) {
    saru::set_last_error("saru_gather_device: invalid call");
    return SARU_E_INVALID;
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    saru::set_last_error(cudaGetErrorString(cudaGetLastError()));
    return SARU_E_CUDA;
  }
  saru::GatherArgs a{};
  a.genome = reinterpret_cast<const uint8_t *>(genome);
  a.genome_len = genome_len;
  a.table = reinterpret_cast<const uint8_t *>(c->read_table);
  a.nreads = c->nreads;
  a.read_index = c->read_index;
  a.positions = c->positions;
  a.goff = c->genome_offsets;
  a.dirs = c->dirs;
  a.n = c->n;
  a.genome_bytes = c->genome_bytes;
  a.m = c->read_length;
  a.k = c->k;
  a.windows = reinterpret_cast<uint8_t *>(windows);
  a.reads = reinterpret_cast<uint8_t *>(reads);
  a.read_offsets = read_offsets;
  a.status = status;
  const cudaError_t e = saru::launch_gather(a, sms, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    saru::set_last_error(cudaGetErrorString(e));
    return SARU_E_CUDA;
  }
  saru::count_launch();
  *batch = saru_batch{windows, reads, c->genome_offsets, read_offsets, c->dirs, c->n, c->k,
                      c->match, c->mismatch, c->first_of_call, c->read_length, c->genome_bytes,
                      c->total_slots};
  return SARU_OK;
}
