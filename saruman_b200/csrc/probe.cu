// probe.cu -- measured integer-issue peak of the current GPU.
//
// The roofline of the banded kernel is integer issue (LOP3 / IADD / SHF
// work, no tensor-core contraction).  This probe runs eight independent
// chains of (lop3, add, funnel-shift) per thread at full occupancy and
// reports 32-bit integer operations per second, the denominator the
// benchmark uses for the kernel's roofline fraction.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/saruman_b200.h"

namespace {

__global__ void __launch_bounds__(256) int_issue_kernel(uint32_t *out, int iters, uint32_t y,
                                                        uint32_t z) {
  uint32_t x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = threadIdx.x * 0x9e3779b9u + blockIdx.x + c * 77u;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        x[c] = (x[c] & y) ^ z;              // one 3-input logic op
        x[c] = x[c] + y;                     // one add
        x[c] = __funnelshift_l(x[c], x[c], 7);  // one shift
      }
    }
  }
  uint32_t r = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) r ^= x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

}  // namespace

extern "C" double saru_int32_issue_probe(int iters) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 8;
  uint32_t *out = nullptr;
  if (cudaMalloc(&out, sizeof(uint32_t) * (size_t)threads * blocks) != cudaSuccess) return -1.0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int_issue_kernel<<<blocks, threads>>>(out, 8, 0x0f0f0f0fu, 0x12345678u);  // warm-up
  cudaEventRecord(a);
  int_issue_kernel<<<blocks, threads>>>(out, iters, 0x0f0f0f0fu, 0x12345678u);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
  const double ops = (double)threads * blocks * iters * 4.0 * 8.0 * 3.0;
  return ops / (ms * 1e-3);
}
