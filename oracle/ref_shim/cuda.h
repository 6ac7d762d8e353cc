/*
 * Host-only stand-in for the CUDA headers, used ONLY to compile the
 * reference's own src/cuda-functions.cu as plain C++ for the oracle build
 * (oracle/_ref).  It is test infrastructure, never part of the product.
 *
 * The reference kernel (src/cuda-functions.cu:74-536) is ordinary C once
 * __global__/__device__ are erased and threadIdx/blockIdx become host
 * variables; its host code (:541-1120) only needs the handful of runtime and
 * driver calls declared below.  They are implemented over host memory in
 * oracle/ref_shim/emul_runtime.cpp, so "device" pointers are host pointers.
 */
#ifndef SARU_REF_SHIM_CUDA_H
#define SARU_REF_SHIM_CUDA_H

#include <stddef.h>

#define __global__
#define __device__
#define __host__

struct uint3 { unsigned int x, y, z; };
struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

/* The emulated launch sets these per emulated thread. */
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;

typedef int cudaError_t;
typedef int CUresult;
typedef int CUdevice;
typedef void *CUcontext;
enum { cudaSuccess = 0, CUDA_SUCCESS = 0 };
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3
};
struct cudaDeviceProp { char name[256]; };

cudaError_t cudaSetDevice(int dev);
cudaError_t cudaMalloc(void **p, size_t n);
cudaError_t cudaFree(void *p);
cudaError_t cudaMemset(void *p, int v, size_t n);
cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind k);
cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int dev);
CUresult cuInit(unsigned int flags);
CUresult cuDeviceGetCount(int *n);
CUresult cuDeviceGet(CUdevice *d, int i);
CUresult cuCtxCreate(CUcontext *c, unsigned int flags, CUdevice d);
CUresult cuMemGetInfo(size_t *free_b, size_t *total_b);
CUresult cuCtxDetach(CUcontext c);

/* The reference's launch `compute_score <<< blocks, threads >>> (...)` is
 * rewritten by the oracle recipe into a call of this serial launcher. */
void emul_launch_compute_score(int blocks, int threads, int match, int mismatch,
                               char *read_sequences, char *genome_sequences,
                               int *read_offsets, int *genome_offsets,
                               char *read_alignments, char *genome_alignments,
                               int sample_size, short int *edit_matrices,
                               int *edit_offsets, int *device_score_array,
                               char *direction_array, int error);

#endif
