// Shared helpers for the sm_100a SEVP library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/sevp_b200.h"

#define SEVP_CUDA_TRY(call)                                                      \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      sevp_internal_set_error(e_, #call, __FILE__, __LINE__);                    \
      return SEVP_CUDA_ERROR;                                                    \
    }                                                                            \
  } while (0)

void sevp_internal_set_error(cudaError_t e, const char *what, const char *file, int line);
void sevp_internal_set_message(const char *msg);
// Status that sevp_last_status() reports for the Fortran-compatible calls.
void sevp_internal_set_status(int status);

namespace sevp {

constexpr int kWarp = 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV doubles; result valid in thread 0.  smem needs
// NV * (blockDim/32) doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x * blockDim.y * blockDim.z) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[k * nw + wid] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += smem[k * nw + w];
      v[k] = s;
    }
  }
}

template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
  return __ldg(p);
}

// Streaming load that is not kept in L1 (data read exactly once).
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace sevp
