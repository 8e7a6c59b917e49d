// Interior dot product that allocates no device memory.
//
// Who needs this: a host model that hands the whole GPU memory to its own
// pool before the time loop starts, or that overlaps solver calls with work
// on other streams, cannot let a library call cudaMalloc/cudaFree inside the
// loop.  An allocation can fail once the pool owns the memory, and cudaFree
// synchronises the whole device, stalling every other stream.  The other
// entry points of this library allocate their scratch per call (the
// Fortran-compatible drop-ins) or per context (the native solver); this one
// keeps its scratch in a fixed array that is part of the loaded library.
//
// Scratch: one partial sum per grid row plus an arrival counter, in a
// file-scope device array of kNoAllocMaxRows + 32 doubles (about 128 KB).
// Every GPU that loads the library holds that array until the process
// exits.  Every call shares it and it keeps the last call's contents, so two
// calls that overlap on the GPU (different streams, no ordering between
// them) race on it and give wrong results; calls in one stream are ordered
// and safe.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kNoAllocMaxRows = 16384;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kRowsPerBlock = 8;  // one warp per row, 8 warps per CTA

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxRows + 32];

// The device address of g_noalloc_scratch for each device.  In host code the
// symbol name is only a host-side stand-in; a kernel must be given the
// address that cudaGetSymbolAddress returns with that device current.
double *g_scratch_ptr[kNoAllocMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Warp w of CTA b sums row j = b*8 + w of the interior (lanes stride over i,
// then a fixed-order shuffle tree) into scratch[j].  The last CTA to arrive
// adds scratch[0..j2-1]: thread t sums rows t, t + 256, ... in order, then a
// fixed-order shuffle and shared-memory tree combines the 256 sums, so the
// result does not depend on which CTA arrives last.
__global__ void __launch_bounds__(32 * kRowsPerBlock)
    k_inprod_rows(const double *r, const double *p, int i2, int j2, double *scratch,
                  double *result) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * kRowsPerBlock + w;
  const int i0 = i2 + 2;
  if (j < j2) {
    const size_t row = (size_t)(j + 1) * i0 + 1;  // padded (2..i2+1, j+2), 1-based
    double s = 0.0;
    for (int i = lane; i < i2; i += 32) s += r[row + i] * p[row + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) scratch[j] = s;
  }
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned *count = reinterpret_cast<unsigned *>(scratch + kNoAllocMaxRows);
    last = (atomicAdd(count, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double t = 0.0;
    for (int k = threadIdx.x; k < j2; k += blockDim.x) t += __ldcg(scratch + k);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __shared__ double warp_sums[kRowsPerBlock];
    if (lane == 0) warp_sums[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int k = 0; k < kRowsPerBlock; ++k) s += warp_sums[k];
      *result = s;
    }
  }
}

}  // namespace

// Declared in include/sevp_b200.h.
extern "C" int sevp_inprod_noalloc(const double *r, const double *p, int i2, int j2,
                                   double *result, void *stream) {
  if (!r || !p || !result || i2 < 1 || j2 < 1) return SEVP_BAD_ARG;
  if (j2 > kNoAllocMaxRows) {
    sevp_internal_set_message("sevp_inprod_noalloc: j2 exceeds the 16384 rows of its static scratch");
    return SEVP_BAD_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "cudaGetDevice", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    sevp_internal_set_message("sevp_inprod_noalloc: device index is 64 or more");
    return SEVP_BAD_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double *scratch = nullptr;
  {
    // first call on this device: look up the array's device address (a
    // runtime call that is not allowed while the stream is being captured)
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      e = cudaStreamIsCapturing(st, &cap);
      if (e == cudaSuccess && cap != cudaStreamCaptureStatusNone) {
        sevp_internal_set_message(
            "sevp_inprod_noalloc: the first call on a device must come before any stream "
            "capture (it looks up the scratch array's device address)");
        return SEVP_BAD_ARG;
      }
      e = cudaGetSymbolAddress((void **)&g_scratch_ptr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        sevp_internal_set_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
        return SEVP_CUDA_ERROR;
      }
    }
    scratch = g_scratch_ptr[dev];
  }
  // the arrival counter must start at zero; the partial sums are overwritten
  e = cudaMemsetAsync(scratch + kNoAllocMaxRows, 0, sizeof(double), st);
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "cudaMemsetAsync", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  const unsigned blocks = (unsigned)((j2 + kRowsPerBlock - 1) / kRowsPerBlock);
  k_inprod_rows<<<blocks, 32 * kRowsPerBlock, 0, st>>>(r, p, i2, j2, scratch, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "k_inprod_rows", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  return SEVP_OK;
}
