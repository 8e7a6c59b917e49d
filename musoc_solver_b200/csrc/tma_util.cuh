// Tensor-memory-accelerator plumbing shared by the TMA-staged passes:
// mbarrier waits with an iteration bound, 2-D tensor copies, plain bulk
// copies, and the host-side encoding of 2-D tensor maps.  Only this GPU's
// memory is read, and no copy uses cluster multicast.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace sevp {
namespace tma {

// Polls of an mbarrier before a wait gives up.
constexpr unsigned kWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory
// before its later async-proxy ones (a buffer that was read is refilled).
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// true once the phase with this parity completed; false after kWaitLimit polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity) {
  for (unsigned k = 0; k < kWaitLimit; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}
// 2-D tensor copy of the box at (c0, c1) (c0 * element size a multiple of
// 16 bytes) into shared memory; completes bytes on bar.
__device__ __forceinline__ void load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                        uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}
// Plain bulk copy (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void load_bulk(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1], %2, [%3];\n" ::"r"(dst),
      "l"((uint64_t)src), "r"(bytes), "r"(bar)
      : "memory");
}

inline PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult qr{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &qr) ==
            cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  });
  return fn;
}

// A 2-D tensor map of an (nx, ny) row-major plane with the given box;
// points outside the plane arrive as zeros.
inline bool encode(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *m, const void *base,
                   bool fp64, int nx, int ny, int bw, int bh) {
  const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
  const cuuint64_t strides[1] = {(cuuint64_t)nx * (fp64 ? 8 : 4)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
             const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace tma
}  // namespace sevp
