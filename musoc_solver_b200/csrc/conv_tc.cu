// 3x3 convolution (forward) of the warm-start U-Net on the fifth-generation
// tensor cores of sm_100a: tcgen05.mma with the FP32 accumulator in tensor
// memory (TMEM), operands staged in shared memory by cp.async.
//
// Implicit GEMM: D[p][n] = sum_{tap, k} In[p + shift(tap)][k] * Wk[tap][n][k]
// over a CTA tile of 128 consecutive output pixels (UMMA M = 128) and all
// output channels (UMMA N = cout <= 256), K = 16 per instruction.  Each
// pipeline step stages one tap and one chunk of kc input channels:
//   A: 128 pixels x kc channels, gathered at the tap's shifted positions
//      (zero outside the image),
//   B: cout x kc weights,
// both K-major in the no-swizzle core-matrix layout: an 8-row x 16-byte
// core matrix is 128 contiguous bytes; core matrices adjacent in K are 128 B
// apart (leading byte offset), adjacent in M/N kc*16 B apart (stride byte
// offset).  One thread issues the MMAs of a step and commits them to the
// stage's mbarrier; a stage is refilled only after that barrier completes.
// Loads run two steps ahead of the MMAs (four stages).
//
// Every wait on an mbarrier is bounded: on timeout the kernel records
// SEVP_TIMEOUT in a device flag (read by sevp_nn_tc_status), skips its
// stores, drains its copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <mutex>

#include "common.cuh"

typedef __nv_bfloat16 bf16;

namespace {

constexpr int kTcM = 128;        // pixels per CTA (UMMA M)
constexpr int kTcThreads = 128;  // 4 warps: warp w reads TMEM lanes 32w..32w+31
constexpr int kTcStages = 4;
constexpr int kTcAhead = kTcStages - 2;  // steps of loads in flight ahead of the MMAs
constexpr unsigned kSpinLimit = 1u << 22;

__device__ int g_tc_error;  // first error recorded by a tensor-core kernel
// Polls allowed to the producer and MMA-issuer waits of k_conv3x3_tma
// (sevp_nn_tc_set_wait_limit; the drains that follow a failure always use
// kSpinLimit, so every copy and MMA in flight completes before the CTA
// releases its shared memory and TMEM).
__device__ unsigned g_tc_wait_limit = kSpinLimit;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
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
// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity,
                                          unsigned limit = kSpinLimit) {
  for (unsigned k = 0; k < limit; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// Shared-memory matrix descriptor: no swizzle, K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}
// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__global__ void __launch_bounds__(kTcThreads)
    k_conv3x3_tc(const bf16 *__restrict__ in, int in_ld, int in_off, int cin,
                 const bf16 *__restrict__ wk, const float *__restrict__ bias, bf16 *__restrict__ out,
                 int out_ld, int out_off, int cout, int B, int H, int W, int relu, int kc,
                 uint32_t tmem_cols) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bars[kTcStages];
  __shared__ uint32_t s_tmem;
  __shared__ int s_py[kTcM], s_px[kTcM];
  __shared__ long long s_pimg[kTcM];  // first pixel of the row's image, -1 past the end
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long P = (long long)B * H * W;
  const long long p0 = (long long)blockIdx.x * kTcM;
  const int kc8 = kc >> 3;
  const uint32_t a_bytes = (uint32_t)kTcM * kc * 2, b_bytes = (uint32_t)cout * kc * 2;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  const uint32_t sbase = smem_u32(sm);
  const int nkc = cin / kc;
  const int T = 9 * nkc;
  const uint32_t core_sbo = (uint32_t)kc8 * 128;  // next 8 rows (M or N)

  {  // pixel coordinates of the tile's rows
    const long long p = p0 + tid;
    if (p < P) {
      const long long img = p / ((long long)H * W);
      const int rem = (int)(p - img * H * W);
      s_py[tid] = rem / W;
      s_px[tid] = rem - (rem / W) * W;
      s_pimg[tid] = img * H * W;
    } else {
      s_py[tid] = 0, s_px[tid] = 0, s_pimg[tid] = -1;
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) mbar_init(smem_u32(&bars[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  auto issue = [&](int s) {
    const int st = s % kTcStages;
    const int tap = s / nkc, c0 = (s - tap * nkc) * kc;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const uint32_t a_s = sbase + st * stage_bytes, b_s = a_s + a_bytes;
    for (int e = tid; e < kTcM * kc8; e += kTcThreads) {
      const int r = e / kc8, c = e - r * kc8;
      const int y = s_py[r] + dy, x = s_px[r] + dx;
      const bool ok = s_pimg[r] >= 0 && y >= 0 && y < H && x >= 0 && x < W;
      const bf16 *src =
          ok ? in + ((s_pimg[r] + (long long)y * W + x) * in_ld + in_off + c0 + c * 8) : in;
      cp_async16(a_s + (r >> 3) * core_sbo + c * 128 + (r & 7) * 16, src, ok);
    }
    for (int e = tid; e < cout * kc8; e += kTcThreads) {
      const int n = e / kc8, c = e - n * kc8;
      const bf16 *src = wk + ((size_t)tap * cout + n) * cin + c0 + c * 8;
      cp_async16(b_s + (n >> 3) * core_sbo + c * 128 + (n & 7) * 16, src, true);
    }
  };

  const uint32_t idesc = instr_desc_bf16(kTcM, cout);
  bool failed = false;
  for (int s = 0; s < kTcAhead && s < T; ++s) {
    issue(s);
    cp_async_commit();
  }
  for (int s = 0; s < T; ++s) {
    const int sn = s + kTcAhead;
    if (sn < T) {
      if (sn >= kTcStages) {  // the stage was last read by the MMAs of step sn - kTcStages
        const int sp = sn - kTcStages;
        if (!mbar_wait(smem_u32(&bars[sp % kTcStages]), (unsigned)(sp / kTcStages) & 1u))
          failed = true;
      }
      if (!failed) issue(sn);
    }
    cp_async_commit();
    cp_async_wait<kTcAhead>();  // this thread's copies of step s have landed
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const int st = s % kTcStages;
      const uint32_t a_s = sbase + st * stage_bytes, b_s = a_s + a_bytes;
      for (int k16 = 0; k16 < (kc >> 4); ++k16) {
        const uint64_t ad = smem_desc(a_s + k16 * 256, 128, core_sbo);
        const uint64_t bd = smem_desc(b_s + k16 * 256, 128, core_sbo);
        tc_mma(tmem, ad, bd, idesc, (s > 0 || k16 > 0) ? 1u : 0u);
      }
      tc_commit(smem_u32(&bars[st]));
    }
  }
  // all MMAs have completed once the last step's commit has arrived
  if (!mbar_wait(smem_u32(&bars[(T - 1) % kTcStages]), (unsigned)((T - 1) / kTcStages) & 1u))
    failed = true;
  cp_async_wait<0>();
  failed = __syncthreads_or(failed) != 0;  // a timeout anywhere voids the whole tile
  tc_fence_after();
  const long long p = p0 + warp * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
  for (int n0 = 0; n0 < cout; n0 += 16) {
    uint32_t v[16];
    tmem_ld16(tl + (uint32_t)n0, v);
    if (p < P && !failed) {
      __align__(16) bf16 o[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        float f = __uint_as_float(v[q]);
        if (bias) f += bias[n0 + q];
        if (relu) f = fmaxf(f, 0.f);
        o[q] = __float2bfloat16(f);
      }
      uint4 *dst = reinterpret_cast<uint4 *>(out + p * out_ld + out_off + n0);
      dst[0] = *reinterpret_cast<const uint4 *>(&o[0]);
      dst[1] = *reinterpret_cast<const uint4 *>(&o[8]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols)
                 : "memory");
  if (failed) atomicCAS(&g_tc_error, 0, SEVP_TIMEOUT);
}


// ------------------------------------------------ weight gradient
// dW[tap][ci][co] += sum_p X[p + shift(tap)][ci] * G[p][co] as an implicit
// GEMM on tcgen05: D[m][n] = sum_k A[m][k] B[n][k] with m = co (a block of
// 128 rows; rows past cout are zero), n = ci (all cin <= 256 channels), k =
// the pixels of this CTA's chunk, kWgK per pipeline step.  G is the packed
// output gradient [P][cout] (already masked by the ReLU).  Both operands lie
// channels-contiguous (NHWC) in memory, so the staging transposes them into
// the K-major no-swizzle core-matrix layout of k_conv3x3_tc: a thread loads
// 8 channels of two neighbouring pixels (two 16-byte loads) and writes eight
// 4-byte (k, k+1) pairs, one per row.  Thread 0 issues the K = 16 MMAs of a
// step and commits them to the stage's mbarrier; with kWgStages stages a
// stage is refilled while the MMAs of the two before it run.  The FP32 tile
// in TMEM is added to dW with atomics (the pixel chunks of a tap are spread
// over CTAs).  Waits are bounded as in k_conv3x3_tc.
constexpr int kWgStages = 3;
constexpr int kWgK = 64;  // pixels per step

__device__ __forceinline__ void store_k_pairs(unsigned char *base, int grp, int k, const uint4 &v0,
                                              const uint4 &v1) {
  // rows 8 grp .. 8 grp + 7, K elements k and k + 1 (k even)
  const uint16_t *a = reinterpret_cast<const uint16_t *>(&v0);
  const uint16_t *b = reinterpret_cast<const uint16_t *>(&v1);
  unsigned char *core = base + (k >> 3) * 128 + grp * (kWgK / 8 * 128) + (k & 7) * 2;
#pragma unroll
  for (int j = 0; j < 8; ++j)
    *reinterpret_cast<uint32_t *>(core + j * 16) = (uint32_t)a[j] | ((uint32_t)b[j] << 16);
}

__global__ void __launch_bounds__(kTcThreads)
    k_conv3x3_wgrad_tc(const bf16 *__restrict__ x, int x_ld, int x_off, int cin,
                       const bf16 *__restrict__ g, int cout, float *__restrict__ dw, int B, int H,
                       int W, long long ppc, uint32_t tmem_cols) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bars[kWgStages];
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long HW = (long long)H * W, P = (long long)B * HW;
  const int cob = (cout + 127) / 128;
  const int tap = blockIdx.y / cob, co0 = (blockIdx.y % cob) * 128;
  const int mrows = min(cout - co0, 128);
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const long long pb = (long long)blockIdx.x * ppc;
  const long long pe = min(P, pb + ppc);
  const int T = pe > pb ? (int)((pe - pb + kWgK - 1) / kWgK) : 0;
  constexpr uint32_t a_bytes = 128 * kWgK * 2;
  const uint32_t stage_bytes = a_bytes + (uint32_t)cin * kWgK * 2;
  const uint32_t sbase = smem_u32(sm);
  constexpr uint32_t core_sbo = kWgK / 8 * 128;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int q = 0; q < kWgStages; ++q) mbar_init(smem_u32(&bars[q]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // A rows past cout stay zero in every stage (8-row groups are 1 KB apart)
  for (int q = 0; q < kWgStages; ++q)
    for (uint32_t e = (uint32_t)(mrows / 8) * core_sbo + tid * 16; e < a_bytes; e += kTcThreads * 16)
      *reinterpret_cast<uint4 *>(sm + q * stage_bytes + e) = make_uint4(0, 0, 0, 0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  auto stage = [&](int s) {
    unsigned char *a_p = sm + (s % kWgStages) * stage_bytes;
    unsigned char *b_p = a_p + a_bytes;
    const long long k0 = pb + (long long)s * kWgK;
    const uint4 zero = make_uint4(0, 0, 0, 0);
    const int mg = mrows / 8, ng = cin / 8;
    for (int e = tid; e < (kWgK / 2) * mg; e += kTcThreads) {
      const int kp = e / mg, grp = e - kp * mg, k = 2 * kp;
      const long long p = k0 + k;
      const uint4 v0 = p < pe ? *reinterpret_cast<const uint4 *>(g + p * cout + co0 + grp * 8) : zero;
      const uint4 v1 =
          p + 1 < pe ? *reinterpret_cast<const uint4 *>(g + (p + 1) * cout + co0 + grp * 8) : zero;
      store_k_pairs(a_p, grp, k, v0, v1);
    }
    for (int e = tid; e < (kWgK / 2) * ng; e += kTcThreads) {
      const int kp = e / ng, grp = e - kp * ng, k = 2 * kp;
      uint4 v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long p = k0 + k + h;
        v[h] = zero;
        if (p < pe) {
          const long long img = p / HW;
          const int rem = (int)(p - img * HW);
          const int yy = rem / W + dy, xx = rem - (rem / W) * W + dx;
          if (yy >= 0 && yy < H && xx >= 0 && xx < W)
            v[h] = *reinterpret_cast<const uint4 *>(
                x + ((img * H + yy) * W + xx) * x_ld + x_off + grp * 8);
        }
      }
      store_k_pairs(b_p, grp, k, v[0], v[1]);
    }
  };

  const uint32_t idesc = instr_desc_bf16(128, cin);
  bool failed = false;
  int issued = 0;  // steps whose MMAs were committed
  for (int s = 0; s < T; ++s) {
    if (s >= kWgStages) {  // the stage was last read by the MMAs of step s - kWgStages
      const int sp = s - kWgStages;
      if (!mbar_wait(smem_u32(&bars[sp % kWgStages]), (unsigned)(sp / kWgStages) & 1u,
                     g_tc_wait_limit))
        failed = true;
    }
    if (__syncthreads_or(failed)) {
      failed = true;
      break;
    }
    stage(s);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_s = sbase + (uint32_t)(s % kWgStages) * stage_bytes, b_s = a_s + a_bytes;
#pragma unroll
      for (int k16 = 0; k16 < kWgK / 16; ++k16) {
        const uint64_t ad = smem_desc(a_s + k16 * 256, 128, core_sbo);
        const uint64_t bd = smem_desc(b_s + k16 * 256, 128, core_sbo);
        tc_mma(tmem, ad, bd, idesc, (s > 0 || k16 > 0) ? 1u : 0u);
      }
      tc_commit(smem_u32(&bars[s % kWgStages]));
    }
    issued = s + 1;
  }
  // every committed MMA has completed once the last commit has arrived (the
  // drain after a failure uses the full limit)
  if (issued > 0 &&
      !mbar_wait(smem_u32(&bars[(issued - 1) % kWgStages]), (unsigned)((issued - 1) / kWgStages) & 1u))
    failed = true;
  failed = __syncthreads_or(failed) != 0;
  tc_fence_after();
  if (issued > 0) {
    const int m = warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    for (int n0 = 0; n0 < cin; n0 += 16) {
      uint32_t v[16];
      tmem_ld16(tl + (uint32_t)n0, v);
      if (!failed && m < mrows) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
          atomicAdd(dw + ((size_t)tap * cin + n0 + q) * cout + co0 + m, __uint_as_float(v[q]));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols)
                 : "memory");
  if (failed) atomicCAS(&g_tc_error, 0, SEVP_TIMEOUT);
}


// ------------------------------------------------ TMA-fed variant (cin % 64 == 0)
// The same implicit GEMM with the operands brought in by the tensor memory
// accelerator: per step one 4-D tensor-map load of the tap-shifted A tile
// (64 channels x 128 pixels of one image row; the unit zero-fills outside the
// image, including negative coordinates) and one 2-D load of the tap's
// K-major weights (64 channels x cout), both in the 128-byte swizzle that the
// MMA's K-major SWIZZLE_128B descriptor reads (rows of 128 B, 8-row atoms
// 1024 B apart, a K step of 16 advances the start address by 32 B).  Warp 0
// lane 0 produces (TMA, full barriers with the byte count), warp 1 lane 0
// issues the MMAs and releases stages (empty barriers), all four warps run
// the epilogue.  The tiles are 128 consecutive pixels of one image row.
constexpr int kTmStages = 4;

// K-major swizzled descriptor for rows of KC BF16 (KC * 2 bytes = the
// swizzle width): 8-row atoms are 8 * KC * 2 bytes apart; layout type 2,
// 4, 6 = 128-, 64-, 32-byte swizzle.
template <int KC>
__device__ __forceinline__ uint64_t smem_desc_sw(uint32_t addr) {
  constexpr uint64_t layout = KC == 64 ? 2 : (KC == 32 ? 4 : 6);
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((8u * KC * 2u) >> 4) << 32;  // stride byte offset: next 8 rows
  d |= (uint64_t)1 << 46;                      // descriptor version of sm_100
  d |= layout << 61;
  return d;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}

template <int KC>
__global__ void __launch_bounds__(kTcThreads)
    k_conv3x3_tma(const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_w,
                  const float *__restrict__ bias, bf16 *__restrict__ out, int out_ld, int out_off,
                  int cin, int cout, int cout_total, int nsplit, int H, int W, int relu,
                  uint32_t tmem_cols) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  __shared__ __align__(8) uint64_t full[kTmStages], empty[kTmStages], done;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // a CTA computes cout output channels (slice `slice` of cout_total) of
  // 128 pixels of one image row
  const int x0 = blockIdx.x * kTcM, y = blockIdx.y, img = blockIdx.z / nsplit;
  const int slice = blockIdx.z - img * nsplit, n_base = slice * cout;
  const uint32_t raw = smem_u32(sm_raw);
  const uint32_t sbase = (raw + 1023u) & ~1023u;  // 1024-byte aligned stages
  const uint32_t a_bytes = (uint32_t)kTcM * KC * 2, b_bytes = (uint32_t)cout * KC * 2;
  const uint32_t tx_bytes = a_bytes + b_bytes;
  const uint32_t stage_bytes = (tx_bytes + 1023u) & ~1023u;  // stages 1024-byte aligned
  const int nkc = cin / KC, T = 9 * nkc;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < kTmStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  bool failed = false;
  int issued = 0;
  const unsigned wait_limit = g_tc_wait_limit;
  if (warp == 0 && lane == 0) {  // producer
    for (int s = 0; s < T; ++s) {
      const int st = s % kTmStages;
      if (s >= kTmStages &&
          !mbar_wait(smem_u32(&empty[st]), (unsigned)((s / kTmStages) - 1) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      const int tap = s / nkc, c0 = (s - tap * nkc) * KC;
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
      const uint32_t a_s = sbase + st * stage_bytes, bar = smem_u32(&full[st]);
      mbar_expect_tx(bar, tx_bytes);
      tma_load_4d(a_s, &tm_in, c0, x0 + dx, y + dy, img, bar);
      tma_load_2d(a_s + a_bytes, &tm_w, c0, tap * cout_total + n_base, bar);
      issued = s + 1;
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = instr_desc_bf16(kTcM, cout);
    for (int s = 0; s < T; ++s) {
      const int st = s % kTmStages;
      if (!mbar_wait(smem_u32(&full[st]), (unsigned)(s / kTmStages) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      tc_fence_after();
      const uint32_t a_s = sbase + st * stage_bytes, b_s = a_s + a_bytes;
#pragma unroll
      for (int k16 = 0; k16 < KC / 16; ++k16)
        tc_mma(tmem, smem_desc_sw<KC>(a_s + k16 * 32), smem_desc_sw<KC>(b_s + k16 * 32), idesc,
               (s > 0 || k16 > 0) ? 1u : 0u);
      tc_commit(smem_u32(&empty[st]));
    }
    // arrives once every MMA issued so far has completed (also after a
    // failed wait, so that none is left running when TMEM is freed)
    tc_commit(smem_u32(&done));
  }
  __syncwarp();
  if (!mbar_wait(smem_u32(&done), 0u)) failed = true;
  failed = __syncthreads_or(failed) != 0;
  if (failed && warp == 0 && lane == 0) {
    // drain the loads that may still be in flight (bounded) before the
    // shared memory they target is released
    for (int s = issued - kTmStages < 0 ? 0 : issued - kTmStages; s < issued; ++s)
      mbar_wait(smem_u32(&full[s % kTmStages]), (unsigned)(s / kTmStages) & 1u);
  }
  tc_fence_after();
  const int x = x0 + warp * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
  bf16 *dst_row = out + (((long long)img * H + y) * W + x) * out_ld + out_off + n_base;
  for (int n0 = 0; n0 < cout; n0 += 16) {
    uint32_t v[16];
    tmem_ld16(tl + (uint32_t)n0, v);
    if (x < W && !failed) {
      __align__(16) bf16 o[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        float f = __uint_as_float(v[q]);
        if (bias) f += bias[n_base + n0 + q];
        if (relu) f = fmaxf(f, 0.f);
        o[q] = __float2bfloat16(f);
      }
      uint4 *d = reinterpret_cast<uint4 *>(dst_row + n0);
      d[0] = *reinterpret_cast<const uint4 *>(&o[0]);
      d[1] = *reinterpret_cast<const uint4 *>(&o[8]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols)
                 : "memory");
  if (failed) atomicCAS(&g_tc_error, 0, SEVP_TIMEOUT);
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  });
  return fn;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

namespace {

// The TMA-fed forward convolution: same arguments and result as
// sevp_nn_conv3x3_tc.  Steps of 64 input channels (128-byte swizzle), or of
// cin = 32 / 16 channels (64- / 32-byte swizzle).
template <int KC>
int launch_conv_tma(const void *in, int in_ld, int in_off, int cin, const void *wk,
                           const float *bias, void *out, int out_ld, int out_off, int cout, int B,
                           int H, int W, int relu, void *stream,
                           PFN_cuTensorMapEncodeTiled_v12000 enc) {
  const CUtensorMapSwizzle sw = KC == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                         : (KC == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                     : CU_TENSOR_MAP_SWIZZLE_32B);
  // small layers (the deep levels of the network) get more CTAs by
  // splitting the output channels into slices of at least 64
  const long long ctas = (long long)((W + kTcM - 1) / kTcM) * H * B;
  int nsplit = 1;
  while (ctas * nsplit < 148 && cout / (nsplit * 2) >= 64 && (cout / (nsplit * 2)) % 16 == 0)
    nsplit *= 2;
  const int ncta = cout / nsplit;
  CUtensorMap tm_in, tm_w;
  {
    // activations: (channel, x, y, image), KC channels x 128 pixels per box
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)in_ld * 2, (cuuint64_t)W * in_ld * 2,
                                   (cuuint64_t)H * W * in_ld * 2};
    const cuuint32_t box[4] = {(cuuint32_t)KC, (cuuint32_t)kTcM, 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    if (enc(&tm_in, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)((const bf16 *)in + in_off), dims,
            strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return SEVP_BAD_ARG;
  }
  {
    // K-major weights (channel, tap * cout + n), KC channels x one slice of
    // the output channels per box
    const cuuint64_t dims[2] = {(cuuint64_t)cin, (cuuint64_t)9 * cout};
    const cuuint64_t strides[1] = {(cuuint64_t)cin * 2};
    const cuuint32_t box[2] = {(cuuint32_t)KC, (cuuint32_t)ncta};
    const cuuint32_t es[2] = {1, 1};
    if (enc(&tm_w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(wk), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return SEVP_BAD_ARG;
  }
  uint32_t cols = 32;
  while (cols < (uint32_t)ncta) cols <<= 1;
  const size_t stage = ((size_t)kTcM * KC * 2 + (size_t)ncta * KC * 2 + 1023) & ~(size_t)1023;
  const size_t smem = (size_t)kTmStages * stage + 1024;
  static size_t set_smem = 0;
  if (smem > set_smem) {
    SEVP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3_tma<KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    set_smem = smem;
  }
  dim3 grid((unsigned)((W + kTcM - 1) / kTcM), (unsigned)H, (unsigned)(B * nsplit));
  k_conv3x3_tma<KC><<<grid, kTcThreads, smem, (cudaStream_t)stream>>>(
      tm_in, tm_w, bias, (bf16 *)out, out_ld, out_off, cin, ncta, cout, nsplit, H, W, relu, cols);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

}  // namespace

extern "C" {

// out[p][out_off + n] = act(bias[n] + sum_{tap, k} in[p + shift(tap)][in_off + k] * wk[tap][n][k])
// with wk the K-major ([9][cout][cin]) weights.  cin in {16, 32, 64, 128, 256},
// cout a multiple of 16 up to 256, leading dimensions and offsets multiples
// of 8 channels, pointers 16-byte aligned.
int sevp_nn_conv3x3_tc(const void *in, int in_ld, int in_off, int cin, const void *wk,
                       const float *bias, void *out, int out_ld, int out_off, int cout, int B, int H,
                       int W, int relu, void *stream) {
  if (!in || !wk || !out || B < 1 || H < 1 || W < 1) return SEVP_BAD_ARG;
  if (!(cin == 16 || cin == 32 || cin == 64 || cin == 128 || cin == 256)) return SEVP_BAD_ARG;
  if (cout < 16 || cout > 256 || cout % 16) return SEVP_BAD_ARG;
  if ((in_ld % 8) || (in_off % 8) || (out_ld % 8) || (out_off % 8) || in_off + cin > in_ld ||
      out_off + cout > out_ld)
    return SEVP_BAD_ARG;
  if (!aligned16(in) || !aligned16(wk) || !aligned16(out)) return SEVP_BAD_ARG;
  const int kc = cin < 64 ? cin : 64;
  uint32_t cols = 32;
  while (cols < (uint32_t)cout) cols <<= 1;
  const size_t smem = (size_t)kTcStages * ((size_t)kTcM * kc * 2 + (size_t)cout * kc * 2);
  static size_t set_smem = 0;
  if (smem > set_smem) {
    SEVP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    set_smem = smem;
  }
  const long long P = (long long)B * H * W;
  const unsigned grid = (unsigned)((P + kTcM - 1) / kTcM);
  k_conv3x3_tc<<<grid, kTcThreads, smem, (cudaStream_t)stream>>>(
      (const bf16 *)in, in_ld, in_off, cin, (const bf16 *)wk, bias, (bf16 *)out, out_ld, out_off,
      cout, B, H, W, relu, kc, cols);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_conv3x3_tma(const void *in, int in_ld, int in_off, int cin, const void *wk,
                        const float *bias, void *out, int out_ld, int out_off, int cout, int B, int H,
                        int W, int relu, void *stream) {
  if (!in || !wk || !out || B < 1 || H < 1 || W < 1) return SEVP_BAD_ARG;
  if (!(cin == 16 || cin == 32 || cin == 64 || cin == 128 || cin == 192 || cin == 256))
    return SEVP_BAD_ARG;
  if (cout < 16 || cout > 256 || cout % 16) return SEVP_BAD_ARG;
  if ((in_ld % 8) || (in_off % 8) || (out_ld % 8) || (out_off % 8) || in_off + cin > in_ld ||
      out_off + cout > out_ld)
    return SEVP_BAD_ARG;
  if (!aligned16(in) || !aligned16(wk) || !aligned16(out)) return SEVP_BAD_ARG;
  auto enc = tensor_map_encoder();
  if (!enc) return SEVP_CUDA_ERROR;
  if (cin == 16)
    return launch_conv_tma<16>(in, in_ld, in_off, cin, wk, bias, out, out_ld, out_off, cout, B, H, W,
                               relu, stream, enc);
  if (cin == 32)
    return launch_conv_tma<32>(in, in_ld, in_off, cin, wk, bias, out, out_ld, out_off, cout, B, H, W,
                               relu, stream, enc);
  return launch_conv_tma<64>(in, in_ld, in_off, cin, wk, bias, out, out_ld, out_off, cout, B, H, W,
                             relu, stream, enc);
}

// dw[tap][ci][co] += sum_p x[p + shift(tap)][x_off + ci] * g[p][co] (FP32),
// with g the packed output gradient [B*H*W][cout] (already masked by the
// ReLU).  cin and cout multiples of 16 up to 256; x_ld and x_off multiples
// of 8; x and g 16-byte aligned.
int sevp_nn_conv3x3_wgrad_tc(const void *x, int x_ld, int x_off, int cin, const void *g, int cout,
                             float *dw, int B, int H, int W, void *stream) {
  if (!x || !g || !dw || B < 1 || H < 1 || W < 1) return SEVP_BAD_ARG;
  if (cin < 16 || cin > 256 || cin % 16 || cout < 16 || cout > 256 || cout % 16)
    return SEVP_BAD_ARG;
  if ((x_ld % 8) || (x_off % 8) || x_off + cin > x_ld || !aligned16(x) || !aligned16(g))
    return SEVP_BAD_ARG;
  const long long P = (long long)B * H * W;
  const int cob = (cout + 127) / 128;
  // enough CTAs to cover the GPU twice, each with whole steps of kWgK pixels
  long long chunks = (2LL * 148 + 9LL * cob - 1) / (9LL * cob);
  long long ppc = (P + chunks - 1) / chunks;
  ppc = (ppc + kWgK - 1) / kWgK * kWgK;
  chunks = (P + ppc - 1) / ppc;
  uint32_t cols = 32;
  while (cols < (uint32_t)cin) cols <<= 1;
  const size_t smem = (size_t)kWgStages * (128 * kWgK * 2 + (size_t)cin * kWgK * 2);
  static size_t set_smem = 0;
  if (smem > set_smem) {
    SEVP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3_wgrad_tc,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set_smem = smem;
  }
  dim3 grid((unsigned)chunks, (unsigned)(9 * cob));
  k_conv3x3_wgrad_tc<<<grid, kTcThreads, smem, (cudaStream_t)stream>>>(
      (const bf16 *)x, x_ld, x_off, cin, (const bf16 *)g, cout, dw, B, H, W, ppc, cols);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_tc_set_wait_limit(unsigned limit) {
  const unsigned v = limit == 0xFFFFFFFFu ? kSpinLimit : limit;
  SEVP_CUDA_TRY(cudaMemcpyToSymbol(g_tc_wait_limit, &v, sizeof(unsigned)));
  SEVP_CUDA_TRY(cudaDeviceSynchronize());
  return SEVP_OK;
}

// First error a tensor-core kernel recorded since the last call (0 if none);
// resets the flag.  Synchronises the device.
int sevp_nn_tc_status(int *code) {
  if (!code) return SEVP_BAD_ARG;
  int v = 0, zero = 0;
  SEVP_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
  SEVP_CUDA_TRY(cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)));
  *code = v;
  return SEVP_OK;
}

}  // extern "C"
