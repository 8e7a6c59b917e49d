// BF16 convolution-network kernels of the learned warm start: 3x3 and 1x1
// convolutions (forward, data gradient, weight gradient) as implicit GEMMs on
// the tensor cores (BF16 operands, FP32 accumulation), 2x2 average pooling,
// nearest 2x upsampling, ReLU backward, the loss, and Adam on FP32 master
// weights.  The network itself (a 4-level U-Net) is assembled by the caller
// from these entry points; none of this exists in the reference.
//
// Activations are NHWC BF16 tensors [B][H][W][ld] where a layer's C channels
// sit at channel offset `off` (so a decoder's concatenated input is one
// buffer that two producers write).  Weights of a 3x3 conv are
// [9 taps][Cin][Cout] (tap = 3*(dy+1) + (dx+1)); Cin and Cout are multiples
// of 16.  Zero padding at the image edges.
#include <cuda_bf16.h>
#include <mma.h>

#include "../../include/sevp_nn.h"
#include "common.cuh"

using namespace nvcuda;
typedef __nv_bfloat16 bf16;

namespace {

constexpr int kTM = 64;   // pixels per CTA tile
constexpr int kTN = 64;   // output channels per CTA tile
constexpr int kTK = 16;   // reduction chunk (input channels of one tap)

// out[p][co] (+)= sum_{tap, ci} in[p + shift(tap)][ci] * w[tap][ci][co]
// FLIP: use the tap mirrored (data gradient) and w laid out [tap][co][ci]
// i.e. the transposed weight (so the same loop computes dX from dY).
template <bool FLIP>
__global__ void __launch_bounds__(128)
    k_conv3x3(const bf16 *__restrict__ in, int in_ld, int in_off, int cin,
              const bf16 *__restrict__ w, const float *__restrict__ bias, bf16 *__restrict__ out,
              int out_ld, int out_off, int cout, int B, int H, int W, int relu,
              const bf16 *__restrict__ mask, int mask_ld, int mask_off) {
  __shared__ __align__(32) bf16 sA[kTM * (kTK + 8)];
  __shared__ __align__(32) bf16 sB[kTK * (kTN + 8)];
  __shared__ __align__(32) float sC[kTM * (kTN + 4)];
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long P = (long long)B * H * W;
  const long long p0 = (long long)blockIdx.x * kTM;
  const int n0 = blockIdx.y * kTN;
  const int wm = warp >> 1, wn = warp & 1;  // 2x2 warps, 32x32 each
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) wmma::fill_fragment(acc[a][b], 0.f);
  // pixel coordinates of the two pixels this thread loads (64 px x 16 ch,
  // 8 channels = 16 B per load)
  const int lp = tid >> 1, lc = (tid & 1) * 8;
  const long long pp = p0 + lp;
  int py = 0, px = 0, pb = 0;
  bool pin = pp < P;
  if (pin) {
    pb = (int)(pp / ((long long)H * W));
    int r = (int)(pp - (long long)pb * H * W);
    py = r / W;
    px = r - py * W;
  }
  for (int tap = 0; tap < 9; ++tap) {
    const int t2 = FLIP ? 8 - tap : tap;
    const int dy = t2 / 3 - 1, dx = t2 % 3 - 1;
    const int sy = py + dy, sx = px + dx;
    const bool ok = pin && sy >= 0 && sy < H && sx >= 0 && sx < W;
    const long long spix = ((long long)pb * H + sy) * W + sx;
    for (int c0 = 0; c0 < cin; c0 += kTK) {
      // A: 64 pixels x 16 channels
      uint4 va = make_uint4(0, 0, 0, 0);
      if (ok) {
        va = *reinterpret_cast<const uint4 *>(in + spix * in_ld + in_off + c0 + lc);
        if (mask) {
          // data gradient: dY masked by the ReLU of its forward output
          uint4 vm = *reinterpret_cast<const uint4 *>(mask + spix * mask_ld + mask_off + c0 + lc);
          bf16 *a = reinterpret_cast<bf16 *>(&va);
          const bf16 *m = reinterpret_cast<const bf16 *>(&vm);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (!(__bfloat162float(m[q]) > 0.f)) a[q] = __float2bfloat16(0.f);
        }
      }
      *reinterpret_cast<uint4 *>(&sA[lp * (kTK + 8) + lc]) = va;
      // B: 16 input channels x 64 output channels
      {
        const int kr = tid >> 3, kc = (tid & 7) * 8;  // 16 rows x 8 chunks of 8
        const bf16 *src = w + ((size_t)tap * cin + c0 + kr) * cout + n0 + kc;
        uint4 vb = make_uint4(0, 0, 0, 0);
        if (n0 + kc < cout) vb = *reinterpret_cast<const uint4 *>(src);
        *reinterpret_cast<uint4 *>(&sB[kr * (kTN + 8) + kc]) = vb;
      }
      __syncthreads();
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> fa[2];
      wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb[2];
#pragma unroll
      for (int a = 0; a < 2; ++a)
        wmma::load_matrix_sync(fa[a], &sA[(wm * 32 + a * 16) * (kTK + 8)], kTK + 8);
#pragma unroll
      for (int b = 0; b < 2; ++b)
        wmma::load_matrix_sync(fb[b], &sB[wn * 32 + b * 16], kTN + 8);
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) wmma::mma_sync(acc[a][b], fa[a], fb[b], acc[a][b]);
      __syncthreads();
    }
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
      wmma::store_matrix_sync(&sC[(wm * 32 + a * 16) * (kTN + 4) + wn * 32 + b * 16], acc[a][b],
                              kTN + 4, wmma::mem_row_major);
  __syncthreads();
  for (int e = tid; e < kTM * kTN; e += 128) {
    const int r = e / kTN, c = e % kTN;
    const long long p = p0 + r;
    const int co = n0 + c;
    if (p >= P || co >= cout) continue;
    float v = sC[r * (kTN + 4) + c];
    if (bias) v += bias[co];
    if (relu) v = fmaxf(v, 0.f);
    out[p * out_ld + out_off + co] = __float2bfloat16(v);
  }
}

// dW[tap][ci][co] += sum_p X[p + shift(tap)][ci] * dY[p][co] over one pixel
// chunk (FP32 atomics into the master-gradient buffer).  dY is masked by the
// ReLU of the forward output when mask is given.  CTA: one tap, 32 input
// channels x 64 output channels, 4 warps (2 x 2 of 16 x 32).
constexpr int kWP = 16;  // pixels per reduction step
__global__ void __launch_bounds__(128)
    k_conv3x3_wgrad(const bf16 *__restrict__ x, int x_ld, int x_off, int cin,
                    const bf16 *__restrict__ dy, int dy_ld, int dy_off, int cout,
                    const bf16 *__restrict__ mask, int mask_ld, int mask_off, float *__restrict__ dw,
                    int B, int H, int W, long long pix_per_cta) {
  __shared__ __align__(32) bf16 sX[kWP * (32 + 8)];  // [pixel][ci]
  __shared__ __align__(32) bf16 sY[kWP * (64 + 8)];  // [pixel][co]
  __shared__ __align__(32) float sC[32 * (64 + 4)];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tap = blockIdx.z % 9;
  const int c0 = (blockIdx.z / 9) * 32;
  const int n0 = blockIdx.y * 64;
  const long long P = (long long)B * H * W;
  const long long pbeg = (long long)blockIdx.x * pix_per_cta;
  const long long pend = min(P, pbeg + pix_per_cta);
  const int dyy = tap / 3 - 1, dxx = tap % 3 - 1;
  const int wm = warp >> 1, wn = warp & 1;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2];
  wmma::fill_fragment(acc[0], 0.f);
  wmma::fill_fragment(acc[1], 0.f);
  for (long long pq = pbeg; pq < pend; pq += kWP) {
    // X: 16 pixels x 32 channels (4 chunks of 8 per pixel -> 64 loads), dY: 16 x 64 (128 loads)
    if (tid < 64) {
      const int lp = tid >> 2, lc = (tid & 3) * 8;
      const long long p = pq + lp;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p < pend) {
        const int b = (int)(p / ((long long)H * W));
        const int r = (int)(p - (long long)b * H * W);
        const int py = r / W, px = r - (r / W) * W;
        const int sy = py + dyy, sx = px + dxx;
        if (sy >= 0 && sy < H && sx >= 0 && sx < W && c0 + lc < cin)
          v = *reinterpret_cast<const uint4 *>(x + (((long long)b * H + sy) * W + sx) * x_ld + x_off +
                                               c0 + lc);
      }
      *reinterpret_cast<uint4 *>(&sX[lp * (32 + 8) + lc]) = v;
    }
    {
      const int lp = tid >> 3, lc = (tid & 7) * 8;
      const long long p = pq + lp;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p < pend && n0 + lc < cout) {
        v = *reinterpret_cast<const uint4 *>(dy + p * dy_ld + dy_off + n0 + lc);
        if (mask) {
          uint4 vm = *reinterpret_cast<const uint4 *>(mask + p * mask_ld + mask_off + n0 + lc);
          bf16 *a = reinterpret_cast<bf16 *>(&v);
          const bf16 *m = reinterpret_cast<const bf16 *>(&vm);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (!(__bfloat162float(m[q]) > 0.f)) a[q] = __float2bfloat16(0.f);
        }
      }
      *reinterpret_cast<uint4 *>(&sY[lp * (64 + 8) + lc]) = v;
    }
    __syncthreads();
    // A = X^T (m = ci, k = pixel): stored [k][m] -> column-major
    wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> fa;
    wmma::load_matrix_sync(fa, &sX[wm * 16], 32 + 8);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb;
      wmma::load_matrix_sync(fb, &sY[wn * 32 + b * 16], 64 + 8);
      wmma::mma_sync(acc[b], fa, fb, acc[b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 2; ++b)
    wmma::store_matrix_sync(&sC[(wm * 16) * (64 + 4) + wn * 32 + b * 16], acc[b], 64 + 4,
                            wmma::mem_row_major);
  __syncthreads();
  for (int e = tid; e < 32 * 64; e += 128) {
    const int r = e / 64, c = e % 64;
    if (c0 + r < cin && n0 + c < cout)
      atomicAdd(&dw[((size_t)tap * cin + c0 + r) * cout + n0 + c], sC[r * (64 + 4) + c]);
  }
}

// db[co] += sum_p dY[p][co] (masked)
__global__ void k_bias_grad(const bf16 *dy, int dy_ld, int dy_off, int cout, const bf16 *mask,
                            int mask_ld, int mask_off, float *db, long long P) {
  const int co = blockIdx.y * blockDim.x + threadIdx.x;
  if (co >= cout) return;
  float s = 0.f;
  for (long long p = blockIdx.x; p < P; p += gridDim.x) {
    float v = __bfloat162float(dy[p * dy_ld + dy_off + co]);
    if (mask && !(__bfloat162float(mask[p * mask_ld + mask_off + co]) > 0.f)) v = 0.f;
    s += v;
  }
  atomicAdd(&db[co], s);
}

// transposed, tap-mirrored copy for the data gradient: wt[tap][co][ci] = w[tap][ci][co]
__global__ void k_weight_transpose(const bf16 *w, bf16 *wt, int cin, int cout) {
  const size_t n = (size_t)9 * cin * cout;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int tap = (int)(e / ((size_t)cin * cout));
    const int rem = (int)(e % ((size_t)cin * cout));
    const int ci = rem / cout, co = rem % cout;
    wt[((size_t)tap * cout + co) * cin + ci] = w[e];
  }
}

// Tap-mirrored copy for the data gradient on the tensor cores:
// wm[tap][ci][co] = w[8 - tap][ci][co].  Read as the [tap][n][k] weights of
// a forward convolution from co input to ci output channels, it gives
// dX[p][ci] = sum_{tap, co} dY[p + shift(tap)][co] w[8 - tap][ci][co].
__global__ void k_weight_mirror(const bf16 *w, bf16 *wm, int cin, int cout) {
  const size_t per_tap = (size_t)cin * cout, n = 9 * per_tap;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t tap = e / per_tap;
    wm[e] = w[(8 - tap) * per_tap + e % per_tap];
  }
}

// Output gradient through the ReLU of the forward output, packed:
// out[p][c] = mask[p][c] > 0 ? dy[p][c] : 0 (c < C), or dy itself when mask
// is null.  8 channels per thread.
__global__ void k_relu_mask8(const bf16 *dy, int dy_ld, int dy_off, const bf16 *mask, int mask_ld,
                             int mask_off, int C8, bf16 *out, long long P) {
  const long long n = P * C8;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / C8;
    const int c = (int)(e % C8) * 8;
    uint4 g = *reinterpret_cast<const uint4 *>(dy + p * dy_ld + dy_off + c);
    if (mask) {
      const uint4 m = *reinterpret_cast<const uint4 *>(mask + p * mask_ld + mask_off + c);
      const bf16 *mv = reinterpret_cast<const bf16 *>(&m);
      bf16 *gv = reinterpret_cast<bf16 *>(&g);
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (!(__bfloat162float(mv[k]) > 0.f)) gv[k] = __float2bfloat16(0.f);
    }
    *reinterpret_cast<uint4 *>(out + p * (long long)C8 * 8 + c) = g;
  }
}

// 2x2 average pooling (H, W even)
__global__ void k_pool_fwd(const bf16 *in, int in_ld, int in_off, bf16 *out, int out_ld,
                           int out_off, int C, int B, int H, int W) {
  const int Ho = H / 2, Wo = W / 2;
  const long long n = (long long)B * Ho * Wo * C;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const long long q = e / C;
    const int x = (int)(q % Wo), y = (int)((q / Wo) % Ho), b = (int)(q / ((long long)Wo * Ho));
    const long long p = ((long long)b * H + 2 * y) * W + 2 * x;
    float s = __bfloat162float(in[p * in_ld + in_off + c]) +
              __bfloat162float(in[(p + 1) * in_ld + in_off + c]) +
              __bfloat162float(in[(p + W) * in_ld + in_off + c]) +
              __bfloat162float(in[(p + W + 1) * in_ld + in_off + c]);
    out[q * out_ld + out_off + c] = __float2bfloat16(0.25f * s);
  }
}
// dIn (+)= dOut / 4 broadcast; accumulate != 0 adds to the existing gradient
__global__ void k_pool_bwd(const bf16 *dout, int dout_ld, int dout_off, bf16 *din, int din_ld,
                           int din_off, int C, int B, int H, int W, int accumulate) {
  const long long n = (long long)B * H * W * C;
  const int Ho = H / 2, Wo = W / 2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const long long p = e / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const long long q = ((long long)b * Ho + y / 2) * Wo + x / 2;
    float v = 0.25f * __bfloat162float(dout[q * dout_ld + dout_off + c]);
    if (accumulate) v += __bfloat162float(din[p * din_ld + din_off + c]);
    din[p * din_ld + din_off + c] = __float2bfloat16(v);
  }
}
// nearest 2x upsampling (output H x W, input H/2 x W/2)
__global__ void k_up_fwd(const bf16 *in, int in_ld, int in_off, bf16 *out, int out_ld, int out_off,
                         int C, int B, int H, int W) {
  const long long n = (long long)B * H * W * C;
  const int Hi = H / 2, Wi = W / 2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const long long p = e / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const long long q = ((long long)b * Hi + y / 2) * Wi + x / 2;
    out[p * out_ld + out_off + c] = in[q * in_ld + in_off + c];
  }
}
// dIn = sum of the 4 output gradients (input H/2 x W/2)
__global__ void k_up_bwd(const bf16 *dout, int dout_ld, int dout_off, bf16 *din, int din_ld,
                         int din_off, int C, int B, int H, int W) {
  const int Hi = H / 2, Wi = W / 2;
  const long long n = (long long)B * Hi * Wi * C;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const long long q = e / C;
    const int x = (int)(q % Wi), y = (int)((q / Wi) % Hi), b = (int)(q / ((long long)Wi * Hi));
    const long long p = ((long long)b * H + 2 * y) * W + 2 * x;
    float s = __bfloat162float(dout[p * dout_ld + dout_off + c]) +
              __bfloat162float(dout[(p + 1) * dout_ld + dout_off + c]) +
              __bfloat162float(dout[(p + W) * dout_ld + dout_off + c]) +
              __bfloat162float(dout[(p + W + 1) * dout_ld + dout_off + c]);
    din[q * din_ld + din_off + c] = __float2bfloat16(s);
  }
}

// 1x1 head: y[p] = sum_c x[p][c] * w[c] + b (C <= 256), FP32 output
__global__ void k_head_fwd(const bf16 *x, int x_ld, int x_off, int C, const float *w,
                           const float *b, float *y, long long P) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    float s = b[0];
    for (int c = 0; c < C; ++c) s += __bfloat162float(x[p * x_ld + x_off + c]) * w[c];
    y[p] = s;
  }
}
// 8-channel (16-byte) versions of the forward pooling, upsampling and head,
// used when channel counts, leading dimensions and offsets are multiples of
// 8: the same arithmetic in the same order as the one-element kernels.
__device__ __forceinline__ void bf8_to_f(const uint4 &v, float (&f)[8]) {
  const bf16 *h = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
  for (int q = 0; q < 8; ++q) f[q] = __bfloat162float(h[q]);
}
__global__ void k_pool_fwd8(const bf16 *in, int in_ld, int in_off, bf16 *out, int out_ld,
                            int out_off, int C8, int B, int H, int W) {
  const int Ho = H / 2, Wo = W / 2;
  const long long n = (long long)B * Ho * Wo * C8;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C8) * 8;
    const long long q = e / C8;
    const int x = (int)(q % Wo);
    const long long t = q / Wo;
    const int y = (int)(t % Ho);
    const long long b = t / Ho;
    const long long p = (b * H + 2 * y) * W + 2 * x;
    float a[8], b1[8], c1[8], d[8];
    bf8_to_f(*reinterpret_cast<const uint4 *>(in + p * in_ld + in_off + c), a);
    bf8_to_f(*reinterpret_cast<const uint4 *>(in + (p + 1) * in_ld + in_off + c), b1);
    bf8_to_f(*reinterpret_cast<const uint4 *>(in + (p + W) * in_ld + in_off + c), c1);
    bf8_to_f(*reinterpret_cast<const uint4 *>(in + (p + W + 1) * in_ld + in_off + c), d);
    __align__(16) bf16 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __float2bfloat16(0.25f * (((a[k] + b1[k]) + c1[k]) + d[k]));
    *reinterpret_cast<uint4 *>(out + q * out_ld + out_off + c) = *reinterpret_cast<const uint4 *>(o);
  }
}
// one thread per input pixel and 8 channels: writes the four output pixels
__global__ void k_up_fwd8(const bf16 *in, int in_ld, int in_off, bf16 *out, int out_ld, int out_off,
                          int C8, int B, int H, int W) {
  const int Hi = H / 2, Wi = W / 2;
  const long long n = (long long)B * Hi * Wi * C8;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C8) * 8;
    const long long q = e / C8;
    const int x = (int)(q % Wi);
    const long long t = q / Wi;
    const int y = (int)(t % Hi);
    const long long b = t / Hi;
    const uint4 v = *reinterpret_cast<const uint4 *>(in + q * in_ld + in_off + c);
    const long long p = (b * H + 2 * y) * W + 2 * x;
    *reinterpret_cast<uint4 *>(out + p * out_ld + out_off + c) = v;
    *reinterpret_cast<uint4 *>(out + (p + 1) * out_ld + out_off + c) = v;
    *reinterpret_cast<uint4 *>(out + (p + W) * out_ld + out_off + c) = v;
    *reinterpret_cast<uint4 *>(out + (p + W + 1) * out_ld + out_off + c) = v;
  }
}
__global__ void k_head_fwd8(const bf16 *x, int x_ld, int x_off, int C, const float *w,
                            const float *b, float *y, long long P) {
  __shared__ float sw[256];
  for (int c = threadIdx.x; c < C; c += blockDim.x) sw[c] = w[c];
  __syncthreads();
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    float s = b[0];
    for (int c = 0; c < C; c += 8) {
      float f[8];
      bf8_to_f(*reinterpret_cast<const uint4 *>(x + p * x_ld + x_off + c), f);
#pragma unroll
      for (int k = 0; k < 8; ++k) s += f[k] * sw[c + k];
    }
    y[p] = s;
  }
}
// head backward: dx[p][c] = dy[p] * w[c] (bf16); dw[c] += sum_p dy[p] x[p][c]; db += sum dy
__global__ void k_head_bwd(const bf16 *x, int x_ld, int x_off, int C, const float *w,
                           const float *dy, bf16 *dx, int dx_ld, int dx_off, float *dw, float *db,
                           long long P) {
  __shared__ float sw[256 + 1];
  for (int c = threadIdx.x; c <= C; c += blockDim.x) sw[c] = 0.f;
  __syncthreads();
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const float g = dy[p];
    for (int c = 0; c < C; ++c) {
      dx[p * dx_ld + dx_off + c] = __float2bfloat16(g * w[c]);
      atomicAdd(&sw[c], g * __bfloat162float(x[p * x_ld + x_off + c]));
    }
    atomicAdd(&sw[C], g);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&dw[c], sw[c]);
  if (threadIdx.x == 0) atomicAdd(db, sw[C]);
}

// loss = mean (y - t)^2 over valid pixels; dy = 2 (y - t) / n
__global__ void k_mse(const float *y, const float *t, const float *valid, float *dy, float *loss,
                      long long P, float inv_n) {
  float s = 0.f;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const float m = valid ? valid[p] : 1.f;
    const float d = (y[p] - t[p]) * m;
    dy[p] = 2.f * d * inv_n;
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_n);
}

// Adam on FP32 master weights; writes the BF16 working copy (or FP32 copy).
__global__ void k_adam(float *w, const float *g, float *m, float *v, bf16 *w16, float *w32, size_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2, float wd) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const float gk = g[k] + wd * w[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + eps);
    w[k] = wk;
    if (w16) w16[k] = __float2bfloat16(wk);
    if (w32) w32[k] = wk;
  }
}

__global__ void k_f32_to_bf16(const float *a, bf16 *b, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    b[k] = __float2bfloat16(a[k]);
}

unsigned ew_grid(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
}

bool bad_channels(int c) { return c < 16 || (c % 16) != 0; }

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int sevp_nn_conv3x3(const void *in, int in_ld, int in_off, int cin, const void *w,
                    const float *bias, void *out, int out_ld, int out_off, int cout, int B, int H,
                    int W, int relu, const void *mask, int mask_ld, int mask_off, int flip,
                    void *stream) {
  if (!in || !w || !out || bad_channels(cin) || bad_channels(cout) || B < 1 || H < 1 || W < 1 ||
      (in_ld % 8) || (in_off % 8) || (mask && ((mask_ld % 8) || (mask_off % 8))))
    return SEVP_BAD_ARG;
  const long long P = (long long)B * H * W;
  dim3 grid((unsigned)((P + kTM - 1) / kTM), (unsigned)((cout + kTN - 1) / kTN));
  cudaStream_t st = (cudaStream_t)stream;
  if (flip)
    k_conv3x3<true><<<grid, 128, 0, st>>>((const bf16 *)in, in_ld, in_off, cin, (const bf16 *)w, bias,
                                          (bf16 *)out, out_ld, out_off, cout, B, H, W, relu,
                                          (const bf16 *)mask, mask_ld, mask_off);
  else
    k_conv3x3<false><<<grid, 128, 0, st>>>((const bf16 *)in, in_ld, in_off, cin, (const bf16 *)w, bias,
                                           (bf16 *)out, out_ld, out_off, cout, B, H, W, relu,
                                           (const bf16 *)mask, mask_ld, mask_off);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_conv3x3_wgrad(const void *x, int x_ld, int x_off, int cin, const void *dy, int dy_ld,
                          int dy_off, int cout, const void *mask, int mask_ld, int mask_off,
                          float *dw, float *db, int B, int H, int W, void *stream) {
  if (!x || !dy || !dw || bad_channels(cin) || bad_channels(cout) || (x_ld % 8) || (x_off % 8) ||
      (dy_ld % 8) || (dy_off % 8))
    return SEVP_BAD_ARG;
  const long long P = (long long)B * H * W;
  // enough CTAs to fill the GPU: pixel chunks x (taps x ci blocks) x co blocks
  const int cib = (cin + 31) / 32, cob = (cout + 63) / 64;
  long long chunks = (148LL * 8 + 9LL * cib * cob - 1) / (9LL * cib * cob);
  if (chunks < 1) chunks = 1;
  long long ppc = (P + chunks - 1) / chunks;
  ppc = ((ppc + kWP - 1) / kWP) * kWP;
  chunks = (P + ppc - 1) / ppc;
  dim3 grid((unsigned)chunks, (unsigned)cob, (unsigned)(9 * cib));
  cudaStream_t st = (cudaStream_t)stream;
  k_conv3x3_wgrad<<<grid, 128, 0, st>>>((const bf16 *)x, x_ld, x_off, cin, (const bf16 *)dy, dy_ld,
                                        dy_off, cout, (const bf16 *)mask, mask_ld, mask_off, dw, B,
                                        H, W, ppc);
  if (db) {
    dim3 g2(256, (unsigned)((cout + 255) / 256));
    k_bias_grad<<<g2, 256, 0, st>>>((const bf16 *)dy, dy_ld, dy_off, cout, (const bf16 *)mask, mask_ld,
                                    mask_off, db, P);
  }
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_weight_mirror(const void *w, void *wm, int cin, int cout, void *stream) {
  if (!w || !wm) return SEVP_BAD_ARG;
  const long long n = 9LL * cin * cout;
  k_weight_mirror<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wm, cin,
                                                                cout);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_conv3x3_dgrad_tc(const void *dy, int dy_ld, int dy_off, int cout, const void *mask,
                             int mask_ld, int mask_off, const void *wm, void *scratch, void *dx,
                             int dx_ld, int dx_off, int cin, int B, int H, int W, void *stream) {
  if (!dy || !wm || !scratch || !dx || bad_channels(cin) || bad_channels(cout) || B < 1 ||
      H < 1 || W < 1 || (dy_ld % 8) || (dy_off % 8) || ((uintptr_t)dy & 15) ||
      ((uintptr_t)scratch & 15) || (mask && ((mask_ld % 8) || (mask_off % 8) ||
                                              ((uintptr_t)mask & 15))))
    return SEVP_BAD_ARG;
  const long long P = (long long)B * H * W;
  cudaStream_t st = (cudaStream_t)stream;
  k_relu_mask8<<<ew_grid(P * (cout / 8)), 256, 0, st>>>((const bf16 *)dy, dy_ld, dy_off,
                                                        (const bf16 *)mask, mask_ld, mask_off,
                                                        cout / 8, (bf16 *)scratch, P);
  SEVP_CUDA_TRY(cudaGetLastError());
  return sevp_nn_conv3x3_tma(scratch, cout, 0, cout, wm, nullptr, dx, dx_ld, dx_off, cin, B, H, W,
                             0, stream);
}

int sevp_nn_conv3x3_backward_tc(const void *x, int x_ld, int x_off, int cin, const void *dy,
                                int dy_ld, int dy_off, int cout, const void *mask, int mask_ld,
                                int mask_off, const void *wm, void *scratch, float *dw, float *db,
                                void *dx, int dx_ld, int dx_off, int B, int H, int W,
                                void *stream) {
  if (!x || !dy || !scratch || !dw || bad_channels(cin) || bad_channels(cout) || B < 1 || H < 1 ||
      W < 1 || (dy_ld % 8) || (dy_off % 8) || ((uintptr_t)dy & 15) || ((uintptr_t)scratch & 15) ||
      (mask && ((mask_ld % 8) || (mask_off % 8) || ((uintptr_t)mask & 15))) || (dx && !wm))
    return SEVP_BAD_ARG;
  const long long P = (long long)B * H * W;
  cudaStream_t st = (cudaStream_t)stream;
  // the ReLU-masked output gradient, packed [P][cout], feeds all three
  k_relu_mask8<<<ew_grid(P * (cout / 8)), 256, 0, st>>>((const bf16 *)dy, dy_ld, dy_off,
                                                        (const bf16 *)mask, mask_ld, mask_off,
                                                        cout / 8, (bf16 *)scratch, P);
  SEVP_CUDA_TRY(cudaGetLastError());
  int s = sevp_nn_conv3x3_wgrad_tc(x, x_ld, x_off, cin, scratch, cout, dw, B, H, W, stream);
  if (s) return s;
  if (db) {
    dim3 g2(256, (unsigned)((cout + 255) / 256));
    k_bias_grad<<<g2, 256, 0, st>>>((const bf16 *)scratch, cout, 0, cout, nullptr, 0, 0, db, P);
    SEVP_CUDA_TRY(cudaGetLastError());
  }
  if (!dx) return SEVP_OK;
  return sevp_nn_conv3x3_tma(scratch, cout, 0, cout, wm, nullptr, dx, dx_ld, dx_off, cin, B, H, W,
                             0, stream);
}

int sevp_nn_weight_transpose(const void *w, void *wt, int cin, int cout, void *stream) {
  if (!w || !wt) return SEVP_BAD_ARG;
  const long long n = 9LL * cin * cout;
  k_weight_transpose<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wt, cin,
                                                                   cout);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_pool(const void *in, int in_ld, int in_off, void *out, int out_ld, int out_off, int C,
                 int B, int H, int W, int backward, int accumulate, void *stream) {
  if (!in || !out || (H % 2) || (W % 2)) return SEVP_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const bool v8 = C % 8 == 0 && in_ld % 8 == 0 && in_off % 8 == 0 && out_ld % 8 == 0 &&
                  out_off % 8 == 0 && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0;
  if (!backward && v8)
    k_pool_fwd8<<<ew_grid((long long)B * H * W * C / 32), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C / 8, B, H, W);
  else if (!backward)
    k_pool_fwd<<<ew_grid((long long)B * H * W * C / 4), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C, B, H, W);
  else  // in = dOut (H/2 x W/2), out = dIn (H x W)
    k_pool_bwd<<<ew_grid((long long)B * H * W * C), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C, B, H, W, accumulate);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_upsample(const void *in, int in_ld, int in_off, void *out, int out_ld, int out_off,
                     int C, int B, int H, int W, int backward, void *stream) {
  if (!in || !out || (H % 2) || (W % 2)) return SEVP_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const bool v8 = C % 8 == 0 && in_ld % 8 == 0 && in_off % 8 == 0 && out_ld % 8 == 0 &&
                  out_off % 8 == 0 && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0;
  if (!backward && v8)  // in: H/2 x W/2, out: H x W
    k_up_fwd8<<<ew_grid((long long)B * H * W * C / 32), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C / 8, B, H, W);
  else if (!backward)
    k_up_fwd<<<ew_grid((long long)B * H * W * C), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C, B, H, W);
  else  // in = dOut (H x W), out = dIn (H/2 x W/2)
    k_up_bwd<<<ew_grid((long long)B * H * W * C / 4), 256, 0, st>>>(
        (const bf16 *)in, in_ld, in_off, (bf16 *)out, out_ld, out_off, C, B, H, W);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_head(const void *x, int x_ld, int x_off, int C, const float *w, const float *b,
                 float *y, const float *dy, void *dx, int dx_ld, int dx_off, float *dw, float *db,
                 long long P, int backward, void *stream) {
  if (!x || !w || C < 1 || C > 256) return SEVP_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (!backward) {
    if (!y || !b) return SEVP_BAD_ARG;
    if (C % 8 == 0 && x_ld % 8 == 0 && x_off % 8 == 0 && ((uintptr_t)x & 15) == 0)
      k_head_fwd8<<<ew_grid(P), 256, 0, st>>>((const bf16 *)x, x_ld, x_off, C, w, b, y, P);
    else
      k_head_fwd<<<ew_grid(P), 256, 0, st>>>((const bf16 *)x, x_ld, x_off, C, w, b, y, P);
  } else {
    if (!dy || !dx || !dw || !db) return SEVP_BAD_ARG;
    k_head_bwd<<<ew_grid(P), 256, 0, st>>>((const bf16 *)x, x_ld, x_off, C, w, dy, (bf16 *)dx, dx_ld,
                                           dx_off, dw, db, P);
  }
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_mse(const float *y, const float *t, const float *valid, float *dy, float *loss,
                long long P, float inv_n, void *stream) {
  if (!y || !t || !dy || !loss) return SEVP_BAD_ARG;
  k_mse<<<ew_grid(P), 256, 0, (cudaStream_t)stream>>>(y, t, valid, dy, loss, P, inv_n);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_adam(float *w, const float *g, float *m, float *v, void *w16, float *w32, long long n,
                 float lr, float b1, float b2, float eps, int step, float wd, void *stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1) return SEVP_BAD_ARG;
  const float c1 = 1.f / (1.f - powf(b1, (float)step));
  const float c2 = 1.f / (1.f - powf(b2, (float)step));
  k_adam<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16 *)w16, w32, (size_t)n, lr, b1,
                                                       b2, eps, c1, c2, wd);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_nn_to_bf16(const float *a, void *b, long long n, void *stream) {
  if (!a || !b) return SEVP_BAD_ARG;
  k_f32_to_bf16<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>(a, (bf16 *)b, (size_t)n);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

}  // extern "C"
