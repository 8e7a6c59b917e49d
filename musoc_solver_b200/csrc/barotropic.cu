// Barotropic pressure correction of FS (M/fs_GLOBAL.f90:1154-1283): the
// ITMASK loop around the elliptic solve.  Each pass
//   1. zeroes the top-layer advection velocity over land      (:1158-1171),
//   2. forms the free-surface right-hand side S from continuity
//      (FLAG_FS branch, :1177-1192): a vertical integration per column,
//   3. solves A X = S                                          (:1213),
//   4. adds ODT X to the surface pressure P0 and corrects U, V in every layer
//      from the gradients of X, accumulating the corrections   (:1216-1265),
//   5. measures the largest top-layer velocity on land faces   (:1267-1276),
// and the loop ends when that is <= TOLERANCE or after MXMASK passes.
//
// Arrays are the reference's, column-major, on the device: U (I0,J0,K1),
// V (I0,J1,K1), IU0 / IV0 (I0,J0) and IU (I0,J0,K1) / IV (I0,J1,K1)
// INTEGER*2, ODX / ODY / OCS (J0), CSV / ODYV (J1), ODZ (K1), S (I2,J2),
// P0 (I0,J0), SCR (I0,J0,4).  X is the solver's unpadded (I2,J2) FP64 field,
// i.e. the interior X(2:I1, 2:J1) of the reference's padded array.  REAL*4
// and REAL*8 steps use round-to-nearest intrinsics in the Fortran order (no
// contraction), so the results equal the oracle's bit for bit.
#include <cstdint>

#include "common.cuh"
#include "sevp_nn.h"

namespace {

#define IDX2(i, j) ((size_t)((j) - 1) * (size_t)i0 + (size_t)((i) - 1))
#define IDX3(ld2, i, j, k) \
  (((size_t)((k) - 1) * (size_t)(ld2) + (size_t)((j) - 1)) * (size_t)i0 + (size_t)((i) - 1))

__global__ void k_fs_mask(int i0, int j0, float *u, float *v, const int16_t *iu0,
                          const int16_t *iv0, int periodic) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1;
  if (i > i0) return;
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, j2 = j0 - 2;
  if (j >= 2 && j <= j1 && ((i >= 2 && i <= i2) || (periodic && (i == 1 || i == i1))))
    u[IDX3(j0, i, j, 1)] = __fmul_rn((float)iu0[IDX2(i, j)], u[IDX3(j0, i, j, 1)]);
  if (j >= 2 && j <= j2 && i >= 2 && i <= i1)
    v[IDX3(j0 - 1, i, j, 1)] = __fmul_rn((float)iv0[IDX2(i, j)], v[IDX3(j0 - 1, i, j, 1)]);
}

// Layers a thread of the column kernels loads before it uses the first of
// them (loads in flight per thread).
constexpr int kFsLayerBatch = 4;

// one thread per interior column: W from the bottom (W(K0) = 0) to the top.
// The layer thicknesses' reciprocals are formed once per CTA (rdz, k1
// floats of dynamic shared memory), and the velocities of kFsLayerBatch
// layers are loaded before they are summed in the reference's order.
__global__ void k_fs_rhs(int i0, int j0, int k0, const float *__restrict__ u,
                         const float *__restrict__ v, const float *odx, const float *ody,
                         const float *ocs, const float *csv, const float *odz,
                         const float *rscale, float *s, double *b) {
  extern __shared__ float rdz[];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2, j = blockIdx.y + 2;
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, k1 = k0 - 1;
  for (int k = threadIdx.x; k < k1; k += blockDim.x) rdz[k] = __fdiv_rn(1.f, odz[k]);
  __syncthreads();
  if (i > i1 || j > j1) return;
  const float temp = __fmul_rn(ocs[j - 1], ody[j - 1]);
  const float dx = odx[j - 1], cn = csv[j - 1], cs = csv[j - 2];
  float w = 0.f;
  auto layer = [&](float ue, float uw, float vn, float vs, int k) {
    const float a = __fmul_rn(__fsub_rn(ue, uw), dx);
    const float bb = __fsub_rn(__fmul_rn(cn, vn), __fmul_rn(cs, vs));
    w = __fadd_rn(w, __fmul_rn(__fadd_rn(a, __fmul_rn(bb, temp)), rdz[k - 1]));
  };
  int k = k1;
  for (; k >= kFsLayerBatch; k -= kFsLayerBatch) {
    float ue[kFsLayerBatch], uw[kFsLayerBatch], vn[kFsLayerBatch], vs[kFsLayerBatch];
#pragma unroll
    for (int q = 0; q < kFsLayerBatch; ++q) {
      ue[q] = u[IDX3(j0, i, j, k - q)];
      uw[q] = u[IDX3(j0, i - 1, j, k - q)];
      vn[q] = v[IDX3(j0 - 1, i, j, k - q)];
      vs[q] = v[IDX3(j0 - 1, i, j - 1, k - q)];
    }
#pragma unroll
    for (int q = 0; q < kFsLayerBatch; ++q) layer(ue[q], uw[q], vn[q], vs[q], k - q);
  }
  for (; k >= 1; --k)
    layer(u[IDX3(j0, i, j, k)], u[IDX3(j0, i - 1, j, k)], v[IDX3(j0 - 1, i, j, k)],
          v[IDX3(j0 - 1, i, j - 1, k)], k);
  const size_t o = (size_t)(j - 2) * i2 + (i - 2);
  if (s) s[o] = w;
  if (b) b[o] = rscale ? (double)w * (double)rscale[j - 2] : (double)w;
}

__device__ __forceinline__ float face_corr(double xr, double xl, float metric) {
  return __double2float_rn(-__dmul_rn(__dsub_rn(xr, xl), (double)metric));
}

// The layers below the top of one U face and one V face:
// f[o + l so] += cf * m[o + l so] (when af) and g[p + l sp] += cg *
// mg[p + l sp] (when ag) for l < nl, with each layer's land mask;
// kFsLayerBatch layers of both faces are loaded before the first is used.
__device__ __forceinline__ void correct_layers(float *f, const int16_t *m, size_t o, size_t so,
                                               bool af, float cf, float *g, const int16_t *mg,
                                               size_t p, size_t sp, bool ag, float cg, int nl) {
  int l = 0;
  for (; l + kFsLayerBatch <= nl; l += kFsLayerBatch) {
    float fv[kFsLayerBatch], gv[kFsLayerBatch];
    int16_t fm[kFsLayerBatch], gm[kFsLayerBatch];
#pragma unroll
    for (int q = 0; q < kFsLayerBatch; ++q) {
      if (af) {
        fv[q] = f[o + (size_t)(l + q) * so];
        fm[q] = m[o + (size_t)(l + q) * so];
      }
      if (ag) {
        gv[q] = g[p + (size_t)(l + q) * sp];
        gm[q] = mg[p + (size_t)(l + q) * sp];
      }
    }
#pragma unroll
    for (int q = 0; q < kFsLayerBatch; ++q) {
      if (af) f[o + (size_t)(l + q) * so] = __fadd_rn(fv[q], __fmul_rn(cf, (float)fm[q]));
      if (ag) g[p + (size_t)(l + q) * sp] = __fadd_rn(gv[q], __fmul_rn(cg, (float)gm[q]));
    }
  }
  for (; l < nl; ++l) {
    if (af)
      f[o + (size_t)l * so] =
          __fadd_rn(f[o + (size_t)l * so], __fmul_rn(cf, (float)m[o + (size_t)l * so]));
    if (ag)
      g[p + (size_t)l * sp] =
          __fadd_rn(g[p + (size_t)l * sp], __fmul_rn(cg, (float)mg[p + (size_t)l * sp]));
  }
}

// one thread per (I, J): P0 at the cell, the U face east of it, the V face
// north of it, all layers; then the land-face maximum of the top layer
__global__ void k_fs_correct(int i0, int j0, int k0, const double *x, float odt, const float *odx,
                             const float *odyv, const int16_t *iu, const int16_t *iv,
                             const int16_t *iu0, const int16_t *iv0, float *p0, float *u, float *v,
                             float *scr, int periodic, float *vmax) {
  // threads past the last column stay for the warp reduction at the end
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1;
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, j2 = j0 - 2, k1 = k0 - 1;
  const size_t plane = (size_t)i0 * j0;
  float *s1 = scr, *s2 = scr + plane, *s3 = scr + 2 * plane, *s4 = scr + 3 * plane;
  auto X = [&](int ii, int jj) { return x[(size_t)(jj - 2) * i2 + (ii - 2)]; };
  float land = 0.f;
  if (i >= 2 && i <= i1 && j >= 2 && j <= j1) {
    const size_t c = IDX2(i, j);
    p0[c] = __double2float_rn(__dadd_rn((double)p0[c], __dmul_rn((double)odt, X(i, j))));
  }
  const bool fu = j >= 2 && j <= j1 && i <= i1;  // U face (I, J), I = 1 .. I1
  const bool fv = i >= 2 && i <= i1 && j <= j1;  // V face (I, J), J = 1 .. J1
  float cu = 0.f, cv = 0.f;
  if (fu) {
    if (i >= 2 && i <= i2)
      cu = face_corr(X(i + 1, j), X(i, j), odx[j - 1]);
    else if (periodic)
      cu = face_corr(X(2, j), X(i1, j), odx[j - 1]);
    const size_t o = IDX2(i, j);
    s1[o] = cu;
    s3[o] = __fadd_rn(s3[o], cu);
    const float top = __fadd_rn(u[IDX3(j0, i, j, 1)], cu);
    u[IDX3(j0, i, j, 1)] = top;
    if (i >= 2 && i <= i2) land = __fmul_rn((float)(1 - iu0[o]), fabsf(top));
  }
  if (fv) {
    if (j >= 2 && j <= j2) cv = face_corr(X(i, j + 1), X(i, j), odyv[j - 1]);
    const size_t o = IDX2(i, j);
    s2[o] = cv;
    s4[o] = __fadd_rn(s4[o], cv);
    const float top = __fadd_rn(v[IDX3(j0 - 1, i, j, 1)], cv);
    v[IDX3(j0 - 1, i, j, 1)] = top;
    if (j >= 2 && j <= j2) land = fmaxf(land, __fmul_rn((float)(1 - iv0[o]), fabsf(top)));
  }
  // the layers below the top, both faces at once
  correct_layers(u, iu, fu ? IDX3(j0, i, j, 2) : 0, plane, fu, cu, v, iv,
                 fv ? IDX3(j0 - 1, i, j, 2) : 0, (size_t)i0 * (j0 - 1), fv, cv, k1 - 1);
  // non-negative floats order like their bit patterns
  for (int o = 16; o > 0; o >>= 1) land = fmaxf(land, __shfl_xor_sync(0xffffffffu, land, o));
  if ((threadIdx.x & 31) == 0 && land > 0.f) atomicMax((int *)vmax, __float_as_int(land));
}

#undef IDX2
#undef IDX3

bool fs_dims_ok(int i0, int j0, int k0) { return i0 >= 4 && j0 >= 4 && k0 >= 2; }

}  // namespace

extern "C" {

int sevp_fs_mask(int i0, int j0, float *u, float *v, const int16_t *iu0, const int16_t *iv0,
                 int periodic, void *stream) {
  if (!fs_dims_ok(i0, j0, 2) || !u || !v || !iu0 || !iv0) return SEVP_BAD_ARG;
  dim3 grid((unsigned)((i0 + 127) / 128), (unsigned)j0);
  k_fs_mask<<<grid, 128, 0, (cudaStream_t)stream>>>(i0, j0, u, v, iu0, iv0, periodic);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_fs_rhs(int i0, int j0, int k0, const float *u, const float *v, const float *odx,
                const float *ody, const float *ocs, const float *csv, const float *odz,
                const float *rscale, float *s, double *b, void *stream) {
  if (!fs_dims_ok(i0, j0, k0) || !u || !v || !odx || !ody || !ocs || !csv || !odz || (!s && !b))
    return SEVP_BAD_ARG;
  dim3 grid((unsigned)((i0 - 2 + 127) / 128), (unsigned)(j0 - 2));
  k_fs_rhs<<<grid, 128, (size_t)(k0 - 1) * sizeof(float), (cudaStream_t)stream>>>(
      i0, j0, k0, u, v, odx, ody, ocs, csv, odz, rscale, s, b);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_fs_correct(int i0, int j0, int k0, const double *x, float odt, const float *odx,
                    const float *odyv, const int16_t *iu, const int16_t *iv, const int16_t *iu0,
                    const int16_t *iv0, float *p0, float *u, float *v, float *scr, int periodic,
                    float *vmax, void *stream) {
  if (!fs_dims_ok(i0, j0, k0) || !x || !odx || !odyv || !iu || !iv || !iu0 || !iv0 || !p0 || !u ||
      !v || !scr || !vmax)
    return SEVP_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  SEVP_CUDA_TRY(cudaMemsetAsync(vmax, 0, sizeof(float), st));
  dim3 grid((unsigned)((i0 + 127) / 128), (unsigned)j0);
  k_fs_correct<<<grid, 128, 0, st>>>(i0, j0, k0, x, odt, odx, odyv, iu, iv, iu0, iv0, p0, u, v, scr,
                                     periodic, vmax);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int sevp_fs_barotropic(sevp_ctx *ctx, int i0, int j0, int k0, float *u, float *v, float *p0,
                       float *scr, const int16_t *iu0, const int16_t *iv0, const int16_t *iu,
                       const int16_t *iv, const float *odx, const float *ody, const float *ocs,
                       const float *csv, const float *odyv, const float *odz, const float *rscale,
                       float odt, int periodic, float tolerance, int mxmask,
                       const sevp_solve_opts *opts,
                       double *b, double *x, float *vmax_dev, int *itmask_out, float *vmax_out,
                       int *iterations_out) {
  if (!ctx || !opts || !b || !x || !vmax_dev || mxmask < 1 || !fs_dims_ok(i0, j0, k0))
    return SEVP_BAD_ARG;
  void *stream = sevp_stream(ctx);
  int s = SEVP_OK, it = 0, iters = 0;
  float tmp = 0.f;
  sevp_solve_opts o = *opts;
  o.use_guess = 0;  // X is the pass's increment, solved from zero
  for (;;) {
    ++it;
    if ((s = sevp_fs_mask(i0, j0, u, v, iu0, iv0, periodic, stream))) break;
    if ((s = sevp_fs_rhs(i0, j0, k0, u, v, odx, ody, ocs, csv, odz, rscale, nullptr, b, stream)))
      break;
    sevp_report rep{};
    s = sevp_solve(ctx, b, x, &o, &rep);
    iters += rep.iterations;
    if (s != SEVP_OK && s != SEVP_MAXITER) break;
    if ((s = sevp_fs_correct(i0, j0, k0, x, odt, odx, odyv, iu, iv, iu0, iv0, p0, u, v, scr,
                             periodic, vmax_dev, stream)))
      break;
    cudaError_t e = cudaMemcpyAsync(&tmp, vmax_dev, sizeof(float), cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) {
      sevp_internal_set_error(e, "read of the land velocity", __FILE__, __LINE__);
      s = SEVP_CUDA_ERROR;
      break;
    }
    if (tmp <= tolerance || it == mxmask) break;
  }
  if (itmask_out) *itmask_out = it;
  if (vmax_out) *vmax_out = tmp;
  if (iterations_out) *iterations_out = iters;
  return s;
}

}  // extern "C"
