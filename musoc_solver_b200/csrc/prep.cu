// PREP's preprocessing for the elliptic solver (P/prep_GLOBAL.f90:143-261):
// the row-block partition IE of the reference's SEVP blocks, and the
// assembly of the five-point coefficient planes AL, AR, AB, AT, AC from the
// grid metrics and the layer masks.
//
// The assembly runs one thread per grid point.  Each thread walks the
// layers K = 2..K1 for its point, accumulating in the order of the
// reference's K loop, so the planes equal PREP's REAL*4 results bit for bit
// (every product, sum and quotient is an explicitly rounded single-precision
// operation: no contraction into fused multiply-adds).
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "common.cuh"

namespace sevp {
namespace {

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

struct PrepIn {
  int i2, j2, k1, dimen, nbir, idealised;
  float gamma;
  // metrics, C index = Fortran index - 1: ODX, ODY, OCS (J0); CSV, ODYV (J1);
  // ODZ (K1)
  const float *odx, *ody, *csv, *ocs, *odyv, *odz;
  // INTEGER*2 masks IU (I0, J0, K1) and IV (I0, J1, K1), column-major
  const int16_t *iu, *iv;
};

// Fortran IU(i, j, k) / IV(i, j, k), 1-based.
__device__ __forceinline__ float mask_at(const int16_t *m, int i0, int jext, int i, int j, int k) {
  return (float)m[((size_t)(k - 1) * jext + (size_t)(j - 1)) * i0 + (size_t)(i - 1)];
}

// The four couplings of point (i, j) (1-based) before the edge rules,
// P/prep_GLOBAL.f90:170-212.
__device__ void couplings(const PrepIn &p, int i, int j, float &vl, float &vr, float &vb,
                          float &vt) {
  if (p.dimen == 2) {
    // :170-181: DZX = ODX(1)**2 / ODZ(1), DZY = ODY(1)**2 / ODZ(1)
    const float dzx = __fdiv_rn(fm(p.odx[0], p.odx[0]), p.odz[0]);
    const float dzy = __fdiv_rn(fm(p.ody[0], p.ody[0]), p.odz[0]);
    vl = vr = dzx;
    vb = vt = dzy;
    return;
  }
  const int i0 = p.i2 + 2, j0 = p.j2 + 2, j1 = p.j2 + 1;
  // Fortran ODX(J+1) is odx[j]; CSV(J) is csv[j - 1]
  const float ox2 = fm(p.odx[j], p.odx[j]);
  const float yb = fm(fm(fm(p.csv[j - 1], p.ocs[j]), p.odyv[j - 1]), p.ody[j]);
  const float yt = fm(fm(fm(p.csv[j], p.ocs[j]), p.odyv[j]), p.ody[j]);
  // top layer all water (:184-196)
  float tmp = __fdiv_rn(1.f, p.odz[0]);
  vl = vr = fm(ox2, tmp);
  vb = fm(yb, tmp);
  vt = fm(yt, tmp);
  // remaining layers (:198-211)
  for (int k = 2; k <= p.k1; ++k) {
    tmp = __fdiv_rn(1.f, p.odz[k - 1]);
    const float dzx = fm(ox2, tmp), dzyb = fm(yb, tmp), dzyt = fm(yt, tmp);
    vl = fa(vl, fm(dzx, mask_at(p.iu, i0, j0, i, j + 1, k)));
    vr = fa(vr, fm(dzx, mask_at(p.iu, i0, j0, i + 1, j + 1, k)));
    vb = fa(vb, fm(dzyb, mask_at(p.iv, i0, j1, i + 1, j, k)));
    vt = fa(vt, fm(dzyt, mask_at(p.iv, i0, j1, i + 1, j + 1, k)));
  }
}

__global__ void k_prep_assemble(PrepIn p, float *al, float *ar, float *ab, float *at, float *ac) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > p.i2 || j > p.j2) return;
  float vl, vr, vb, vt;
  couplings(p, i, j, vl, vr, vb, vt);
  // closed side walls (:214-219), south and north edges (:221-224)
  if (p.nbir == 1) {
    if (i == 1) vl = 0.f;
    if (i == p.i2) vr = 0.f;
  }
  if (j == 1) vb = 0.f;
  if (j == p.j2) vt = 0.f;
  // pin down pressure (:227-229): AB(I2/2, 1) = AB(I2/2, 2), the assembled
  // value of row 2 (the edge rules leave row 2's AB alone)
  if (p.nbir == 1 && p.j2 >= 2 && j == 1 && i == p.i2 / 2) {
    float ql, qr, qb, qt;
    couplings(p, i, 2, ql, qr, qb, qt);
    vb = qb;
  }
  // :238-242
  float vc = fs(fs(fs(fs(-vl, vr), vb), vt), p.gamma);
  if (p.idealised) {
    // the constant test stencil and Neumann rows of :244-258
    vl = vb = vr = vt = -0.25f;
    vc = 1.0f;
    if (j == p.j2) {
      vc = fa(vc, vt);
      vt = 0.f;
    }
    if (j == 1) {
      vc = fa(vc, vb);
      vb = 0.f;
    }
  }
  const size_t o = (size_t)(j - 1) * p.i2 + (size_t)(i - 1);
  al[o] = vl;
  ar[o] = vr;
  ab[o] = vb;
  at[o] = vt;
  ac[o] = vc;
}

}  // namespace
}  // namespace sevp

using namespace sevp;

extern "C" int sevp_block_partition(int j2, int nb0, int dimen, int *ie) {
  if (!ie || j2 < 1 || nb0 < 2 || (dimen != 2 && dimen != 3)) {
    sevp_internal_set_message("sevp_block_partition: needs j2 >= 1, nb0 >= 2, dimen 2 or 3");
    return SEVP_BAD_ARG;
  }
  const int j1 = j2 + 1;
  // NN = ANINT(REAL(J2) / REAL(NB0)): single-precision quotient, rounded half
  // away from zero
  const float q = (float)j2 / (float)nb0;
  const int nn = (int)lroundf(q);
  for (int n = 1; n <= nb0; ++n) ie[n - 1] = 1 + nn * n < j1 ? 1 + nn * n : j1;
  // the reference's validity test: the last block must be nonempty and not
  // longer than NN + 1 rows (2-D) or NN + 3 rows (3-D)
  const int slack = dimen == 2 ? 1 : 3;
  const bool ok = ie[nb0 - 1] > ie[nb0 - 2] && j1 < ie[nb0 - 2] + nn + slack;
  ie[nb0 - 1] = j1;
  if (!ok) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "sevp_block_partition: IE(NB1)=%d, J1=%d not properly defined (J2=%d, NB0=%d)",
             ie[nb0 - 2], j1, j2, nb0);
    sevp_internal_set_message(msg);
    return SEVP_BAD_ARG;
  }
  return SEVP_OK;
}

static int prep_check(int i2, int j2, int k1, int dimen, int nbir) {
  if (i2 < 1 || j2 < 1 || k1 < 1 || (dimen != 2 && dimen != 3) || (nbir != 1 && nbir != 2)) {
    sevp_internal_set_message("sevp_prep_assemble: bad grid size, dimen or nbir");
    return SEVP_BAD_ARG;
  }
  return SEVP_OK;
}

extern "C" int sevp_prep_assemble(int i2, int j2, int k1, int dimen, const float *odx,
                                  const float *ody, const float *csv, const float *ocs,
                                  const float *odyv, const float *odz, const int16_t *iu,
                                  const int16_t *iv, int nbir, float gamma, int idealised,
                                  float *al, float *ar, float *ab, float *at, float *ac,
                                  void *stream) {
  int s = prep_check(i2, j2, k1, dimen, nbir);
  if (s) return s;
  if (!odx || !ody || !odz || !al || !ar || !ab || !at || !ac ||
      (dimen == 3 && (!csv || !ocs || !odyv || (k1 > 1 && (!iu || !iv))))) {
    sevp_internal_set_message("sevp_prep_assemble: null array");
    return SEVP_BAD_ARG;
  }
  PrepIn p{i2, j2, k1, dimen, nbir, idealised ? 1 : 0, gamma, odx, ody, csv, ocs, odyv, odz, iu, iv};
  const dim3 blk(32, 8), grd((unsigned)((i2 + 31) / 32), (unsigned)((j2 + 7) / 8));
  k_prep_assemble<<<grd, blk, 0, (cudaStream_t)stream>>>(p, al, ar, ab, at, ac);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

extern "C" int sevp_prep_assemble_host(int i2, int j2, int k1, int dimen, const float *odx,
                                       const float *ody, const float *csv, const float *ocs,
                                       const float *odyv, const float *odz, const int16_t *iu,
                                       const int16_t *iv, int nbir, float gamma, int idealised,
                                       float *al, float *ar, float *ab, float *at, float *ac) {
  int s = prep_check(i2, j2, k1, dimen, nbir);
  if (s) return s;
  const size_t i0 = (size_t)i2 + 2, j0 = (size_t)j2 + 2, j1 = (size_t)j2 + 1;
  const bool masks = dimen == 3 && k1 > 1;
  if (!odx || !ody || !odz || !al || !ar || !ab || !at || !ac ||
      (dimen == 3 && (!csv || !ocs || !odyv)) || (masks && (!iu || !iv))) {
    sevp_internal_set_message("sevp_prep_assemble_host: null array");
    return SEVP_BAD_ARG;
  }
  // one device block: metrics (J0 each, ODZ K1), masks, the five planes
  const size_t nmet = 5 * j0 + (size_t)k1;
  const size_t nu = masks ? i0 * j0 * k1 : 0, nv = masks ? i0 * j1 * k1 : 0;
  const size_t npl = (size_t)i2 * j2;
  const size_t bytes = nmet * 4 + (nu + nv) * 2 + 16 + 5 * npl * 4;
  char *d = nullptr;
  SEVP_CUDA_TRY(cudaMalloc((void **)&d, bytes));
  float *met = (float *)d;
  float *d_odx = met, *d_ody = met + j0, *d_csv = met + 2 * j0, *d_ocs = met + 3 * j0,
        *d_odyv = met + 4 * j0, *d_odz = met + 5 * j0;
  int16_t *d_iu = (int16_t *)(d + nmet * 4), *d_iv = d_iu + nu;
  float *pl = (float *)(((uintptr_t)(d_iv + nv) + 15) & ~(uintptr_t)15);
  cudaError_t e = cudaSuccess;
  auto up = [&](void *dst, const void *src, size_t n) {
    if (e == cudaSuccess && src) e = cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
  };
  up(d_odx, odx, j0 * 4);
  up(d_ody, ody, j0 * 4);
  if (dimen == 3) {
    up(d_csv, csv, j1 * 4);
    up(d_ocs, ocs, j0 * 4);
    up(d_odyv, odyv, j1 * 4);
  }
  up(d_odz, odz, (size_t)k1 * 4);
  if (masks) {
    up(d_iu, iu, nu * 2);
    up(d_iv, iv, nv * 2);
  }
  if (e == cudaSuccess) {
    s = sevp_prep_assemble(i2, j2, k1, dimen, d_odx, d_ody, d_csv, d_ocs, d_odyv, d_odz,
                           masks ? d_iu : nullptr, masks ? d_iv : nullptr, nbir, gamma, idealised,
                           pl, pl + npl, pl + 2 * npl, pl + 3 * npl, pl + 4 * npl, nullptr);
    float *outs[5] = {al, ar, ab, at, ac};
    for (int k = 0; k < 5 && !s && e == cudaSuccess; ++k)
      e = cudaMemcpy(outs[k], pl + k * npl, npl * 4, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "sevp_prep_assemble_host", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  return s;
}
