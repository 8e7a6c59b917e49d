// Krylov drop-ins of the reference on the GPU: operator apply p_sqprod
// (M/sevp.f90:696-713), its transpose p_sqprod_T (:714-742), the interior dot
// product p_inprod (:743-757), the periodic ghost refresh
// solver_boundary_update (:773-787), restarted BiCGSTAB p_bicgstab_le
// (:443-552), Chebyshev semi-iteration p_csi (:553-616) and the two-sided
// Lanczos eigen bound lanczos (:618-694) with figi (:838-904) and ratqr
// (:906-1006).
//
// Arrays are the reference's padded (i2+2, j2+2) column-major FP64 fields and
// (i2, j2) FP32 coefficients.  Element-wise steps use explicitly rounded
// intrinsics in the reference's evaluation order (bit-identical to the
// Fortran); dot products are a fixed-order parallel tree (deterministic, but
// rounded differently from the serial Fortran sum).
#include <cmath>
#include <memory>
#include <vector>

#include "common.cuh"
#include "dropin.cuh"

namespace sevp {

#define IXK(ld, i, j) ((size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1))

namespace {
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
}  // namespace

// r(i+1,j+1) = ab*x_S + al*x_W + ac*x_C + ar*x_E + at*x_N, left to right
__global__ void k_sqprod(const float *al, const float *ab, const float *ac, const float *ar,
                         const float *at, const double *x, double *r, int i2, int j2) {
  const int i0 = i2 + 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > i2 || j > j2) return;
  const size_t c = IXK(i2, i, j);
  double t = mul((double)ab[c], x[IXK(i0, i + 1, j)]);
  t = add(t, mul((double)al[c], x[IXK(i0, i, j + 1)]));
  t = add(t, mul((double)ac[c], x[IXK(i0, i + 1, j + 1)]));
  t = add(t, mul((double)ar[c], x[IXK(i0, i + 2, j + 1)]));
  t = add(t, mul((double)at[c], x[IXK(i0, i + 1, j + 2)]));
  r[IXK(i0, i + 1, j + 1)] = t;
}

// transpose: neighbour cell's coefficient, zero outside the interior
__device__ __forceinline__ double padc(const float *a, int i2, int j2, int i, int j) {
  return (i >= 2 && i <= i2 + 1 && j >= 2 && j <= j2 + 1) ? (double)a[IXK(i2, i - 1, j - 1)] : 0.0;
}
__global__ void k_sqprod_t(const float *al, const float *ab, const float *ac, const float *ar,
                           const float *at, const double *x, double *r, int i2, int j2) {
  const int i0 = i2 + 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > i2 || j > j2) return;
  double t = mul(padc(at, i2, j2, i + 1, j), x[IXK(i0, i + 1, j)]);
  t = add(t, mul(padc(ar, i2, j2, i, j + 1), x[IXK(i0, i, j + 1)]));
  t = add(t, mul((double)ac[IXK(i2, i, j)], x[IXK(i0, i + 1, j + 1)]));
  t = add(t, mul(padc(al, i2, j2, i + 2, j + 1), x[IXK(i0, i + 2, j + 1)]));
  t = add(t, mul(padc(ab, i2, j2, i + 1, j + 2), x[IXK(i0, i + 1, j + 2)]));
  r[IXK(i0, i + 1, j + 1)] = t;
}

// Deterministic interior dot product: each CTA sums a fixed slice of rows,
// the last CTA sums the partials in CTA order and stores the result.
constexpr int kDotThreads = 256;
__global__ void __launch_bounds__(kDotThreads)
    k_inprod(const double *r, const double *p, int i2, int j2, double *partials, unsigned *ticket,
             double *out) {
  const int i0 = i2 + 2;
  const size_t n = (size_t)i2 * j2;
  double s = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(e % i2), j = 2 + (int)(e / i2);
    s += r[IXK(i0, i, j)] * p[IXK(i0, i, j)];
  }
  __shared__ double red[32];
  __shared__ int last;
  double v[1] = {s};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += __ldcg(&partials[b]);
    *out = t;
    *ticket = 0u;
  }
}

__global__ void k_boundary(double *x, int i2, int j2) {
  const int i0 = i2 + 2;
  for (int j = 2 + blockIdx.x * blockDim.x + threadIdx.x; j <= j2 + 1; j += gridDim.x * blockDim.x) {
    x[IXK(i0, 1, j)] = x[IXK(i0, i2 + 1, j)];
    x[IXK(i0, i2 + 2, j)] = x[IXK(i0, 2, j)];
  }
}

// r(interior) = b - r(interior)
__global__ void k_rhs_minus(const float *b, double *r, int i2, int j2) {
  const int i0 = i2 + 2;
  const size_t n = (size_t)i2 * j2;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(e % i2), j = 1 + (int)(e / i2);
    r[IXK(i0, i + 1, j + 1)] = sub((double)b[IXK(i2, i, j)], r[IXK(i0, i + 1, j + 1)]);
  }
}

// r(interior) = b - s(interior)
__global__ void k_b_minus(const float *b, const double *s, double *r, int i2, int j2) {
  const int i0 = i2 + 2;
  const size_t n = (size_t)i2 * j2;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(e % i2), j = 1 + (int)(e / i2);
    r[IXK(i0, i + 1, j + 1)] = sub((double)b[IXK(i2, i, j)], s[IXK(i0, i + 1, j + 1)]);
  }
}

// Element-wise kernels over all (i2+2)(j2+2) points.  Scalars are read from
// device memory (sc) so that no host round trip sits between them.
enum Scal { S_RHO, S_RHN, S_ALPHA, S_BETA, S_W, S_TMP, S_TP, S_RES, S_TT, S_TS, S_NSC };

__global__ void k_bicg_scal(double *sc, int which) {
  if (which == 0) {  // beta = (rhn/rho)*(alpha/w)
    sc[S_BETA] = __dmul_rn(__ddiv_rn(sc[S_RHN], sc[S_RHO]), __ddiv_rn(sc[S_ALPHA], sc[S_W]));
  } else if (which == 1) {  // alpha = rhn/tmp
    sc[S_ALPHA] = __ddiv_rn(sc[S_RHN], sc[S_TMP]);
  } else if (which == 2) {  // w = (t,s)/(t,t)
    sc[S_W] = __ddiv_rn(sc[S_TS], sc[S_TT]);
  } else if (which == 3) {  // rho = rhn
    sc[S_RHO] = sc[S_RHN];
  } else if (which == 4) {  // restart: rho = alpha = w = 1
    sc[S_RHO] = 1.0, sc[S_ALPHA] = 1.0, sc[S_W] = 1.0;
  }
}

// p = r + beta*(p - w*v); ph = p
__global__ void k_bicg_p(const double *r, double *p, const double *v, double *ph, const double *sc,
                         size_t n) {
  const double beta = sc[S_BETA], w = sc[S_W];
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double pv = add(r[k], mul(beta, sub(p[k], mul(w, v[k]))));
    p[k] = pv;
    ph[k] = pv;
  }
}
// s = r - alpha*v; sh = s
__global__ void k_bicg_s(const double *r, const double *v, double *s, double *sh, const double *sc,
                         size_t n) {
  const double alpha = sc[S_ALPHA];
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double sv = sub(r[k], mul(alpha, v[k]));
    s[k] = sv;
    sh[k] = sv;
  }
}
// x = x + alpha*ph + w*sh; r = s - w*t
__global__ void k_bicg_xr(double *x, double *r, const double *ph, const double *sh,
                          const double *s, const double *t, const double *sc, size_t n) {
  const double alpha = sc[S_ALPHA], w = sc[S_W];
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] = add(add(x[k], mul(alpha, ph[k])), mul(w, sh[k]));
    r[k] = sub(s[k], mul(w, t[k]));
  }
}

// ---------------------------------------------- one-CTA BiCGSTAB (small grids)
// The whole restarted BiCGSTAB of dev_bicgstab below in ONE thread block:
// on the reference's own grid (182 x 92) the multi-launch loop spends its
// time in some 16 launches and a host round trip per iteration, while each
// pass touches only 130 KB.  Here 1024 threads run every pass between block
// barriers and keep the scalars in shared memory; the arithmetic of every
// element-wise step is that of the kernels above (k_sqprod, k_rhs_minus,
// k_bicg_*), the control flow that of the host loop (restart quirk and
// stopping tests included).  Dot products are a fixed-order block tree
// (deterministic; rounded differently from the multi-CTA tree).
constexpr int kCtaThreads = 1024;
// padded grids up to this many points run dev_bicgstab in one thread block
// (the vectors stay in L2); larger ones run the multi-launch loop
constexpr size_t kCtaMaxPoints = (size_t)1 << 17;

struct BicgVecs {
  double *r, *rh, *p, *v, *s, *t, *ph, *sh;
};

// The passes below take restrict-qualified pointers (the vectors are
// distinct buffers) and unroll by four, so a thread issues the loads of
// several elements before the first store: each pass costs a few memory
// round trips instead of one per element.
__device__ double cta_dot(const double *__restrict__ a, const double *__restrict__ b, int i2,
                          int j2, double *red, double *out) {
  const int i0 = i2 + 2;
  const size_t n = (size_t)i2 * j2;
  double v[1] = {0.0};
#pragma unroll 4
  for (size_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = 2 + (int)(e % i2), j = 2 + (int)(e / i2);
    v[0] += a[IXK(i0, i, j)] * b[IXK(i0, i, j)];
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) *out = v[0];
  __syncthreads();
  return *out;
}
__device__ void cta_apply(const float *__restrict__ al, const float *__restrict__ ab,
                          const float *__restrict__ ac, const float *__restrict__ ar,
                          const float *__restrict__ at, const double *__restrict__ x,
                          double *__restrict__ r, int i2, int j2) {
  const int i0 = i2 + 2;
  const size_t n = (size_t)i2 * j2;
#pragma unroll 4
  for (size_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = 1 + (int)(e % i2), j = 1 + (int)(e / i2);
    const size_t c = IXK(i2, i, j);
    double t = mul((double)ab[c], x[IXK(i0, i + 1, j)]);
    t = add(t, mul((double)al[c], x[IXK(i0, i, j + 1)]));
    t = add(t, mul((double)ac[c], x[IXK(i0, i + 1, j + 1)]));
    t = add(t, mul((double)ar[c], x[IXK(i0, i + 2, j + 1)]));
    t = add(t, mul((double)at[c], x[IXK(i0, i + 1, j + 2)]));
    r[IXK(i0, i + 1, j + 1)] = t;
  }
  __syncthreads();
}
// b - r on the interior
__device__ void cta_rhs_minus(const float *__restrict__ b, double *__restrict__ r, int i2,
                              int j2) {
  const int i0 = i2 + 2;
  const size_t ni = (size_t)i2 * j2;
#pragma unroll 4
  for (size_t e = threadIdx.x; e < ni; e += blockDim.x) {
    const int i = 1 + (int)(e % i2), j = 1 + (int)(e / i2);
    r[IXK(i0, i + 1, j + 1)] = sub((double)b[IXK(i2, i, j)], r[IXK(i0, i + 1, j + 1)]);
  }
  __syncthreads();
}
__device__ void cta_copy(const double *__restrict__ a, double *__restrict__ c, size_t n) {
#pragma unroll 4
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) c[k] = a[k];
  __syncthreads();
}
// p = r + beta*(p - w*v); ph = p
__device__ void cta_p(const double *__restrict__ r, double *__restrict__ p,
                      const double *__restrict__ v, double *__restrict__ ph, double beta, double w,
                      size_t n) {
#pragma unroll 4
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) {
    const double pv = add(r[k], mul(beta, sub(p[k], mul(w, v[k]))));
    p[k] = pv;
    ph[k] = pv;
  }
  __syncthreads();
}
// s = r - alpha*v; sh = s
__device__ void cta_s(const double *__restrict__ r, const double *__restrict__ v,
                      double *__restrict__ s, double *__restrict__ sh, double alpha, size_t n) {
#pragma unroll 4
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) {
    const double sv = sub(r[k], mul(alpha, v[k]));
    s[k] = sv;
    sh[k] = sv;
  }
  __syncthreads();
}
// x = x + alpha*ph + w*sh; r = s - w*t
__device__ void cta_xr(double *__restrict__ x, double *__restrict__ r,
                       const double *__restrict__ ph, const double *__restrict__ sh,
                       const double *__restrict__ s, const double *__restrict__ t, double alpha,
                       double w, size_t n) {
#pragma unroll 4
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) {
    x[k] = add(add(x[k], mul(alpha, ph[k])), mul(w, sh[k]));
    r[k] = sub(s[k], mul(w, t[k]));
  }
  __syncthreads();
}
__device__ void cta_boundary(double *x, int i2, int j2, int periodic) {
  if (!periodic) return;
  const int i0 = i2 + 2;
  for (int j = 2 + threadIdx.x; j <= j2 + 1; j += blockDim.x) {
    x[IXK(i0, 1, j)] = x[IXK(i0, i2 + 1, j)];
    x[IXK(i0, i2 + 2, j)] = x[IXK(i0, 2, j)];
  }
  __syncthreads();
}

// out[0] = iterations, out[1] = final r.r, out[2] = 1 when r.r became
// non-finite (the host loop's early return, without the last ghost refresh)
__global__ void __launch_bounds__(kCtaThreads, 1)
    k_bicgstab_cta(const float *al, const float *ab, const float *ac, const float *ar,
                   const float *at, const float *b, double *x, BicgVecs V, int i2, int j2,
                   int periodic, double tol, double *out) {
  __shared__ double red[32];
  __shared__ double sc[S_NSC];
  const int tid = threadIdx.x;
  const size_t n = (size_t)(i2 + 2) * (j2 + 2);
  int iter = 0;
  bool nonfinite = false;
  double tp = 1.0, res = 0.0;
  cta_boundary(x, i2, j2, periodic);
  while (sqrt(tp) > tol && iter < 1000) {
    if (tid == 0) sc[S_RHO] = 1.0, sc[S_ALPHA] = 1.0, sc[S_W] = 1.0;
    cta_apply(al, ab, ac, ar, at, x, V.r, i2, j2);
    cta_rhs_minus(b, V.r, i2, j2);
    cta_boundary(V.r, i2, j2, periodic);
    cta_copy(V.r, V.rh, n);
    tp = cta_dot(V.r, V.r, i2, j2, red, &sc[S_TP]);
    res = sqrt(tp);
    if (res < tol) break;
    while (sqrt(tp) / res > tol) {
      iter = iter + 1;
      const double rhn = cta_dot(V.r, V.rh, i2, j2, red, &sc[S_RHN]);
      if (tid == 0)
        sc[S_BETA] = __dmul_rn(__ddiv_rn(rhn, sc[S_RHO]), __ddiv_rn(sc[S_ALPHA], sc[S_W]));
      __syncthreads();
      cta_p(V.r, V.p, V.v, V.ph, sc[S_BETA], sc[S_W], n);
      cta_boundary(V.ph, i2, j2, periodic);
      cta_apply(al, ab, ac, ar, at, V.ph, V.v, i2, j2);
      cta_boundary(V.v, i2, j2, periodic);
      const double tmp = cta_dot(V.rh, V.v, i2, j2, red, &sc[S_TMP]);
      if (tid == 0) sc[S_ALPHA] = __ddiv_rn(rhn, tmp);
      __syncthreads();
      cta_s(V.r, V.v, V.s, V.sh, sc[S_ALPHA], n);
      cta_boundary(V.sh, i2, j2, periodic);
      cta_apply(al, ab, ac, ar, at, V.sh, V.t, i2, j2);
      cta_boundary(V.t, i2, j2, periodic);
      const double tt = cta_dot(V.t, V.t, i2, j2, red, &sc[S_TT]);
      const double ts = cta_dot(V.t, V.s, i2, j2, red, &sc[S_TS]);
      if (tid == 0) sc[S_W] = __ddiv_rn(ts, tt);
      __syncthreads();
      cta_xr(x, V.r, V.ph, V.sh, V.s, V.t, sc[S_ALPHA], sc[S_W], n);
      tp = cta_dot(V.r, V.r, i2, j2, red, &sc[S_TP]);
      if (tid == 0) sc[S_RHO] = rhn;
      __syncthreads();
      if (!isfinite(tp)) {
        nonfinite = true;
        break;
      }
      if (iter % 100 == 0) break;
    }
    if (nonfinite) break;
  }
  if (!nonfinite) cta_boundary(x, i2, j2, periodic);
  if (tid == 0) {
    out[0] = (double)iter;
    out[1] = tp;
    out[2] = nonfinite ? 1.0 : 0.0;
  }
}

// CSI: q = omega*work1 + (csy*omega - 1)*q; x = x + q
__global__ void k_csi_qx(const double *work1, double *q, double *x, double omega, double csy,
                         size_t n, int first) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double qv;
    if (first)
      qv = mul(__ddiv_rn(1.0, csy), work1[k]);
    else
      qv = add(mul(omega, work1[k]), mul(sub(mul(csy, omega), 1.0), q[k]));
    q[k] = qv;
    x[k] = add(x[k], qv);
  }
}

// Lanczos: out = a - alpha*b - c ; or out = a / d
__global__ void k_lz_update(double *v, const double *s, const double *work, double alpha, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    v[k] = sub(sub(s[k], mul(alpha, v[k])), work[k]);
}
__global__ void k_scale_copy(double *dst, const double *src, double a, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = mul(a, src[k]);
}
__global__ void k_div(double *v, double d, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    v[k] = __ddiv_rn(v[k], d);
}
__global__ void k_fill(double *v, double a, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    v[k] = a;
}

// ------------------------------------------------------------ host side
namespace {
struct Work {
  std::vector<double *> bufs;
  double *partials = nullptr;
  unsigned *ticket = nullptr;
  double *sc = nullptr;  // device scalars
  double *hsc = nullptr; // pinned mirror
  ~Work() {
    for (double *b : bufs) cudaFree(b);
    if (partials) cudaFree(partials);
    if (ticket) cudaFree(ticket);
    if (sc) cudaFree(sc);
    if (hsc) cudaFreeHost(hsc);
  }
  // the state init leaves: every buffer, the ticket and the scalars zero
  int zero(size_t n, cudaStream_t st) {
    for (double *b : bufs) SEVP_CUDA_TRY(cudaMemsetAsync(b, 0, n * 8, st));
    SEVP_CUDA_TRY(cudaMemsetAsync(ticket, 0, 8, st));
    SEVP_CUDA_TRY(cudaMemsetAsync(sc, 0, S_NSC * 8, st));
    return SEVP_OK;
  }
  int init(int nvec, size_t n, cudaStream_t st) {
    bufs.assign(nvec, nullptr);
    for (auto &b : bufs) {
      SEVP_CUDA_TRY(cudaMalloc((void **)&b, n * 8));
      SEVP_CUDA_TRY(cudaMemsetAsync(b, 0, n * 8, st));
    }
    SEVP_CUDA_TRY(cudaMalloc((void **)&partials, 1024 * 8));
    SEVP_CUDA_TRY(cudaMalloc((void **)&ticket, 8));
    SEVP_CUDA_TRY(cudaMemsetAsync(ticket, 0, 8, st));
    SEVP_CUDA_TRY(cudaMalloc((void **)&sc, S_NSC * 8));
    SEVP_CUDA_TRY(cudaMemsetAsync(sc, 0, S_NSC * 8, st));
    SEVP_CUDA_TRY(cudaMallocHost((void **)&hsc, S_NSC * 8));
    return SEVP_OK;
  }
};

// Work buffers kept between calls while the drop-in cache is on
// (sevp_dropin_cache): one set per (device, vectors, length), zeroed again
// for every call, so repeated calls allocate nothing (the pinned scalar
// mirror costs the most).
struct KeptWork {
  int device, nvec;
  size_t n;
  Work *w;
};
std::vector<KeptWork> g_kept_work;

// The buffers of one Krylov call: the kept set while caching is on, else a
// set owned by the call.
class CallWork {
  std::unique_ptr<Work> own_;
  Work *w_ = nullptr;

 public:
  int acquire(int nvec, size_t n, cudaStream_t st) {
    if (dropin_cache_on()) {
      int dev = 0;
      SEVP_CUDA_TRY(cudaGetDevice(&dev));
      for (const KeptWork &k : g_kept_work)
        if (k.device == dev && k.nvec == nvec && k.n == n) {
          w_ = k.w;
          return w_->zero(n, st);
        }
      std::unique_ptr<Work> w(new Work);
      int s = w->init(nvec, n, st);
      if (s) return s;
      w_ = w.get();
      g_kept_work.push_back(KeptWork{dev, nvec, n, w.release()});
      return SEVP_OK;
    }
    own_.reset(new Work);
    w_ = own_.get();
    return w_->init(nvec, n, st);
  }
  Work &get() { return *w_; }
};

unsigned dot_blocks(int i2, int j2) {
  size_t n = (size_t)i2 * j2;
  size_t b = (n + kDotThreads * 8 - 1) / (kDotThreads * 8);
  return (unsigned)std::max<size_t>(1, std::min<size_t>(b, 1024));
}
unsigned ew_blocks(size_t n) { return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 4096)); }
}  // namespace

int dev_sqprod(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
               const double *x, double *r, int i2, int j2, int transpose, cudaStream_t st) {
  dim3 blk(32, 8), grd((i2 + 31) / 32, (j2 + 7) / 8);
  if (transpose)
    k_sqprod_t<<<grd, blk, 0, st>>>(al, ab, ac, ar, at, x, r, i2, j2);
  else
    k_sqprod<<<grd, blk, 0, st>>>(al, ab, ac, ar, at, x, r, i2, j2);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

static int dot_into(const double *a, const double *b, int i2, int j2, double *out_dev, Work &w,
                    cudaStream_t st) {
  k_inprod<<<dot_blocks(i2, j2), kDotThreads, 0, st>>>(a, b, i2, j2, w.partials, w.ticket, out_dev);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int dev_inprod(const double *r, const double *p, int i2, int j2, double *result_host,
               cudaStream_t st) {
  CallWork cw;
  int s = cw.acquire(0, 1, st);
  if (s) return s;
  Work &w = cw.get();
  s = dot_into(r, p, i2, j2, w.sc, w, st);
  if (s) return s;
  SEVP_CUDA_TRY(cudaMemcpyAsync(result_host, w.sc, 8, cudaMemcpyDeviceToHost, st));
  SEVP_CUDA_TRY(cudaStreamSynchronize(st));
  return SEVP_OK;
}

int dev_boundary(double *x, int i2, int j2, cudaStream_t st) {
  k_boundary<<<std::max(1, (j2 + 255) / 256), 256, 0, st>>>(x, i2, j2);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

#define TRY(e)            \
  do {                    \
    int s_ = (e);         \
    if (s_) return s_;    \
  } while (0)

// M/sevp.f90:443-552
int dev_bicgstab(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const float *b, double *x, int i2, int j2, int periodic,
                 int *iters, double *final_res, cudaStream_t st) {
  const size_t n = (size_t)(i2 + 2) * (j2 + 2);
  CallWork cw;
  TRY(cw.acquire(8, n, st));
  Work &w = cw.get();
  double *r = w.bufs[0], *rh = w.bufs[1], *p = w.bufs[2], *v = w.bufs[3], *s = w.bufs[4],
         *t = w.bufs[5], *ph = w.bufs[6], *sh = w.bufs[7];
  const double tol = (double)1e-8f;
  if (n <= kCtaMaxPoints) {
    // small grid: the whole solve in one thread block, one launch
    k_bicgstab_cta<<<1, kCtaThreads, 0, st>>>(al, ab, ac, ar, at, b, x,
                                              BicgVecs{r, rh, p, v, s, t, ph, sh}, i2, j2,
                                              periodic, tol, w.partials);
    SEVP_CUDA_TRY(cudaGetLastError());
    double out[3];
    SEVP_CUDA_TRY(cudaMemcpyAsync(out, w.partials, sizeof out, cudaMemcpyDeviceToHost, st));
    SEVP_CUDA_TRY(cudaStreamSynchronize(st));
    *iters = (int)out[0];
    if (out[2] != 0.0) {
      *final_res = out[1];
      return SEVP_NONFINITE;
    }
    *final_res = std::sqrt(out[1]);
    return (std::sqrt(out[1]) > tol) ? SEVP_MAXITER : SEVP_OK;
  }
  auto bdry = [&](double *a) { return periodic ? dev_boundary(a, i2, j2, st) : SEVP_OK; };
  auto fetch = [&]() -> int {
    SEVP_CUDA_TRY(cudaMemcpyAsync(w.hsc, w.sc, S_NSC * 8, cudaMemcpyDeviceToHost, st));
    SEVP_CUDA_TRY(cudaStreamSynchronize(st));
    return SEVP_OK;
  };
  int iter = 0;
  double tp = 1.0, res = 0.0;
  TRY(bdry(x));
  while (std::sqrt(tp) > tol && iter < 1000) {
    k_bicg_scal<<<1, 1, 0, st>>>(w.sc, 4);
    TRY(dev_sqprod(al, ab, ac, ar, at, x, r, i2, j2, 0, st));
    k_rhs_minus<<<ew_blocks((size_t)i2 * j2), 256, 0, st>>>(b, r, i2, j2);
    TRY(bdry(r));
    SEVP_CUDA_TRY(cudaMemcpyAsync(rh, r, n * 8, cudaMemcpyDeviceToDevice, st));
    TRY(dot_into(r, r, i2, j2, w.sc + S_TP, w, st));
    TRY(fetch());
    tp = w.hsc[S_TP];
    res = std::sqrt(tp);
    if (res < tol) break;
    while (std::sqrt(tp) / res > tol) {
      iter = iter + 1;
      TRY(dot_into(r, rh, i2, j2, w.sc + S_RHN, w, st));
      k_bicg_scal<<<1, 1, 0, st>>>(w.sc, 0);
      k_bicg_p<<<ew_blocks(n), 256, 0, st>>>(r, p, v, ph, w.sc, n);
      TRY(bdry(ph));
      TRY(dev_sqprod(al, ab, ac, ar, at, ph, v, i2, j2, 0, st));
      TRY(bdry(v));
      TRY(dot_into(rh, v, i2, j2, w.sc + S_TMP, w, st));
      k_bicg_scal<<<1, 1, 0, st>>>(w.sc, 1);
      k_bicg_s<<<ew_blocks(n), 256, 0, st>>>(r, v, s, sh, w.sc, n);
      TRY(bdry(sh));
      TRY(dev_sqprod(al, ab, ac, ar, at, sh, t, i2, j2, 0, st));
      TRY(bdry(t));
      TRY(dot_into(t, t, i2, j2, w.sc + S_TT, w, st));
      TRY(dot_into(t, s, i2, j2, w.sc + S_TS, w, st));
      k_bicg_scal<<<1, 1, 0, st>>>(w.sc, 2);
      k_bicg_xr<<<ew_blocks(n), 256, 0, st>>>(x, r, ph, sh, s, t, w.sc, n);
      TRY(dot_into(r, r, i2, j2, w.sc + S_TP, w, st));
      k_bicg_scal<<<1, 1, 0, st>>>(w.sc, 3);
      TRY(fetch());
      tp = w.hsc[S_TP];
      if (!std::isfinite(tp)) {
        *iters = iter;
        *final_res = tp;
        return SEVP_NONFINITE;
      }
      if (iter % 100 == 0) break;
    }
  }
  TRY(bdry(x));
  SEVP_CUDA_TRY(cudaStreamSynchronize(st));
  *iters = iter;
  *final_res = std::sqrt(tp);
  return (std::sqrt(tp) > tol) ? SEVP_MAXITER : SEVP_OK;
}

// M/sevp.f90:553-616
int dev_csi(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
            double mineig, double maxeig, const float *b, double *x, int i2, int j2, int periodic,
            int *iters, double *final_res, cudaStream_t st) {
  const size_t n = (size_t)(i2 + 2) * (j2 + 2);
  CallWork cw;
  TRY(cw.acquire(4, n, st));  // r, s, q, work1 all start at zero, as in the reference
  Work &w = cw.get();
  double *r = w.bufs[0], *s = w.bufs[1], *q = w.bufs[2], *work1 = w.bufs[3];
  auto bdry = [&](double *a) { return periodic ? dev_boundary(a, i2, j2, st) : SEVP_OK; };
  const double tol = (double)1e-7f;
  int iter = 0;
  double tp = 1.0;
  const double alpha = 2.0 / (maxeig - mineig);
  const double beta = (maxeig + mineig) / (maxeig - mineig);
  const double csy = beta / alpha;
  double omega = 2.0 / csy;
  const unsigned eb = ew_blocks(n), ebi = ew_blocks((size_t)i2 * j2);
  TRY(bdry(x));
  TRY(dev_sqprod(al, ab, ac, ar, at, x, s, i2, j2, 0, st));
  TRY(bdry(s));
  k_b_minus<<<ebi, 256, 0, st>>>(b, s, r, i2, j2);
  SEVP_CUDA_TRY(cudaMemcpyAsync(work1, r, n * 8, cudaMemcpyDeviceToDevice, st));
  TRY(bdry(work1));
  k_csi_qx<<<eb, 256, 0, st>>>(work1, q, x, omega, csy, n, 1);
  TRY(dev_sqprod(al, ab, ac, ar, at, x, s, i2, j2, 0, st));
  TRY(bdry(s));
  k_b_minus<<<ebi, 256, 0, st>>>(b, s, r, i2, j2);
  while (std::sqrt(tp) > tol && iter < 1000) {
    omega = 1.0 / (csy - omega / (4.0 * alpha * alpha));
    SEVP_CUDA_TRY(cudaMemcpyAsync(work1, r, n * 8, cudaMemcpyDeviceToDevice, st));
    TRY(bdry(work1));
    k_csi_qx<<<eb, 256, 0, st>>>(work1, q, x, omega, csy, n, 0);
    TRY(dev_sqprod(al, ab, ac, ar, at, x, s, i2, j2, 0, st));
    k_b_minus<<<ebi, 256, 0, st>>>(b, s, r, i2, j2);
    TRY(bdry(r));
    TRY(dot_into(r, r, i2, j2, w.sc + S_TP, w, st));
    SEVP_CUDA_TRY(cudaMemcpyAsync(w.hsc, w.sc, S_NSC * 8, cudaMemcpyDeviceToHost, st));
    SEVP_CUDA_TRY(cudaStreamSynchronize(st));
    tp = w.hsc[S_TP];
    iter = iter + 1;
    if (!std::isfinite(tp)) {
      *iters = iter;
      *final_res = tp;
      return SEVP_NONFINITE;
    }
  }
  TRY(bdry(x));
  SEVP_CUDA_TRY(cudaStreamSynchronize(st));
  *iters = iter;
  *final_res = std::sqrt(tp);
  return (std::sqrt(tp) > tol) ? SEVP_MAXITER : SEVP_OK;
}

// M/sevp.f90:618-694.  The reference writes sigma(m+1)/beta(m+1) one past
// its arrays and leaves the ghost ring of its locals s and q uninitialised;
// here those arrays have m+2 entries and the locals start at zero.
int dev_lanczos(const float *al, const float *ab, const float *ac, const float *ar,
                const float *at, int i2, int j2, double *mineig, double *maxeig, cudaStream_t st) {
  enum { M = 10 };
  const size_t n = (size_t)(i2 + 2) * (j2 + 2);
  CallWork cw;
  TRY(cw.acquire(7, n, st));
  Work &w = cw.get();
  double *v = w.bufs[0], *ww = w.bufs[1], *vp = w.bufs[2], *wp = w.bufs[3], *s = w.bufs[4],
         *q = w.bufs[5], *work = w.bufs[6];
  const unsigned eb = ew_blocks(n);
  double alpha[M + 2] = {0}, beta[M + 2] = {0}, sigma[M + 2] = {0};
  auto dot = [&](const double *a, const double *b2, double *out) -> int {
    TRY(dot_into(a, b2, i2, j2, w.sc + S_TP, w, st));
    SEVP_CUDA_TRY(cudaMemcpyAsync(w.hsc, w.sc, S_NSC * 8, cudaMemcpyDeviceToHost, st));
    SEVP_CUDA_TRY(cudaStreamSynchronize(st));
    *out = w.hsc[S_TP];
    return SEVP_OK;
  };
  double tp;
  k_fill<<<eb, 256, 0, st>>>(v, 1.0, n);
  TRY(dot(v, v, &tp));
  k_scale_copy<<<eb, 256, 0, st>>>(v, v, 1 / std::sqrt(tp), n);
  SEVP_CUDA_TRY(cudaMemcpyAsync(ww, v, n * 8, cudaMemcpyDeviceToDevice, st));
  int iter = 0;
  while (iter < M) {
    iter = iter + 1;
    TRY(dev_sqprod(al, ab, ac, ar, at, v, s, i2, j2, 0, st));
    TRY(dot(s, ww, &tp));
    alpha[iter] = tp;
    k_scale_copy<<<eb, 256, 0, st>>>(work, vp, beta[iter], n);
    SEVP_CUDA_TRY(cudaMemcpyAsync(vp, v, n * 8, cudaMemcpyDeviceToDevice, st));
    k_lz_update<<<eb, 256, 0, st>>>(v, s, work, alpha[iter], n);
    TRY(dev_sqprod(al, ab, ac, ar, at, ww, q, i2, j2, 1, st));
    k_scale_copy<<<eb, 256, 0, st>>>(work, wp, sigma[iter], n);
    SEVP_CUDA_TRY(cudaMemcpyAsync(wp, ww, n * 8, cudaMemcpyDeviceToDevice, st));
    k_lz_update<<<eb, 256, 0, st>>>(ww, q, work, alpha[iter], n);
    TRY(dot(v, ww, &tp));
    sigma[iter + 1] = std::sqrt(std::fabs(tp));
    beta[iter + 1] = std::copysign(sigma[iter + 1], tp);
    k_div<<<eb, 256, 0, st>>>(v, sigma[iter + 1], n);
    k_div<<<eb, 256, 0, st>>>(ww, beta[iter + 1], n);
  }
  TRY(dev_sqprod(al, ab, ac, ar, at, v, s, i2, j2, 0, st));
  TRY(dot(s, ww, &tp));
  alpha[M] = tp;
  double t[M * 3] = {0}, mcsa[M] = {0}, mcsb[M] = {0}, mcsb2[M] = {0};
  for (int k = 2; k <= M; ++k) t[IXK(M, k, 1)] = sigma[k];
  for (int k = 1; k <= M; ++k) t[IXK(M, k, 2)] = alpha[k];
  for (int k = 1; k <= M - 1; ++k) t[IXK(M, k, 3)] = sigma[k + 1];
  int ierr = host_figi(M, t, mcsa, mcsb, mcsb2);
  double mx = mcsa[0] + mcsb[0];
  for (int k = 2; k <= M; ++k) mx = std::max(mx, mcsa[k - 1] + mcsb[k - 1] + mcsb[k - 2]);
  *maxeig = mx;
  int ierr2 = host_ratqr(M, 1.0e-6, mcsa, mcsb, mineig);
  return (ierr == 0 && ierr2 == 0) ? SEVP_OK : SEVP_BREAKDOWN;
}

// M/sevp.f90:838-904
int host_figi(int n, const double *t, double *d, double *e, double *e2) {
  for (int i = 1; i <= n; ++i) {
    if (1 < i) {
      e2[i - 1] = t[IXK(n, i, 1)] * t[IXK(n, i - 1, 3)];
      if (e2[i - 1] < 0.0) return n + i;
      if (e2[i - 1] == 0.0) {
        if (t[IXK(n, i, 1)] != 0.0 || t[IXK(n, i - 1, 3)] != 0.0) return -3 * n - i;
        e[i - 1] = 0.0;
      } else {
        e[i - 1] = std::sqrt(e2[i - 1]);
      }
    }
    d[i - 1] = t[IXK(n, i, 2)];
  }
  return 0;
}

// M/sevp.f90:906-1006: smallest eigenvalue of a positive definite symmetric
// tridiagonal matrix by rational QR with Newton corrections.
int host_ratqr(int n, double eps1, const double *d, const double *e, double *mineig) {
  std::vector<double> bd(n + 1, 0.0), wv(n + 1, 0.0);
  int i;
  double f, ep, delta = 0.0, err = 0.0, p, q = 0.0, qp = 0.0, r, s = 0.0, tot;
  for (i = 1; i <= n; ++i) wv[i] = d[i - 1];
  tot = wv[1];
  for (i = 1; i <= n; ++i) {
    p = q;
    bd[i] = e[i - 1] * e[i - 1];
    q = 0.0;
    if (i != n) q = std::fabs(e[i]);
    tot = std::min(wv[i] - p - q, tot);
  }
  bd[1] = 0.0;
  if (tot < 0.0)
    tot = 0.0;
  else
    for (i = 1; i <= n; ++i) wv[i] = wv[i] - tot;
  // The reference loops without bound; NaN/Inf input never meets its exits,
  // so stop after 100000 sweeps and report ierr = 2.
  for (int sweep = 0;; ++sweep) {
    if (sweep >= 100000) return 2;
    tot = tot + s;
    delta = wv[n] - s;
    i = n;
    if (delta <= eps1) break;
    f = bd[n] / delta;
    qp = delta + f;
    p = 1.0;
    for (int ii = 1; ii <= n - 1; ++ii) {
      i = n - ii;
      q = wv[i] - s - f;
      r = q / qp;
      p = p * r + 1.0;
      ep = f * r;
      wv[i + 1] = qp + ep;
      delta = q - ep;
      if (delta <= eps1) break;
      f = bd[i] / q;
      qp = delta + f;
      bd[i + 1] = qp * ep;
    }
    if (delta <= eps1) break;
    wv[1] = qp;
    s = qp / p;
    if (tot + s <= tot) return 1;
  }
  wv[1] = tot;
  err = err + std::fabs(delta);
  bd[1] = err;
  *mineig = wv[1];
  return 0;
}

// Frees the Work sets kept for the drop-in cache (sevp_dropin_cache).
void release_kept_work() {
  for (const KeptWork &k : g_kept_work) delete k.w;
  g_kept_work.clear();
}

}  // namespace sevp

