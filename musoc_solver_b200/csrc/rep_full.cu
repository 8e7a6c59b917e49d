// Reference-faithful SEVP drop-ins on the GPU: the full-width and strip
// marching solves (REP1, REP, REPBIR, REPBIR_PERIOD, M/sevp.f90:11-438), the
// influence precompute (PRE1, PRE, P/prep_GLOBAL.f90:327-513), the
// no-pivoting Gauss-Jordan inverse (MATINV, P/prep_GLOBAL.f90:516-568) and the
// overlapping-strip sweeps of FS_SOLVER (M/fs_GLOBAL.f90:1904-1966).
//
// Every floating-point step uses explicitly rounded intrinsics (__dmul_rn,
// __dadd_rn, __dsub_rn, __ddiv_rn: no contraction into fused multiply-adds)
// and the reference's evaluation order, including the serial order of the
// mat-vec and GEMM sums, so the results are bit-identical to an IEEE-754
// double evaluation of the Fortran (the CPU oracle is that evaluation).
// Parallelism is across columns (marching), across unit responses (PRE) and
// across matrix elements (MATINV, GEMM); the sequential structure of the
// method (rows, blocks) is kept.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "dropin.cuh"

namespace sevp {

#define IXD(ld, i, j) ((size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1))

__device__ __forceinline__ double c64(const float *a, int ld, int i, int j) {
  return (double)a[IXD(ld, i, j)];
}
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// (F - AX*V_W - AY*V_S - BB*V_C - CX*V_E) / CY   (M/sevp.f90:29-30)
__device__ __forceinline__ double march_val(const MarchArgs &a, const double *v, int ldv, int i,
                                            int j, double f) {
  double t = sub(f, mul(c64(a.ax, a.ldc, i, j), v[IXD(ldv, i, j + 1)]));
  t = sub(t, mul(c64(a.ay, a.ldc, i, j), v[IXD(ldv, i + 1, j)]));
  t = sub(t, mul(c64(a.bb, a.ldc, i, j), v[IXD(ldv, i + 1, j + 1)]));
  t = sub(t, mul(c64(a.cx, a.ldc, i, j), v[IXD(ldv, i + 2, j + 1)]));
  return dvd(t, c64(a.cy, a.ldc, i, j));
}

// residual of equation row j (M/sevp.f90:37-38)
__device__ __forceinline__ double resid_val(const MarchArgs &a, int i, int j) {
  const double *x = a.x;
  const int ld = a.ldx;
  double t = sub((double)a.f[IXD(a.ldf, i, j)], mul(c64(a.ax, a.ldc, i, j), x[IXD(ld, i, j + 1)]));
  t = sub(t, mul(c64(a.ay, a.ldc, i, j), x[IXD(ld, i + 1, j)]));
  t = sub(t, mul(c64(a.bb, a.ldc, i, j), x[IXD(ld, i + 1, j + 1)]));
  t = sub(t, mul(c64(a.cx, a.ldc, i, j), x[IXD(ld, i + 2, j + 1)]));
  t = sub(t, mul(c64(a.cy, a.ldc, i, j), x[IXD(ld, i + 1, j + 2)]));
  return t;
}

__device__ __forceinline__ void ghost_row(double *v, int ld, int gi0, int j) {
  if (threadIdx.x == 0) {
    v[IXD(ld, 1, j)] = v[IXD(ld, gi0 - 1, j)];
    v[IXD(ld, gi0, j)] = v[IXD(ld, 2, j)];
  }
}

// out(n) = sum_m in(m) * R(m, n), serial in m, one thread per n.  The
// column's elements are loaded kVecmatBatch at a time before they are
// summed (one memory round trip per batch instead of per element); the sum
// keeps the reference's order.
constexpr int kVecmatBatch = 16;
__device__ __forceinline__ void vecmat_serial(const double *in, const double *R, int m2,
                                              double *out) {
  for (int n = threadIdx.x; n < m2; n += blockDim.x) {
    const double *col = R + (size_t)n * m2;
    double s = 0.0;
    int k = 0;
    for (; k + kVecmatBatch <= m2; k += kVecmatBatch) {
      double c[kVecmatBatch], v[kVecmatBatch];
#pragma unroll
      for (int q = 0; q < kVecmatBatch; ++q) {
        c[q] = col[k + q];
        v[q] = in[k + q];
      }
#pragma unroll
      for (int q = 0; q < kVecmatBatch; ++q) s = add(s, mul(v[q], c[q]));
    }
    for (; k < m2; ++k) s = add(s, mul(in[k], col[k]));
    out[n] = s;
  }
}

// One CTA runs the whole marching solve (forward and backward sweeps).
__global__ void __launch_bounds__(1024) k_march_solve(MarchArgs a) {
  const int m2 = a.m2;
  const size_t msz = (size_t)m2 * m2;
  double *X = a.x, *H = a.h;
  const int ldx = a.ldx, ldh = a.ldh;
  const int tid = threadIdx.x, nt = blockDim.x;
  int js = 1;
  for (int nb = 1; nb <= a.nblk; ++nb) {
    const int jf = a.ie[nb - 1] - 2;
    for (int j = js; j <= jf; ++j) {
      if (a.periodic) ghost_row(X, ldx, a.gi0, j + 1);
      __syncthreads();
      for (int i = 1 + tid; i <= m2; i += nt)
        X[IXD(ldx, i + 1, j + 2)] = march_val(a, X, ldx, i, j, (double)a.f[IXD(a.ldf, i, j)]);
      __syncthreads();
    }
    if (a.periodic) ghost_row(X, ldx, a.gi0, jf + 2);
    __syncthreads();
    if (nb != a.nblk) {
      int j = a.ie[nb - 1] - 1;
      for (int i = 1 + tid; i <= m2; i += nt) a.dum1[i - 1] = resid_val(a, i, j);
      __syncthreads();
      j = a.ie[nb - 1];
      vecmat_serial(a.dum1, a.rinv1 + (size_t)(nb - 1) * msz, m2, a.dum2);
      __syncthreads();
      for (int n = 1 + tid; n <= m2; n += nt) {
        a.dum0[IXD(m2, n, nb)] = X[IXD(ldx, n + 1, j)];
        X[IXD(ldx, n + 1, j)] = sub(X[IXD(ldx, n + 1, j)], a.dum2[n - 1]);
      }
      __syncthreads();
      if (a.periodic) ghost_row(X, ldx, a.gi0, j);
      __syncthreads();
    }
    js = a.ie[nb - 1];
  }
  for (int nbs = 1; nbs <= a.nblk; ++nbs) {
    const int nb = a.nblk - nbs + 1;
    js = (nb != 1) ? a.ie[nb - 2] : 1;
    const int jf = a.ie[nb - 1] - 2;
    if (nb != a.nblk) {
      const int j = a.ie[nb - 1];
      for (int n = 1 + tid; n <= m2; n += nt) X[IXD(ldx, n + 1, j)] = a.dum0[IXD(m2, n, nb)];
    }
    for (int j = js; j <= a.ie[nb - 1]; ++j)
      for (int i = 1 + tid; i <= a.hzero; i += nt) H[IXD(ldh, i, j)] = 0.0;
    __syncthreads();
    int j = a.ie[nb - 1] - 1;
    if (a.periodic) ghost_row(X, ldx, a.gi0, j + 1);
    __syncthreads();
    for (int i = 1 + tid; i <= m2; i += nt) a.dum1[i - 1] = resid_val(a, i, j);
    __syncthreads();
    vecmat_serial(a.dum1, a.rinv + (size_t)(nb - 1) * msz, m2, a.dum2);
    __syncthreads();
    for (int n = 1 + tid; n <= m2; n += nt) {
      H[IXD(ldh, n + 1, js + 1)] = a.dum2[n - 1];
      X[IXD(ldx, n + 1, js + 1)] = add(X[IXD(ldx, n + 1, js + 1)], a.dum2[n - 1]);
    }
    __syncthreads();
    if (a.periodic) {
      ghost_row(H, ldh, a.gi0, js + 1);
      ghost_row(X, ldx, a.gi0, js + 1);
    }
    __syncthreads();
    if (nb != 1) {
      for (int k = 1 + tid; k <= m2; k += nt)
        a.dum1[k - 1] = mul(H[IXD(ldh, k + 1, js + 1)], c64(a.cy, a.ldc, k, js - 1));
      __syncthreads();
      j = a.ie[nb - 2];
      vecmat_serial(a.dum1, a.rinv1 + (size_t)(nb - 2) * msz, m2, a.dum2);
      __syncthreads();
      for (int n = 1 + tid; n <= m2; n += nt) H[IXD(ldh, n + 1, j)] = a.dum2[n - 1];
      __syncthreads();
      if (a.periodic) ghost_row(H, ldh, a.gi0, j);
      __syncthreads();
    }
    for (j = js; j <= jf; ++j) {
      if (a.periodic) ghost_row(H, ldh, a.gi0, j + 1);
      __syncthreads();
      for (int i = 1 + tid; i <= m2; i += nt) {
        double hv = march_val(a, H, ldh, i, j, 0.0);
        H[IXD(ldh, i + 1, j + 2)] = hv;
        X[IXD(ldx, i + 1, j + 2)] = add(X[IXD(ldx, i + 1, j + 2)], hv);
      }
      __syncthreads();
      if (a.periodic) ghost_row(X, ldx, a.gi0, j + 2);
      __syncthreads();
    }
  }
  if (a.periodic) {
    for (int j = 2 + tid; j <= a.ie[a.nblk - 1]; j += nt) {
      X[IXD(ldx, 1, j)] = X[IXD(ldx, a.gi0 - 1, j)];
      X[IXD(ldx, a.gi0, j)] = X[IXD(ldx, 2, j)];
    }
  }
}

// ---------------------------------------------------------------- PRE
// One CTA per unit response NG of block nb.  Its H slice has leading
// dimension ldh and holds padded rows jl .. jhp (local row = row - jl).
__device__ __forceinline__ double lhs4(const PreArgs &p, const double *H, int i, int j, int jl) {
  const int ld = p.ldh;
  double t = mul(c64(p.ax, p.ldc, i, j), H[IXD(ld, i, j + 1 - jl + 1)]);
  t = add(t, mul(c64(p.ay, p.ldc, i, j), H[IXD(ld, i + 1, j - jl + 1)]));
  t = add(t, mul(c64(p.bb, p.ldc, i, j), H[IXD(ld, i + 1, j + 1 - jl + 1)]));
  t = add(t, mul(c64(p.cx, p.ldc, i, j), H[IXD(ld, i + 2, j + 1 - jl + 1)]));
  return t;
}

__device__ __forceinline__ void ghost_local(double *H, int ld, int gi0, int row_local) {
  if (threadIdx.x == 0) {
    H[IXD(ld, 1, row_local)] = H[IXD(ld, gi0 - 1, row_local)];
    H[IXD(ld, gi0, row_local)] = H[IXD(ld, 2, row_local)];
  }
}

__global__ void __launch_bounds__(256) k_pre_units(PreArgs p, int nb, int jl) {
  const int ng = blockIdx.x + 1;
  const int m2 = p.m2;
  const size_t msz = (size_t)m2 * m2;
  const int jh = p.ie[nb - 1], jhp = jh + 1, jhm = jh - 2, jg = jl + 1, ig = ng + 1;
  const int rows = jhp - jl + 1;
  double *H = p.hwork + (size_t)blockIdx.x * p.ldh * rows;  // local rows 1..rows
  const int tid = threadIdx.x, nt = blockDim.x;
  double *R = p.rinv + (size_t)(nb - 1) * msz;
  double *Rs = p.rinv + (size_t)(p.nblk - 1) * msz;
  // local row index of padded row r is r - jl + 1
#define LR(r) ((r) - jl + 1)
  for (int e = tid; e < p.hzero * rows; e += nt) H[e % p.hzero + (size_t)(e / p.hzero) * p.ldh] = 0.0;
  __syncthreads();
  if (tid == 0) H[IXD(p.ldh, ig, LR(jg))] = 1.0;
  __syncthreads();
  if (p.periodic) ghost_local(H, p.ldh, p.gi0, LR(jg));
  __syncthreads();
  if (nb != 1) {
    const double *R1p = p.rinv1 + (size_t)(nb - 2) * msz;
    const double cyv = c64(p.cy, p.ldc, ig - 1, jg - 2);
    for (int n = 1 + tid; n <= m2; n += nt) H[IXD(p.ldh, n + 1, LR(jl))] = mul(R1p[IXD(m2, ng, n)], cyv);
    __syncthreads();
  }
  for (int j = jl; j <= jhm; ++j) {
    if (p.periodic) ghost_local(H, p.ldh, p.gi0, LR(j + 1));
    __syncthreads();
    for (int i = 1 + tid; i <= m2; i += nt) {
      double t = lhs4(p, H, i, j, jl);
      H[IXD(p.ldh, i + 1, LR(j + 2))] = -dvd(t, c64(p.cy, p.ldc, i, j));
    }
    __syncthreads();
  }
  int j = jh - 1;
  if (p.periodic) ghost_local(H, p.ldh, p.gi0, LR(j + 1));
  __syncthreads();
  for (int i = 1 + tid; i <= m2; i += nt) R[IXD(m2, ng, i)] = lhs4(p, H, i, j, jl);
  if (nb != p.nblk) {
    j = p.ie[nb - 1];
    for (int n = 1 + tid; n <= m2; n += nt) Rs[IXD(m2, ng, n)] = H[IXD(p.ldh, n + 1, LR(j))];
    __syncthreads();
    if (p.periodic && tid == 0) {
      H[IXD(p.ldh, 1, LR(jg))] = 0.0;
      H[IXD(p.ldh, p.gi0, LR(jg))] = 0.0;
    }
  }
  __syncthreads();
  if (tid == 0) H[IXD(p.ldh, ig, LR(jg))] = 0.0;
#undef LR
}

// RINV1(I,J) = -sum_K RINV(I,K) * S(K,J), serial in K (P/prep_GLOBAL.f90:379-383)
__global__ void k_rinv1_gemm(const double *R, const double *S, double *R1, int m2) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > m2 || j > m2) return;
  double s = 0.0;
  for (int k = 1; k <= m2; ++k) s = sub(s, mul(R[IXD(m2, i, k)], S[IXD(m2, k, j)]));
  R1[IXD(m2, i, j)] = s;
}

// ------------------------------------------------------------- MATINV
// Small matrices: whole inverse in one CTA.
__global__ void __launch_bounds__(1024) k_matinv_cta(double *B, int n, double *b1, double *b2,
                                                   int *bad) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = 1; i <= n - 1; ++i) {
    const double piv = B[IXD(n, i, i)];
    if (tid == 0 && piv == 0.0) *bad = 1;
    const double r = dvd(1.0, piv);
    __syncthreads();
    if (tid == 0) B[IXD(n, i, i)] = 1.0;
    __syncthreads();
    for (int j = 1 + tid; j <= n; j += nt) B[IXD(n, i, j)] = mul(B[IXD(n, i, j)], r);
    for (int ia = i + 1 + tid; ia <= n; ia += nt) b1[ia] = B[IXD(n, ia, i)];
    __syncthreads();
    for (int ia = i + 1 + tid; ia <= n; ia += nt) B[IXD(n, ia, i)] = 0.0;
    for (int j = 1 + tid; j <= n; j += nt) b2[j] = B[IXD(n, i, j)];
    __syncthreads();
    const int rows = n - i;
    for (int e = tid; e < rows * n; e += nt) {
      const int ia = i + 1 + e % rows, j = 1 + e / rows;
      B[IXD(n, ia, j)] = sub(B[IXD(n, ia, j)], mul(b1[ia], b2[j]));
    }
    __syncthreads();
  }
  {
    const double piv = B[IXD(n, n, n)];
    if (tid == 0 && piv == 0.0) *bad = 1;
    const double r = dvd(1.0, piv);
    __syncthreads();
    if (tid == 0) B[IXD(n, n, n)] = 1.0;
    __syncthreads();
    for (int j = 1 + tid; j <= n; j += nt) B[IXD(n, n, j)] = mul(B[IXD(n, n, j)], r);
    __syncthreads();
  }
  for (int i = 2; i <= n; ++i) {
    for (int ib = 1 + tid; ib <= i; ib += nt) b1[ib] = B[IXD(n, ib, i)];
    __syncthreads();
    for (int ib = 1 + tid; ib <= i - 1; ib += nt) B[IXD(n, ib, i)] = 0.0;
    for (int j = 1 + tid; j <= n; j += nt) b2[j] = B[IXD(n, i, j)];
    __syncthreads();
    const int rows = i - 1;
    for (int e = tid; e < rows * n; e += nt) {
      const int ib = 1 + e % rows, j = 1 + e / rows;
      B[IXD(n, ib, j)] = sub(B[IXD(n, ib, j)], mul(b1[ib], b2[j]));
    }
    __syncthreads();
  }
}

// Large matrices: one launch per elimination step.
__global__ void k_mi_pivot_row(double *B, int n, int i, double *b1, double *b2, int *bad) {
  // row i scaled by 1/B(i,i) with B(i,i) first set to 1; column below saved
  const double piv = B[IXD(n, i, i)];
  const double r = dvd(1.0, piv);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (piv == 0.0) *bad = 1;
    B[IXD(n, i, i)] = 1.0;
  }
  __syncthreads();
  for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x) {
    double v = mul(B[IXD(n, i, j)], r);
    B[IXD(n, i, j)] = v;
    b2[j] = v;
  }
  for (int ia = i + 1 + threadIdx.x; ia <= n; ia += blockDim.x) {
    b1[ia] = B[IXD(n, ia, i)];
    B[IXD(n, ia, i)] = 0.0;
  }
}
__global__ void k_mi_update(double *B, int n, int r0, int r1, const double *b1, const double *b2) {
  const int rows = r1 - r0 + 1;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)rows * n) return;
  const int ia = r0 + (int)(e % rows), j = 1 + (int)(e / rows);
  B[IXD(n, ia, j)] = sub(B[IXD(n, ia, j)], mul(b1[ia], b2[j]));
}
__global__ void k_mi_back_prep(double *B, int n, int i, double *b1, double *b2) {
  for (int ib = 1 + threadIdx.x; ib <= i; ib += blockDim.x) b1[ib] = B[IXD(n, ib, i)];
  __syncthreads();
  for (int ib = 1 + threadIdx.x; ib <= i - 1; ib += blockDim.x) B[IXD(n, ib, i)] = 0.0;
  for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x) b2[j] = B[IXD(n, i, j)];
}

// ------------------------------------------------------- strip copies
// Extracts the wrapped last BIR strip (M/fs_GLOBAL.f90:1924-1944) or a plain
// strip source (:1910-1915).  mode 0: SRC only; mode 1: SRC, CL..CT, XX sides.
__global__ void k_strip_extract(StripArgs s, int il, int mode) {
  const int ibir = s.ibir, inc = ibir / 2, i2 = s.i2, i0 = i2 + 2;
  const int ir = il + inc, ir2 = il + ibir - 1;
  const size_t total = (size_t)ibir * s.j2;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int ii = 1 + (int)(e % ibir), j = 1 + (int)(e / ibir);
    if (mode == 0) {
      s.src[IXD(ibir, ii, j)] = s.s[IXD(i2, il + ii - 1, j)];
      continue;
    }
    const int i = il + ii - 1;
    const int is = (i <= ir - 1) ? i : i - ir + 1;
    if (s.s) s.src[IXD(ibir, ii, j)] = s.s[IXD(i2, is, j)];
    s.cl[IXD(ibir, ii, j)] = s.al[IXD(i2, is, j)];
    s.cr[IXD(ibir, ii, j)] = s.ar[IXD(i2, is, j)];
    s.cb[IXD(ibir, ii, j)] = s.ab[IXD(i2, is, j)];
    s.ct[IXD(ibir, ii, j)] = s.at[IXD(i2, is, j)];
    s.cc[IXD(ibir, ii, j)] = s.ac[IXD(i2, is, j)];
    if (ii == 1 && s.x) {
      s.xx[IXD(ibir + 2, 1, j)] = s.x[IXD(i0, il, j)];
      s.xx[IXD(ibir + 2, ibir + 2, j)] = s.x[IXD(i0, inc + 2, j)];
    }
    (void)ir2;
  }
  if (mode == 1 && s.x && blockIdx.x == 0 && threadIdx.x == 0)
    for (int j = s.j2 + 1; j <= s.side_rows; ++j) {
      s.xx[IXD(ibir + 2, 1, j)] = s.x[IXD(i0, il, j)];
      s.xx[IXD(ibir + 2, ibir + 2, j)] = s.x[IXD(i0, inc + 2, j)];
    }
}

// Copies the solved wrapped strip back (M/fs_GLOBAL.f90:1947-1962).
__global__ void k_strip_scatter(StripArgs s, int il, int periodic) {
  const int ibir = s.ibir, inc = ibir / 2, i2 = s.i2, i0 = i2 + 2, j1 = s.j2 + 1;
  const int ir = il + inc, ir2 = il + ibir - 1;
  const size_t total = (size_t)ibir * (j1 - 1);
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = il + (int)(e % ibir), j = 2 + (int)(e / ibir);
    if (i <= ir - 1)
      s.x[IXD(i0, i + 1, j)] = s.xx[IXD(ibir + 2, i - il + 2, j)];
    else if (i <= ir2)
      s.x[IXD(i0, i - ir + 2, j)] = s.xx[IXD(ibir + 2, i - il + 2, j)];
  }
}
__global__ void k_periodic_cols(double *x, int i2, int j2) {
  const int i0 = i2 + 2;
  for (int j = 2 + blockIdx.x * blockDim.x + threadIdx.x; j <= j2 + 1; j += gridDim.x * blockDim.x) {
    x[IXD(i0, 1, j)] = x[IXD(i0, i2 + 1, j)];
    x[IXD(i0, i0, j)] = x[IXD(i0, 2, j)];
  }
}

// ------------------------------------------------------------ host side
int dev_march_solve(const MarchArgs &a, cudaStream_t st) {
  int threads = std::min(1024, std::max(32, ((a.m2 + 31) / 32) * 32));
  k_march_solve<<<1, threads, 0, st>>>(a);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

int dev_matinv(double *B, int n, double *b1, double *b2, int *bad, cudaStream_t st) {
  if (n <= 320) {
    k_matinv_cta<<<1, 1024, 0, st>>>(B, n, b1, b2, bad);
    SEVP_CUDA_TRY(cudaGetLastError());
    return SEVP_OK;
  }
  const int T = 256;
  for (int i = 1; i <= n - 1; ++i) {
    k_mi_pivot_row<<<1, 1024, 0, st>>>(B, n, i, b1, b2, bad);
    size_t e = (size_t)(n - i) * n;
    k_mi_update<<<(unsigned)((e + T - 1) / T), T, 0, st>>>(B, n, i + 1, n, b1, b2);
  }
  k_mi_pivot_row<<<1, 1024, 0, st>>>(B, n, n, b1, b2, bad);
  for (int i = 2; i <= n; ++i) {
    k_mi_back_prep<<<1, 1024, 0, st>>>(B, n, i, b1, b2);
    size_t e = (size_t)(i - 1) * n;
    k_mi_update<<<(unsigned)((e + T - 1) / T), T, 0, st>>>(B, n, 1, i - 1, b1, b2);
  }
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

// PRE1 / PRE: blocks in sequence; per block all unit responses in parallel,
// then MATINV and the RINV1 product.  hfinal (ldh x J0) receives the H rows
// the reference leaves behind (the last unit response of each block).
int dev_pre(const PreArgs &p, double *hfinal, int *bad, cudaStream_t st) {
  const int m2 = p.m2;
  const size_t msz = (size_t)m2 * m2;
  int jl = 1;
  for (int nb = 1; nb <= p.nblk; ++nb) {
    const int jh = p.ie_host[nb - 1];
    const int rows = jh + 1 - jl + 1;
    k_pre_units<<<m2, 256, 0, st>>>(p, nb, jl);
    SEVP_CUDA_TRY(cudaGetLastError());
    if (hfinal) {
      // last unit response's rows jl .. jh+1
      const double *src = p.hwork + (size_t)(m2 - 1) * p.ldh * rows;
      SEVP_CUDA_TRY(cudaMemcpyAsync(hfinal + (size_t)(jl - 1) * p.ldh, src,
                                    sizeof(double) * p.ldh * rows, cudaMemcpyDeviceToDevice, st));
    }
    int s = dev_matinv(p.rinv + (size_t)(nb - 1) * msz, m2, p.b1, p.b2, bad, st);
    if (s) return s;
    if (nb == p.nblk) break;
    dim3 blk(16, 16), grd((m2 + 15) / 16, (m2 + 15) / 16);
    k_rinv1_gemm<<<grd, blk, 0, st>>>(p.rinv + (size_t)(nb - 1) * msz,
                                      p.rinv + (size_t)(p.nblk - 1) * msz,
                                      p.rinv1 + (size_t)(nb - 1) * msz, m2);
    SEVP_CUDA_TRY(cudaGetLastError());
    jl = jh;
  }
  return SEVP_OK;
}

int dev_strip_extract(const StripArgs &s, int il, int mode, cudaStream_t st) {
  k_strip_extract<<<128, 256, 0, st>>>(s, il, mode);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}
int dev_strip_scatter(const StripArgs &s, int il, int periodic, cudaStream_t st) {
  k_strip_scatter<<<128, 256, 0, st>>>(s, il, periodic);
  if (periodic) k_periodic_cols<<<8, 128, 0, st>>>(s.x, s.i2, s.j2);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

}  // namespace sevp
