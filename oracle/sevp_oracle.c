/*
 * sevp_oracle.c -- CPU FP64 oracle for the TIMCOM barotropic elliptic solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it.  The product
 * (the CUDA library under musoc_solver_b200/) never links or calls it.
 *
 * It restates, in plain C, the reference Fortran routines of the SEVP
 * (stabilized error-vector propagation) path.  Paths are relative to the
 * reference project; M/ = MAIN/template/GLOBAL/src/, P/ = PREP/template/GLOBAL/src/.
 *
 *   or_rep1            M/sevp.f90:11-107    periodic full-width marching solve
 *   or_repbir_period   M/sevp.f90:109-217   periodic strip solve (unused upstream)
 *   or_repbir          M/sevp.f90:218-328   strip solve with Dirichlet side columns
 *   or_rep             M/sevp.f90:335-438   non-periodic full-width solve
 *   or_pre1            P/prep_GLOBAL.f90:327-386   periodic influence precompute
 *   or_pre             P/prep_GLOBAL.f90:457-513   strip influence precompute
 *   or_matinv          P/prep_GLOBAL.f90:516-568   Gauss-Jordan inverse, no pivoting
 *   or_block_partition P/prep_GLOBAL.f90:148-168   block boundaries IE
 *   or_assemble(_dim)  P/prep_GLOBAL.f90:170-261   5-point coefficients (2-D and 3-D)
 *   or_sqprod          M/sevp.f90:696-713   operator apply
 *   or_sqprod_t        M/sevp.f90:714-742   transpose apply
 *   or_inprod          M/sevp.f90:743-757   interior dot product
 *   or_bicgstab_le     M/sevp.f90:443-552   restarted BiCGSTAB
 *   or_csi             M/sevp.f90:553-616   Chebyshev semi-iteration
 *   or_lanczos         M/sevp.f90:618-694   two-sided Lanczos eigen bounds
 *   or_figi            M/sevp.f90:838-904
 *   or_ratqr           M/sevp.f90:906-1006
 *   or_bir_sweeps      M/fs_GLOBAL.f90:1904-1966  overlapping-strip Schwarz sweeps
 *
 * Arithmetic follows the Fortran: REAL*4 coefficients and right-hand sides are
 * promoted exactly to double inside each expression, expressions are evaluated
 * left to right, and this file is compiled with -ffp-contract=off so no fused
 * multiply-add changes the rounding.
 *
 * Arrays are column-major and 1-based as in Fortran; the IX macro maps
 * (i, j) with leading dimension ld to a C offset.
 *
 * The second half holds the oracle of the new method that the GPU library
 * adds (it has no counterpart in the reference): a conjugate-gradient solve
 * preconditioned by block-Jacobi tiles, each tile solved exactly by the same
 * SEVP marching (PRE + REP on the tile, with an FP64 right-hand side and a
 * partially pivoted inverse).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define IX(ld, i, j) ((size_t)((j) - 1) * (size_t)(ld) + (size_t)((i) - 1))
#define IX3(ld1, ld2, i, j, k) \
  (((size_t)((k) - 1) * (size_t)(ld2) + (size_t)((j) - 1)) * (size_t)(ld1) + (size_t)((i) - 1))

/* Single-precision literals of the reference's stopping tests (1e-8, 1e-7). */
#define TOL_1EM8 ((double)1e-8f)
#define TOL_1EM7 ((double)1e-7f)

/* ------------------------------------------------------------------------ */
/* Marching core shared by REP1 / REPBIR_PERIOD / REPBIR / REP.               */
/* ------------------------------------------------------------------------ */

typedef struct {
  const float *ax, *ay, *bb, *cx, *cy; /* west, south, centre, east, north */
  int ldc;                             /* leading dimension of coefficients */
  const double *f;                     /* right-hand side, promoted */
  int ldf;
  const double *rinv, *rinv1; /* (m2, m2, *) */
  int m2;                     /* matrix order = marched columns */
  double *dum0, *dum1, *dum2;
  double *h;
  int ldh, hzero; /* H leading dimension, columns zeroed per block */
  double *x;
  int ldx;
  int periodic; /* refresh ghost columns 1 and i0 from i1 and 2 */
  int gi0;      /* ghost column index "I0" for the periodic refresh */
  const int *ie;
  int nblk;
} march_t;

static inline double c_at(const float *a, int ld, int i, int j) { return (double)a[IX(ld, i, j)]; }

/* X(I+1,J+2) = (F - AX*W - AY*S - BB*C - CX*E) / CY, M/sevp.f90:29-30 */
static inline double march_value(const march_t *m, const double *v, int ldv, int i, int j,
                                 double f) {
  double t = f - c_at(m->ax, m->ldc, i, j) * v[IX(ldv, i, j + 1)];
  t = t - c_at(m->ay, m->ldc, i, j) * v[IX(ldv, i + 1, j)];
  t = t - c_at(m->bb, m->ldc, i, j) * v[IX(ldv, i + 1, j + 1)];
  t = t - c_at(m->cx, m->ldc, i, j) * v[IX(ldv, i + 2, j + 1)];
  return t / c_at(m->cy, m->ldc, i, j);
}

/* residual of equation row j, M/sevp.f90:37-38 */
static inline double resid_value(const march_t *m, int i, int j) {
  const double *x = m->x;
  int ld = m->ldx;
  double t = m->f[IX(m->ldf, i, j)] - c_at(m->ax, m->ldc, i, j) * x[IX(ld, i, j + 1)];
  t = t - c_at(m->ay, m->ldc, i, j) * x[IX(ld, i + 1, j)];
  t = t - c_at(m->bb, m->ldc, i, j) * x[IX(ld, i + 1, j + 1)];
  t = t - c_at(m->cx, m->ldc, i, j) * x[IX(ld, i + 2, j + 1)];
  t = t - c_at(m->cy, m->ldc, i, j) * x[IX(ld, i + 1, j + 2)];
  return t;
}

static inline void ghost(double *v, int ld, int gi0, int j) {
  v[IX(ld, 1, j)] = v[IX(ld, gi0 - 1, j)];
  v[IX(ld, gi0, j)] = v[IX(ld, 2, j)];
}

/* DUM2(N) = sum_M DUM1(M) * R(M,N) */
static void vecmat(const double *dum1, const double *r, int m2, double *dum2) {
  for (int n = 1; n <= m2; ++n) {
    double s = 0.0;
    for (int k = 1; k <= m2; ++k) s = s + dum1[k - 1] * r[IX(m2, k, n)];
    dum2[n - 1] = s;
  }
}

static void march_solve(const march_t *m) {
  const int m2 = m->m2;
  const size_t msz = (size_t)m2 * m2;
  double *X = m->x, *H = m->h;
  const int ldx = m->ldx, ldh = m->ldh;
  /* forward sweep: particular solution, block-top corrections (sevp.f90:21-49) */
  int js = 1;
  for (int nb = 1; nb <= m->nblk; ++nb) {
    int jf = m->ie[nb - 1] - 2;
    for (int j = js; j <= jf; ++j) {
      if (m->periodic) ghost(X, ldx, m->gi0, j + 1);
      for (int i = 1; i <= m2; ++i)
        X[IX(ldx, i + 1, j + 2)] = march_value(m, X, ldx, i, j, m->f[IX(m->ldf, i, j)]);
    }
    if (m->periodic) ghost(X, ldx, m->gi0, jf + 2);
    if (nb != m->nblk) {
      int j = m->ie[nb - 1] - 1;
      for (int i = 1; i <= m2; ++i) m->dum1[i - 1] = resid_value(m, i, j);
      j = m->ie[nb - 1];
      vecmat(m->dum1, m->rinv1 + (size_t)(nb - 1) * msz, m2, m->dum2);
      for (int n = 1; n <= m2; ++n) {
        m->dum0[IX(m2, n, nb)] = X[IX(ldx, n + 1, j)];
        X[IX(ldx, n + 1, j)] = X[IX(ldx, n + 1, j)] - m->dum2[n - 1];
      }
      if (m->periodic) ghost(X, ldx, m->gi0, j);
    }
    js = m->ie[nb - 1];
  }
  /* backward sweep: guess-row corrections and homogeneous fields (sevp.f90:50-101) */
  for (int nbs = 1; nbs <= m->nblk; ++nbs) {
    int nb = m->nblk - nbs + 1;
    js = (nb != 1) ? m->ie[nb - 2] : 1;
    int jf = m->ie[nb - 1] - 2;
    if (nb != m->nblk) {
      int j = m->ie[nb - 1];
      for (int n = 1; n <= m2; ++n) X[IX(ldx, n + 1, j)] = m->dum0[IX(m2, n, nb)];
    }
    for (int j = js; j <= m->ie[nb - 1]; ++j)
      for (int i = 1; i <= m->hzero; ++i) H[IX(ldh, i, j)] = 0.0;
    int j = m->ie[nb - 1] - 1;
    if (m->periodic) ghost(X, ldx, m->gi0, j + 1);
    for (int i = 1; i <= m2; ++i) m->dum1[i - 1] = resid_value(m, i, j);
    vecmat(m->dum1, m->rinv + (size_t)(nb - 1) * msz, m2, m->dum2);
    for (int n = 1; n <= m2; ++n) {
      H[IX(ldh, n + 1, js + 1)] = m->dum2[n - 1];
      X[IX(ldx, n + 1, js + 1)] = X[IX(ldx, n + 1, js + 1)] + m->dum2[n - 1];
    }
    if (m->periodic) {
      ghost(H, ldh, m->gi0, js + 1);
      ghost(X, ldx, m->gi0, js + 1);
    }
    if (nb != 1) {
      for (int k = 1; k <= m2; ++k)
        m->dum1[k - 1] = H[IX(ldh, k + 1, js + 1)] * c_at(m->cy, m->ldc, k, js - 1);
      j = m->ie[nb - 2];
      vecmat(m->dum1, m->rinv1 + (size_t)(nb - 2) * msz, m2, m->dum2);
      for (int n = 1; n <= m2; ++n) H[IX(ldh, n + 1, j)] = m->dum2[n - 1];
      if (m->periodic) ghost(H, ldh, m->gi0, j);
    }
    for (j = js; j <= jf; ++j) {
      if (m->periodic) ghost(H, ldh, m->gi0, j + 1);
      for (int i = 1; i <= m2; ++i) {
        double hv = march_value(m, H, ldh, i, j, 0.0);
        H[IX(ldh, i + 1, j + 2)] = hv;
        X[IX(ldx, i + 1, j + 2)] = X[IX(ldx, i + 1, j + 2)] + hv;
      }
      if (m->periodic) ghost(X, ldx, m->gi0, j + 2);
    }
  }
  if (m->periodic)
    for (int j = 2; j <= m->ie[m->nblk - 1]; ++j) ghost(X, ldx, m->gi0, j);
}

/* The reference homogeneous march is (-AX*H_W - AY*H_S - BB*H_C - CX*H_E)/CY.
 * march_value with f = 0 computes (((0 - a) - b) - c) - d, which equals
 * (((-a) - b) - c) - d bit for bit (0 - a == -a for every non-NaN a, and the
 * sign of a zero result does not survive the following subtractions/division
 * differently). */

static double *promote(const float *f, size_t n) {
  double *d = (double *)malloc(n * sizeof(double));
  for (size_t k = 0; k < n; ++k) d[k] = (double)f[k];
  return d;
}

/* M/sevp.f90:11-107 */
void or_rep1(const float *AX, const float *AY, const float *BB, const float *CX, const float *CY,
             const double *RINV, const double *RINV1, double *DUM0, double *DUM1, double *DUM2,
             const float *F, double *H, double *X, const int *IE, int I0, int I2, int NBLK) {
  size_t nf = (size_t)I2 * (size_t)(IE[NBLK - 1]);
  double *fd = promote(F, nf);
  march_t m = {AX, AY, BB, CX, CY, I2, fd, I2, RINV, RINV1, I2, DUM0, DUM1, DUM2, H, I0, I0, X, I0,
               1, I0, IE, NBLK};
  march_solve(&m);
  free(fd);
}

/* M/sevp.f90:335-438 */
void or_rep(const float *AX, const float *AY, const float *BB, const float *CX, const float *CY,
            const double *RINV, const double *RINV1, double *DUM0, double *DUM1, double *DUM2,
            const float *F, double *H, double *X, const int *IE, int I0, int I2, int NBLK) {
  size_t nf = (size_t)I2 * (size_t)(IE[NBLK - 1]);
  double *fd = promote(F, nf);
  march_t m = {AX, AY, BB, CX, CY, I2, fd, I2, RINV, RINV1, I2, DUM0, DUM1, DUM2, H, I0, I0, X, I0,
               0, I0, IE, NBLK};
  march_solve(&m);
  free(fd);
}

/* M/sevp.f90:218-328 */
void or_repbir(const float *AX, const float *AY, const float *BB, const float *CX, const float *CY,
               const double *RINV, const double *RINV1, double *DUM0, double *DUM1, double *DUM2,
               const float *F, double *H, double *X, const int *IE, int I0, int I2, int M0, int M2,
               int NBLK) {
  size_t nf = (size_t)M2 * (size_t)(IE[NBLK - 1]);
  double *fd = promote(F, nf);
  march_t m = {AX, AY, BB, CX, CY, I2, fd, M2, RINV, RINV1, M2, DUM0, DUM1, DUM2, H, M0, M0, X, I0,
               0, I0, IE, NBLK};
  march_solve(&m);
  free(fd);
}

/* M/sevp.f90:109-217.  The reference refreshes H ghosts at columns I0-1 and I0
 * of an array whose leading dimension is M0, so it is only defined for
 * M0 == I0; other shapes return -1. */
int or_repbir_period(const float *AX, const float *AY, const float *BB, const float *CX,
                     const float *CY, const double *RINV, const double *RINV1, double *DUM0,
                     double *DUM1, double *DUM2, const float *F, double *H, double *X,
                     const int *IE, int I0, int I2, int M0, int M2, int NBLK) {
  if (M0 != I0) return -1;
  size_t nf = (size_t)M2 * (size_t)(IE[NBLK - 1]);
  double *fd = promote(F, nf);
  march_t m = {AX, AY, BB, CX, CY, I2, fd, M2, RINV, RINV1, M2, DUM0, DUM1, DUM2, H, M0, M0, X, I0,
               1, I0, IE, NBLK};
  march_solve(&m);
  free(fd);
  return 0;
}

/* FP64 right-hand-side variant used by the tile preconditioner oracle. */
static void rep_f64(const float *AX, const float *AY, const float *BB, const float *CX,
                    const float *CY, int ldc, const double *RINV, const double *RINV1,
                    double *DUM0, double *DUM1, double *DUM2, const double *F, int ldf, double *H,
                    double *X, const int *IE, int I0, int M2, int NBLK) {
  march_t m = {AX, AY, BB, CX, CY, ldc, F, ldf, RINV, RINV1, M2, DUM0, DUM1, DUM2, H, I0, I0, X, I0,
               0, I0, IE, NBLK};
  march_solve(&m);
}

/* ------------------------------------------------------------------------ */
/* MATINV: in-place Gauss-Jordan inverse without pivoting,                  */
/* P/prep_GLOBAL.f90:516-568.  Returns 0, or 1 when a pivot is exactly zero */
/* (the reference would divide by zero).                                     */
/* ------------------------------------------------------------------------ */
int or_matinv(double *B, int N) {
  double *b1 = (double *)calloc((size_t)N + 1, sizeof(double));
  double *b2 = (double *)calloc((size_t)N + 1, sizeof(double));
  int bad = 0;
  for (int i = 1; i <= N - 1; ++i) {
    if (B[IX(N, i, i)] == 0.0) bad = 1;
    b1[1] = 1. / B[IX(N, i, i)];
    B[IX(N, i, i)] = 1.0;
    for (int j = 1; j <= N; ++j) B[IX(N, i, j)] = B[IX(N, i, j)] * b1[1];
    for (int ia = i + 1; ia <= N; ++ia) b1[ia] = B[IX(N, ia, i)];
    for (int ia = i + 1; ia <= N; ++ia) B[IX(N, ia, i)] = 0.;
    for (int j = 1; j <= N; ++j) b2[j] = B[IX(N, i, j)];
    for (int ia = i + 1; ia <= N; ++ia)
      for (int j = 1; j <= N; ++j) B[IX(N, ia, j)] = B[IX(N, ia, j)] - b1[ia] * b2[j];
  }
  if (B[IX(N, N, N)] == 0.0) bad = 1;
  b1[1] = 1. / B[IX(N, N, N)];
  B[IX(N, N, N)] = 1.;
  for (int j = 1; j <= N; ++j) B[IX(N, N, j)] = B[IX(N, N, j)] * b1[1];
  for (int i = 2; i <= N; ++i) {
    for (int ib = 1; ib <= i; ++ib) b1[ib] = B[IX(N, ib, i)];
    for (int ib = 1; ib <= i - 1; ++ib) B[IX(N, ib, i)] = 0.;
    for (int j = 1; j <= N; ++j) b2[j] = B[IX(N, i, j)];
    for (int ib = 1; ib <= i - 1; ++ib)
      for (int j = 1; j <= N; ++j) B[IX(N, ib, j)] = B[IX(N, ib, j)] - b1[ib] * b2[j];
  }
  free(b1);
  free(b2);
  return bad;
}

/* Gauss-Jordan inverse with partial (row) pivoting; used by the tile
 * preconditioner of the new method only.  Returns 0, or 1 if singular. */
int or_matinv_pivot(double *B, int N) {
  /* B is column-major N x N.  Work on an augmented copy [B | I]. */
  double *a = (double *)malloc(sizeof(double) * (size_t)N * 2 * N);
  for (int r = 0; r < N; ++r)
    for (int c = 0; c < 2 * N; ++c)
      a[(size_t)r * 2 * N + c] = (c < N) ? B[(size_t)c * N + r] : (c - N == r ? 1.0 : 0.0);
  int bad = 0;
  for (int k = 0; k < N; ++k) {
    int piv = k;
    double best = fabs(a[(size_t)k * 2 * N + k]);
    for (int r = k + 1; r < N; ++r) {
      double v = fabs(a[(size_t)r * 2 * N + k]);
      if (v > best) best = v, piv = r;
    }
    if (best == 0.0) {
      bad = 1;
      break;
    }
    if (piv != k)
      for (int c = 0; c < 2 * N; ++c) {
        double t = a[(size_t)k * 2 * N + c];
        a[(size_t)k * 2 * N + c] = a[(size_t)piv * 2 * N + c];
        a[(size_t)piv * 2 * N + c] = t;
      }
    double inv = 1.0 / a[(size_t)k * 2 * N + k];
    for (int c = 0; c < 2 * N; ++c) a[(size_t)k * 2 * N + c] *= inv;
    for (int r = 0; r < N; ++r) {
      if (r == k) continue;
      double f = a[(size_t)r * 2 * N + k];
      if (f == 0.0) continue;
      for (int c = 0; c < 2 * N; ++c) a[(size_t)r * 2 * N + c] -= f * a[(size_t)k * 2 * N + c];
    }
  }
  if (!bad)
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c) B[(size_t)c * N + r] = a[(size_t)r * 2 * N + N + c];
  free(a);
  return bad;
}

/* ------------------------------------------------------------------------ */
/* Influence-matrix precompute, PRE1 (periodic) and PRE (strip).             */
/* ------------------------------------------------------------------------ */
typedef struct {
  const float *ax, *ay, *bb, *cx, *cy;
  int ldc;
  double *rinv, *rinv1;
  int m2;
  double *h;
  int ldh, hzero;
  int periodic, gi0;
  const int *ie;
  int nblk;
  int pivot; /* 0: reference MATINV, 1: partial pivoting */
} pre_t;

static inline double lhs4(const pre_t *p, int i, int j) {
  const double *H = p->h;
  int ld = p->ldh;
  double t = c_at(p->ax, p->ldc, i, j) * H[IX(ld, i, j + 1)];
  t = t + c_at(p->ay, p->ldc, i, j) * H[IX(ld, i + 1, j)];
  t = t + c_at(p->bb, p->ldc, i, j) * H[IX(ld, i + 1, j + 1)];
  t = t + c_at(p->cx, p->ldc, i, j) * H[IX(ld, i + 2, j + 1)];
  return t;
}

static int pre_core(const pre_t *p) {
  const int m2 = p->m2;
  const size_t msz = (size_t)m2 * m2;
  double *H = p->h;
  const int ldh = p->ldh;
  int jl = 1;
  int status = 0;
  for (int nb = 1; nb <= p->nblk; ++nb) {
    int jh = p->ie[nb - 1], jhp = jh + 1, jhm = jh - 2, jg = jl + 1;
    double *R = p->rinv + (size_t)(nb - 1) * msz;
    double *Rs = p->rinv + (size_t)(p->nblk - 1) * msz; /* scratch slot */
    for (int ng = 1; ng <= m2; ++ng) {
      int ig = ng + 1;
      for (int j = jl; j <= jhp; ++j)
        for (int i = 1; i <= p->hzero; ++i) H[IX(ldh, i, j)] = 0.;
      H[IX(ldh, ig, jg)] = 1.;
      if (p->periodic) ghost(H, ldh, p->gi0, jg);
      if (nb != 1) {
        const double *R1p = p->rinv1 + (size_t)(nb - 2) * msz;
        for (int n = 1; n <= m2; ++n)
          H[IX(ldh, n + 1, jl)] = R1p[IX(m2, ng, n)] * c_at(p->cy, p->ldc, ig - 1, jg - 2);
      }
      for (int j = jl; j <= jhm; ++j)
        for (int i = 1; i <= m2; ++i) {
          if (p->periodic) ghost(H, ldh, p->gi0, j + 1);
          H[IX(ldh, i + 1, j + 2)] = -(lhs4(p, i, j) / c_at(p->cy, p->ldc, i, j));
        }
      int j = jh - 1;
      for (int i = 1; i <= m2; ++i) {
        if (p->periodic) ghost(H, ldh, p->gi0, j + 1);
        R[IX(m2, ng, i)] = lhs4(p, i, j);
      }
      if (nb != p->nblk) {
        j = p->ie[nb - 1];
        for (int n = 1; n <= m2; ++n) Rs[IX(m2, ng, n)] = H[IX(ldh, n + 1, j)];
        if (p->periodic) {
          H[IX(ldh, 1, jg)] = 0.;
          H[IX(ldh, p->gi0, jg)] = 0.;
        }
      }
      H[IX(ldh, ig, jg)] = 0.;
    }
    status |= p->pivot ? or_matinv_pivot(R, m2) : or_matinv(R, m2);
    if (nb == p->nblk) return status;
    double *R1 = p->rinv1 + (size_t)(nb - 1) * msz;
    for (int i = 1; i <= m2; ++i)
      for (int j2 = 1; j2 <= m2; ++j2) {
        double s = 0.;
        for (int k = 1; k <= m2; ++k) s = s - R[IX(m2, i, k)] * Rs[IX(m2, k, j2)];
        R1[IX(m2, i, j2)] = s;
      }
    jl = jh;
  }
  return status;
}

/* P/prep_GLOBAL.f90:327-386 */
int or_pre1(const float *AX, const float *AY, const float *BB, const float *CX, const float *CY,
            double *RINV, double *RINV1, double *H, const int *IE, int I0, int I2, int NBLK) {
  pre_t p = {AX, AY, BB, CX, CY, I2, RINV, RINV1, I2, H, I0, I0, 1, I0, IE, NBLK, 0};
  return pre_core(&p);
}

/* P/prep_GLOBAL.f90:457-513 */
int or_pre(const float *AX, const float *AY, const float *BB, const float *CX, const float *CY,
           double *RINV, double *RINV1, double *H, const int *IE, int I2, int M0, int M2,
           int NBLK) {
  pre_t p = {AX, AY, BB, CX, CY, I2, RINV, RINV1, M2, H, M0, M0, 0, M0, IE, NBLK, 0};
  return pre_core(&p);
}

/* ------------------------------------------------------------------------ */
/* Block partition, P/prep_GLOBAL.f90:148-168.  Returns 0 if the partition  */
/* passes the reference's validity test, 1 otherwise (the reference stops). */
/* ------------------------------------------------------------------------ */
int or_block_partition(int J2, int NB0, int dimen, int *IE) {
  int J1 = J2 + 1;
  float q = (float)J2 / (float)NB0; /* REAL quotient */
  int nn = (int)lroundf(q);         /* ANINT: half away from zero */
  for (int n = 1; n <= NB0; ++n) {
    int v = 1 + nn * n;
    IE[n - 1] = v < J1 ? v : J1;
  }
  int ok = 0;
  if (NB0 >= 2) {
    int extra = (dimen == 2) ? 1 : 3;
    ok = IE[NB0 - 1] > IE[NB0 - 2] && J1 < IE[NB0 - 2] + nn + extra;
  }
  IE[NB0 - 1] = J1;
  return ok ? 0 : 1;
}

/* ------------------------------------------------------------------------ */
/* Coefficient assembly, P/prep_GLOBAL.f90:170-261 (dimen 2: :170-181).     */
/* Metric arrays are indexed 1..J0 (ODX, ODY, CSV, OCS, ODYV); ODZ 1..K1;   */
/* IU, IV are (I0, J0, K0) integer masks.  idealised != 0 applies the        */
/* constant test stencil and Neumann rows of :246-261.                        */
/* ------------------------------------------------------------------------ */
void or_assemble_dim(int I2, int J2, int K1, int dimen, const float *ODX, const float *ODY,
                     const float *CSV, const float *OCS, const float *ODYV, const float *ODZ,
                     const int *IU, const int *IV, int nbir, float gamma, int idealised, float *AL,
                     float *AR, float *AB, float *AT, float *AC) {
  int I0 = I2 + 2, J0 = J2 + 2;
  if (dimen == 2) {
    /* :170-181 */
    float dzx = ODX[0] * ODX[0] / ODZ[0];
    float dzy = ODY[0] * ODY[0] / ODZ[0];
    for (size_t k = 0; k < (size_t)I2 * J2; ++k) {
      AL[k] = dzx;
      AR[k] = dzx;
      AB[k] = dzy;
      AT[k] = dzy;
    }
    K1 = 0; /* no layer loop */
  }
  /* top layer all water */
  float tmp = 1.f / ODZ[0];
  for (int j = 1; j <= J2 && dimen == 3; ++j) {
    float dzx = ODX[j] * ODX[j] * tmp;
    float dzyb = CSV[j - 1] * OCS[j] * ODYV[j - 1] * ODY[j] * tmp;
    float dzyt = CSV[j] * OCS[j] * ODYV[j] * ODY[j] * tmp;
    for (int i = 1; i <= I2; ++i) {
      AL[IX(I2, i, j)] = dzx;
      AR[IX(I2, i, j)] = dzx;
      AB[IX(I2, i, j)] = dzyb;
      AT[IX(I2, i, j)] = dzyt;
    }
  }
  for (int k = 2; k <= K1; ++k) {
    tmp = 1.f / ODZ[k - 1];
    for (int j = 1; j <= J2; ++j) {
      float dzx = ODX[j] * ODX[j] * tmp;
      float dzyb = CSV[j - 1] * OCS[j] * ODYV[j - 1] * ODY[j] * tmp;
      float dzyt = CSV[j] * OCS[j] * ODYV[j] * ODY[j] * tmp;
      for (int i = 1; i <= I2; ++i) {
        AL[IX(I2, i, j)] = AL[IX(I2, i, j)] + dzx * (float)IU[IX3(I0, J0, i, j + 1, k)];
        AR[IX(I2, i, j)] = AR[IX(I2, i, j)] + dzx * (float)IU[IX3(I0, J0, i + 1, j + 1, k)];
        AB[IX(I2, i, j)] = AB[IX(I2, i, j)] + dzyb * (float)IV[IX3(I0, J0, i + 1, j, k)];
        AT[IX(I2, i, j)] = AT[IX(I2, i, j)] + dzyt * (float)IV[IX3(I0, J0, i + 1, j + 1, k)];
      }
    }
  }
  if (nbir == 1)
    for (int j = 1; j <= J2; ++j) {
      AL[IX(I2, 1, j)] = 0.f;
      AR[IX(I2, I2, j)] = 0.f;
    }
  for (int i = 1; i <= I2; ++i) {
    AB[IX(I2, i, 1)] = 0.f;
    AT[IX(I2, i, J2)] = 0.f;
  }
  if (nbir == 1 && J2 >= 2) AB[IX(I2, I2 / 2, 1)] = AB[IX(I2, I2 / 2, 2)];
  for (int j = 1; j <= J2; ++j)
    for (int i = 1; i <= I2; ++i)
      AC[IX(I2, i, j)] =
          -AL[IX(I2, i, j)] - AR[IX(I2, i, j)] - AB[IX(I2, i, j)] - AT[IX(I2, i, j)] - gamma;
  if (idealised) {
    for (size_t k = 0; k < (size_t)I2 * J2; ++k) {
      AL[k] = -0.25f;
      AB[k] = -0.25f;
      AC[k] = 1.0f;
      AR[k] = -0.25f;
      AT[k] = -0.25f;
    }
    for (int i = 1; i <= I2; ++i) {
      AC[IX(I2, i, J2)] = AC[IX(I2, i, J2)] + AT[IX(I2, i, J2)];
      AT[IX(I2, i, J2)] = 0.f;
      AC[IX(I2, i, 1)] = AC[IX(I2, i, 1)] + AB[IX(I2, i, 1)];
      AB[IX(I2, i, 1)] = 0.f;
    }
  }
}

/* The 3-D branch (the one PREP takes for the global model). */
void or_assemble(int I2, int J2, int K1, const float *ODX, const float *ODY, const float *CSV,
                 const float *OCS, const float *ODYV, const float *ODZ, const int *IU,
                 const int *IV, int nbir, float gamma, int idealised, float *AL, float *AR,
                 float *AB, float *AT, float *AC) {
  or_assemble_dim(I2, J2, K1, 3, ODX, ODY, CSV, OCS, ODYV, ODZ, IU, IV, nbir, gamma, idealised, AL,
                  AR, AB, AT, AC);
}

/* ------------------------------------------------------------------------ */
/* Krylov kernels on padded (i2+2, j2+2) FP64 arrays.                        */
/* ------------------------------------------------------------------------ */

/* M/sevp.f90:696-713 */
void or_sqprod(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
               const double *x, double *r, int i2, int j2) {
  int i0 = i2 + 2;
  for (int j = 1; j <= j2; ++j)
    for (int i = 1; i <= i2; ++i) {
      double t = (double)ab[IX(i2, i, j)] * x[IX(i0, i + 1, j)];
      t = t + (double)al[IX(i2, i, j)] * x[IX(i0, i, j + 1)];
      t = t + (double)ac[IX(i2, i, j)] * x[IX(i0, i + 1, j + 1)];
      t = t + (double)ar[IX(i2, i, j)] * x[IX(i0, i + 2, j + 1)];
      t = t + (double)at[IX(i2, i, j)] * x[IX(i0, i + 1, j + 2)];
      r[IX(i0, i + 1, j + 1)] = t;
    }
}

/* M/sevp.f90:714-742: coefficients of the neighbour cell, zero outside. */
void or_sqprod_t(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const double *x, double *r, int i2, int j2) {
  int i0 = i2 + 2;
#define PADC(a, i, j) (((i) >= 2 && (i) <= i2 + 1 && (j) >= 2 && (j) <= j2 + 1) ? (double)(a)[IX(i2, (i) - 1, (j) - 1)] : 0.0)
  for (int j = 1; j <= j2; ++j)
    for (int i = 1; i <= i2; ++i) {
      double t = PADC(at, i + 1, j) * x[IX(i0, i + 1, j)];
      t = t + PADC(ar, i, j + 1) * x[IX(i0, i, j + 1)];
      t = t + (double)ac[IX(i2, i, j)] * x[IX(i0, i + 1, j + 1)];
      t = t + PADC(al, i + 2, j + 1) * x[IX(i0, i + 2, j + 1)];
      t = t + PADC(ab, i + 1, j + 2) * x[IX(i0, i + 1, j + 2)];
      r[IX(i0, i + 1, j + 1)] = t;
    }
#undef PADC
}

/* M/sevp.f90:743-757 */
double or_inprod(const double *r, const double *p, int i2, int j2) {
  int i0 = i2 + 2;
  double tp = 0.0;
  for (int j = 2; j <= j2 + 1; ++j)
    for (int i = 2; i <= i2 + 1; ++i) tp = tp + r[IX(i0, i, j)] * p[IX(i0, i, j)];
  return tp;
}

/* M/sevp.f90:773-787 */
static void bdry(double *x, int i2, int j2, int periodic) {
  if (!periodic) return;
  int i0 = i2 + 2;
  for (int j = 2; j <= j2 + 1; ++j) {
    x[IX(i0, 1, j)] = x[IX(i0, i2 + 1, j)];
    x[IX(i0, i2 + 2, j)] = x[IX(i0, 2, j)];
  }
}

/* M/sevp.f90:443-552.  Returns the iteration count.  The identity
 * preconditioner of the reference (:759-772) is a copy. */
int or_bicgstab_le(const float *al, const float *ab, const float *ac, const float *ar,
                   const float *at, const float *b, double *x, int i2, int j2, int periodic,
                   double *final_res) {
  int i0 = i2 + 2, j0 = j2 + 2;
  size_t n = (size_t)i0 * j0;
  double *r = calloc(n, 8), *rh = calloc(n, 8), *p = calloc(n, 8), *v = calloc(n, 8);
  double *s = calloc(n, 8), *t = calloc(n, 8), *ph = calloc(n, 8), *sh = calloc(n, 8);
  int iter = 0;
  double tp = 1.0, rho, rhn, alpha, beta, w, res, tmp;
  bdry(x, i2, j2, periodic);
  while (sqrt(tp) > TOL_1EM8 && iter < 1000) {
    rho = 1.0;
    alpha = 1.0;
    w = 1.0;
    or_sqprod(al, ab, ac, ar, at, x, r, i2, j2);
    for (int j = 1; j <= j2; ++j)
      for (int i = 1; i <= i2; ++i)
        r[IX(i0, i + 1, j + 1)] = (double)b[IX(i2, i, j)] - r[IX(i0, i + 1, j + 1)];
    bdry(r, i2, j2, periodic);
    memcpy(rh, r, n * 8);
    tp = or_inprod(r, r, i2, j2);
    res = sqrt(tp);
    if (res < TOL_1EM8) break;
    while (sqrt(tp) / res > TOL_1EM8) {
      iter = iter + 1;
      rhn = or_inprod(r, rh, i2, j2);
      beta = (rhn / rho) * (alpha / w);
      for (size_t k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - w * v[k]);
      memcpy(ph, p, n * 8);
      bdry(ph, i2, j2, periodic);
      or_sqprod(al, ab, ac, ar, at, ph, v, i2, j2);
      bdry(v, i2, j2, periodic);
      tmp = or_inprod(rh, v, i2, j2);
      alpha = rhn / tmp;
      for (size_t k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
      memcpy(sh, s, n * 8);
      bdry(sh, i2, j2, periodic);
      or_sqprod(al, ab, ac, ar, at, sh, t, i2, j2);
      bdry(t, i2, j2, periodic);
      tmp = or_inprod(t, t, i2, j2);
      w = or_inprod(t, s, i2, j2);
      w = w / tmp;
      for (size_t k = 0; k < n; ++k) x[k] = x[k] + alpha * ph[k] + w * sh[k];
      for (size_t k = 0; k < n; ++k) r[k] = s[k] - w * t[k];
      tp = or_inprod(r, r, i2, j2);
      rho = rhn;
      if (iter % 100 == 0) break;
    }
  }
  bdry(x, i2, j2, periodic);
  if (final_res) *final_res = sqrt(tp);
  free(r), free(rh), free(p), free(v), free(s), free(t), free(ph), free(sh);
  return iter;
}

/* M/sevp.f90:553-616.  Returns the iteration count. */
int or_csi(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
           double mineig, double maxeig, const float *b, double *x, int i2, int j2, int periodic,
           double *final_res) {
  int i0 = i2 + 2, j0 = j2 + 2;
  size_t n = (size_t)i0 * j0;
  double *r = calloc(n, 8), *s = calloc(n, 8), *q = calloc(n, 8), *work1 = calloc(n, 8);
  int iter = 0;
  double tp = 1.0;
  double alpha = 2.0 / (maxeig - mineig);
  double beta = (maxeig + mineig) / (maxeig - mineig);
  double csy = beta / alpha;
  double omega = 2.0 / csy;
  bdry(x, i2, j2, periodic);
  or_sqprod(al, ab, ac, ar, at, x, s, i2, j2);
  bdry(s, i2, j2, periodic);
  for (int j = 1; j <= j2; ++j)
    for (int i = 1; i <= i2; ++i)
      r[IX(i0, i + 1, j + 1)] = (double)b[IX(i2, i, j)] - s[IX(i0, i + 1, j + 1)];
  memcpy(work1, r, n * 8);
  bdry(work1, i2, j2, periodic);
  for (size_t k = 0; k < n; ++k) q[k] = (1.0 / csy) * work1[k];
  for (size_t k = 0; k < n; ++k) x[k] = x[k] + q[k];
  or_sqprod(al, ab, ac, ar, at, x, s, i2, j2);
  bdry(s, i2, j2, periodic);
  for (int j = 1; j <= j2; ++j)
    for (int i = 1; i <= i2; ++i)
      r[IX(i0, i + 1, j + 1)] = (double)b[IX(i2, i, j)] - s[IX(i0, i + 1, j + 1)];
  while (sqrt(tp) > TOL_1EM7 && iter < 1000) {
    omega = 1.0 / (csy - omega / (4.0 * alpha * alpha));
    memcpy(work1, r, n * 8);
    bdry(work1, i2, j2, periodic);
    for (size_t k = 0; k < n; ++k) q[k] = omega * work1[k] + (csy * omega - 1.0) * q[k];
    for (size_t k = 0; k < n; ++k) x[k] = x[k] + q[k];
    or_sqprod(al, ab, ac, ar, at, x, s, i2, j2);
    for (int j = 1; j <= j2; ++j)
      for (int i = 1; i <= i2; ++i)
        r[IX(i0, i + 1, j + 1)] = (double)b[IX(i2, i, j)] - s[IX(i0, i + 1, j + 1)];
    bdry(r, i2, j2, periodic);
    tp = or_inprod(r, r, i2, j2);
    iter = iter + 1;
  }
  bdry(x, i2, j2, periodic);
  if (final_res) *final_res = sqrt(tp);
  free(r), free(s), free(q), free(work1);
  return iter;
}

/* M/sevp.f90:838-904 */
int or_figi(int n, const double *t, double *d, double *e, double *e2) {
  for (int i = 1; i <= n; ++i) {
    if (1 < i) {
      e2[i - 1] = t[IX(n, i, 1)] * t[IX(n, i - 1, 3)];
      if (e2[i - 1] < 0.0) return n + i;
      if (e2[i - 1] == 0.0) {
        if (t[IX(n, i, 1)] != 0.0 || t[IX(n, i - 1, 3)] != 0.0) return -3 * n - i;
        e[i - 1] = 0.0;
      } else {
        e[i - 1] = sqrt(e2[i - 1]);
      }
    }
    d[i - 1] = t[IX(n, i, 2)];
  }
  return 0;
}

/* M/sevp.f90:906-1006 */
int or_ratqr(int n, double eps1, const double *d, const double *e, double *mineig) {
  double *e2 = calloc((size_t)n + 1, 8), *bd = calloc((size_t)n + 1, 8), *w = calloc((size_t)n + 1, 8);
  (void)e2;
  int ierr = 0, i;
  double f, ep, delta = 0.0, err, p, q, qp = 0.0, r, s, tot;
  for (i = 1; i <= n; ++i) w[i] = d[i - 1];
  err = 0.0;
  s = 0.0;
  tot = w[1];
  q = 0.0;
  for (i = 1; i <= n; ++i) {
    p = q;
    bd[i] = e[i - 1] * e[i - 1];
    q = 0.0;
    if (i != n) q = fabs(e[i]);
    double cand = w[i] - p - q;
    tot = cand < tot ? cand : tot;
  }
  bd[1] = 0.0;
  if (tot < 0.0)
    tot = 0.0;
  else
    for (i = 1; i <= n; ++i) w[i] = w[i] - tot;
  /* The reference loops without bound; a NaN/Inf input never meets its
   * exits, so the restatement stops after 100000 sweeps with ierr = 2. */
  for (int sweep = 0;; ++sweep) {
    if (sweep >= 100000) {
      free(e2), free(bd), free(w);
      return 2;
    }
    tot = tot + s;
    delta = w[n] - s;
    i = n;
    if (delta <= eps1) break;
    f = bd[n] / delta;
    qp = delta + f;
    p = 1.0;
    for (int ii = 1; ii <= n - 1; ++ii) {
      i = n - ii;
      q = w[i] - s - f;
      r = q / qp;
      p = p * r + 1.0;
      ep = f * r;
      w[i + 1] = qp + ep;
      delta = q - ep;
      if (delta <= eps1) break;
      f = bd[i] / q;
      qp = delta + f;
      bd[i + 1] = qp * ep;
    }
    if (delta <= eps1) break;
    w[1] = qp;
    s = qp / p;
    if (tot + s <= tot) {
      ierr = 1;
      free(e2), free(bd), free(w);
      return ierr;
    }
  }
  w[1] = tot;
  err = err + fabs(delta);
  bd[1] = err;
  *mineig = w[1];
  free(e2), free(bd), free(w);
  return ierr;
}

/* M/sevp.f90:618-694.  The reference writes sigma(m+1)/beta(m+1) one past
 * its arrays and reads the uninitialised ghost points of its locals s and q;
 * this restatement sizes those arrays m+1 and zero-initialises the locals. */
int or_lanczos(const float *al, const float *ab, const float *ac, const float *ar,
               const float *at, int i2, int j2, double *mineig, double *maxeig, double *alpha_out,
               double *sigma_out) {
  enum { M = 10 };
  int i0 = i2 + 2, j0 = j2 + 2;
  size_t n = (size_t)i0 * j0;
  double *v = calloc(n, 8), *w = calloc(n, 8), *vp = calloc(n, 8), *wp = calloc(n, 8);
  double *s = calloc(n, 8), *q = calloc(n, 8), *work = calloc(n, 8);
  double alpha[M + 2] = {0}, beta[M + 2] = {0}, sigma[M + 2] = {0};
  double mcsa[M] = {0}, mcsb[M] = {0}, mcsb2[M] = {0}, t[M * 3] = {0};
  double tp;
  for (size_t k = 0; k < n; ++k) v[k] = 1.;
  tp = or_inprod(v, v, i2, j2);
  for (size_t k = 0; k < n; ++k) v[k] = 1 / sqrt(tp) * v[k];
  memcpy(w, v, n * 8);
  int iter = 0;
  while (iter < M) {
    iter = iter + 1;
    or_sqprod(al, ab, ac, ar, at, v, s, i2, j2);
    tp = or_inprod(s, w, i2, j2);
    alpha[iter] = tp;
    for (size_t k = 0; k < n; ++k) work[k] = beta[iter] * vp[k];
    memcpy(vp, v, n * 8);
    for (size_t k = 0; k < n; ++k) v[k] = s[k] - alpha[iter] * v[k] - work[k];
    or_sqprod_t(al, ab, ac, ar, at, w, q, i2, j2);
    for (size_t k = 0; k < n; ++k) work[k] = sigma[iter] * wp[k];
    memcpy(wp, w, n * 8);
    for (size_t k = 0; k < n; ++k) w[k] = q[k] - alpha[iter] * w[k] - work[k];
    tp = or_inprod(v, w, i2, j2);
    sigma[iter + 1] = sqrt(fabs(tp));
    beta[iter + 1] = copysign(sigma[iter + 1], tp);
    for (size_t k = 0; k < n; ++k) v[k] = v[k] / sigma[iter + 1];
    for (size_t k = 0; k < n; ++k) w[k] = w[k] / beta[iter + 1];
  }
  or_sqprod(al, ab, ac, ar, at, v, s, i2, j2);
  tp = or_inprod(s, w, i2, j2);
  alpha[M] = tp;
  /* t(2:m,1)=sigma(2:m); t(1:m,2)=alpha(1:m); t(1:m-1,3)=sigma(2:m) */
  for (int k = 2; k <= M; ++k) t[IX(M, k, 1)] = sigma[k];
  for (int k = 1; k <= M; ++k) t[IX(M, k, 2)] = alpha[k];
  for (int k = 1; k <= M - 1; ++k) t[IX(M, k, 3)] = sigma[k + 1];
  int ierr = or_figi(M, t, mcsa, mcsb, mcsb2);
  double mx = mcsa[0] + mcsb[0];
  for (int k = 2; k <= M; ++k) {
    double c = mcsa[k - 1] + mcsb[k - 1] + mcsb[k - 2];
    mx = c > mx ? c : mx;
  }
  *maxeig = mx;
  int ierr2 = or_ratqr(M, 1.0e-6, mcsa, mcsb, mineig);
  if (alpha_out)
    for (int k = 0; k < M; ++k) alpha_out[k] = alpha[k + 1];
  if (sigma_out)
    for (int k = 0; k < M + 1; ++k) sigma_out[k] = sigma[k + 1];
  free(v), free(w), free(vp), free(wp), free(s), free(q), free(work);
  return ierr != 0 ? ierr : ierr2;
}

/* M/fs_GLOBAL.f90:1904-1966: NITER sweeps of overlapping BIR strips.
 * The reference sets the wrapped strip's side boundaries XX(1,J) and
 * XX(IBIR+2,J) for J = 1..J2 only (:1925-1926), so the top interior row
 * J2+1 keeps a stale (zero) boundary; fix_wrap != 0 also copies rows J2+1
 * and J2+2 (an opt-in correction, not reference behaviour).
 * S (I2,J2) FP32; AL..AT (I2,J2); X (I0,J0); RINV (IBIR,IBIR,NB0,NBIR),
 * RINV1 (IBIR,IBIR,NB0-1,NBIR); workspaces SRC/CL..CT (IBIR,J2), XX and H
 * (IBIR+2,J0), DUM0 (IBIR,NB0-1), DUM1/DUM2 (IBIR).  XX is caller-owned so
 * that its interior persists across calls as the reference's module array. */
void or_bir_sweeps(const float *AL, const float *AB, const float *AC, const float *AR,
                   const float *AT, const float *S, const double *RINV, const double *RINV1,
                   double *X, double *XX, double *H, float *SRC, float *CL, float *CB, float *CC,
                   float *CR, float *CT, double *DUM0, double *DUM1, double *DUM2, const int *IE,
                   int I2, int J2, int NB0, int NBIR, int niter, int periodic, int fix_wrap) {
  int I0 = I2 + 2, I1 = I2 + 1, J1 = J2 + 1;
  int IBIR = 2 * I2 / NBIR, INC = IBIR / 2;
  size_t rstride = (size_t)IBIR * IBIR * NB0, r1stride = (size_t)IBIR * IBIR * (NB0 > 1 ? NB0 - 1 : 1);
  for (int it = 1; it <= niter; ++it) {
    for (int n = 1; n <= NBIR; ++n) {
      int il = (n - 1) * INC + 1;
      const double *R = RINV + (size_t)(n - 1) * rstride;
      const double *R1 = RINV1 + (size_t)(n - 1) * r1stride;
      if (n != NBIR) {
        for (int j = 1; j <= J2; ++j)
          for (int i = 1; i <= IBIR; ++i) SRC[IX(IBIR, i, j)] = S[IX(I2, il + i - 1, j)];
        or_repbir(AL + (il - 1), AB + (il - 1), AC + (il - 1), AR + (il - 1), AT + (il - 1), R,
                  R1, DUM0, DUM1, DUM2, SRC, H, X + (il - 1), IE, I0, I2, IBIR + 2, IBIR, NB0);
      } else {
        int ir = il + INC, ir2 = il + IBIR - 1;
        if (fix_wrap)
          for (int j = J2 + 1; j <= J2 + 2; ++j) {
            XX[IX(IBIR + 2, 1, j)] = X[IX(I0, il, j)];
            XX[IX(IBIR + 2, IBIR + 2, j)] = X[IX(I0, INC + 2, j)];
          }
        for (int j = 1; j <= J2; ++j) {
          XX[IX(IBIR + 2, 1, j)] = X[IX(I0, il, j)];
          XX[IX(IBIR + 2, IBIR + 2, j)] = X[IX(I0, INC + 2, j)];
          for (int i = il; i <= ir - 1; ++i) {
            SRC[IX(IBIR, i - il + 1, j)] = S[IX(I2, i, j)];
            CL[IX(IBIR, i - il + 1, j)] = AL[IX(I2, i, j)];
            CR[IX(IBIR, i - il + 1, j)] = AR[IX(I2, i, j)];
            CB[IX(IBIR, i - il + 1, j)] = AB[IX(I2, i, j)];
            CT[IX(IBIR, i - il + 1, j)] = AT[IX(I2, i, j)];
            CC[IX(IBIR, i - il + 1, j)] = AC[IX(I2, i, j)];
          }
          for (int i = ir; i <= ir2; ++i) {
            SRC[IX(IBIR, i - il + 1, j)] = S[IX(I2, i - ir + 1, j)];
            CL[IX(IBIR, i - il + 1, j)] = AL[IX(I2, i - ir + 1, j)];
            CR[IX(IBIR, i - il + 1, j)] = AR[IX(I2, i - ir + 1, j)];
            CB[IX(IBIR, i - il + 1, j)] = AB[IX(I2, i - ir + 1, j)];
            CT[IX(IBIR, i - il + 1, j)] = AT[IX(I2, i - ir + 1, j)];
            CC[IX(IBIR, i - il + 1, j)] = AC[IX(I2, i - ir + 1, j)];
          }
        }
        or_repbir(CL, CB, CC, CR, CT, R, R1, DUM0, DUM1, DUM2, SRC, H, XX, IE, IBIR + 2, IBIR,
                  IBIR + 2, IBIR, NB0);
        for (int j = 2; j <= J1; ++j) {
          for (int i = il; i <= ir - 1; ++i) X[IX(I0, i + 1, j)] = XX[IX(IBIR + 2, i - il + 2, j)];
          for (int i = ir; i <= ir2; ++i) X[IX(I0, i - ir + 2, j)] = XX[IX(IBIR + 2, i - il + 2, j)];
        }
        if (periodic)
          for (int j = 2; j <= J1; ++j) {
            X[IX(I0, 1, j)] = X[IX(I0, I1, j)];
            X[IX(I0, I0, j)] = X[IX(I0, 2, j)];
          }
      }
    }
  }
}

/* Strip influence precompute for all BIR strips (P/prep_GLOBAL.f90:286-317),
 * including the wrapped last strip.  CL..CT are (IBIR, J2) workspaces. */
int or_pre_strips(const float *AL, const float *AB, const float *AC, const float *AR,
                  const float *AT, double *RINV, double *RINV1, double *H, const int *IE, int I2,
                  int J2, int NB0, int NBIR, float *CL, float *CB, float *CC, float *CR,
                  float *CT) {
  int IBIR = 2 * I2 / NBIR, INC = IBIR / 2;
  if (IBIR * NBIR != 2 * I2) return -1;
  size_t rstride = (size_t)IBIR * IBIR * NB0, r1stride = (size_t)IBIR * IBIR * (NB0 > 1 ? NB0 - 1 : 1);
  int st = 0;
  for (int n = 1; n <= NBIR; ++n) {
    int il = (n - 1) * INC + 1;
    double *R = RINV + (size_t)(n - 1) * rstride;
    double *R1 = RINV1 + (size_t)(n - 1) * r1stride;
    if (NBIR == 1 || n != NBIR) {
      st |= or_pre(AL + (il - 1), AB + (il - 1), AC + (il - 1), AR + (il - 1), AT + (il - 1), R,
                   R1, H, IE, I2, IBIR + 2, IBIR, NB0);
    } else {
      int ir = il + INC - 1, ir2 = il + IBIR - 1;
      for (int j = 1; j <= J2; ++j) {
        for (int i = il; i <= ir; ++i) {
          CL[IX(IBIR, i - il + 1, j)] = AL[IX(I2, i, j)];
          CR[IX(IBIR, i - il + 1, j)] = AR[IX(I2, i, j)];
          CB[IX(IBIR, i - il + 1, j)] = AB[IX(I2, i, j)];
          CT[IX(IBIR, i - il + 1, j)] = AT[IX(I2, i, j)];
          CC[IX(IBIR, i - il + 1, j)] = AC[IX(I2, i, j)];
        }
        for (int i = ir + 1; i <= ir2; ++i) {
          CL[IX(IBIR, i - il + 1, j)] = AL[IX(I2, i - ir, j)];
          CR[IX(IBIR, i - il + 1, j)] = AR[IX(I2, i - ir, j)];
          CB[IX(IBIR, i - il + 1, j)] = AB[IX(I2, i - ir, j)];
          CT[IX(IBIR, i - il + 1, j)] = AT[IX(I2, i - ir, j)];
          CC[IX(IBIR, i - il + 1, j)] = AC[IX(I2, i - ir, j)];
        }
      }
      st |= or_pre(CL, CB, CC, CR, CT, R, R1, H, IE, IBIR, IBIR + 2, IBIR, NB0);
    }
  }
  return st;
}

/* ======================================================================== */
/* New method (no reference counterpart): block-Jacobi tile SEVP            */
/* preconditioned CG on unpadded row-major-in-j (i fastest) FP64 vectors.   */
/* ======================================================================== */

/* Tile layout: tiles of at most tm columns x th rows, clipped at the domain
 * edge.  A tile of hh rows is split into nb sub-blocks (given per tile) with
 * boundaries k_t = (t * hh) / nb, t = 0..nb. */
typedef struct {
  int nx, ny, tm, th, tx, ty;
  const int *tile_nb; /* sub-blocks per tile (ty * tx entries, tile rows first) */
} tiles_t;

static void tile_geom(const tiles_t *T, int a, int b, int *i0, int *j0, int *mw, int *hh, int *nb) {
  *i0 = a * T->tm;
  *j0 = b * T->th;
  *mw = T->nx - *i0 < T->tm ? T->nx - *i0 : T->tm;
  *hh = T->ny - *j0 < T->th ? T->ny - *j0 : T->th;
  int v = T->tile_nb[b * T->tx + a];
  if (v < 1) v = 1;
  if (v > *hh) v = *hh;
  *nb = v;
}

/* Influence data of one tile (RINV, RINV1 in the reference's (m,m,nb)
 * column-major layout) plus its block boundaries IE (1-based padded rows). */
typedef struct {
  double *rinv, *rinv1;
  int *ie;
  int mw, hh, nb, i0, j0;
} tile_data_t;

typedef struct {
  tiles_t T;
  tile_data_t *td;
  int ntiles;
} tile_pc_t;

static void tile_coeffs(const float *c, int nx, int i0, int j0, int mw, int hh, float *out) {
  for (int k = 0; k < hh; ++k)
    for (int i = 0; i < mw; ++i) out[(size_t)k * mw + i] = c[(size_t)(j0 + k) * nx + i0 + i];
}

/* Builds the tile preconditioner.  Coefficients are (nx, ny) column-major:
 * element (i, j) (0-based) at j * nx + i.  Returns NULL on a singular tile. */
tile_pc_t *or_tile_setup(const float *al, const float *ab, const float *ac, const float *ar,
                         const float *at, int nx, int ny, int tm, int th, const int *tile_nb,
                         int *status) {
  tile_pc_t *pc = (tile_pc_t *)calloc(1, sizeof(tile_pc_t));
  pc->T.nx = nx, pc->T.ny = ny, pc->T.tm = tm, pc->T.th = th;
  pc->T.tx = (nx + tm - 1) / tm;
  pc->T.ty = (ny + th - 1) / th;
  int *sr = (int *)malloc(sizeof(int) * pc->T.ty * pc->T.tx);
  memcpy(sr, tile_nb, sizeof(int) * pc->T.ty * pc->T.tx);
  pc->T.tile_nb = sr;
  pc->ntiles = pc->T.tx * pc->T.ty;
  pc->td = (tile_data_t *)calloc((size_t)pc->ntiles, sizeof(tile_data_t));
  int st = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : st)
  for (int t = 0; t < pc->ntiles; ++t) {
    int a = t % pc->T.tx, b = t / pc->T.tx;
    tile_data_t *d = &pc->td[t];
    tile_geom(&pc->T, a, b, &d->i0, &d->j0, &d->mw, &d->hh, &d->nb);
    int mw = d->mw, hh = d->hh, nb = d->nb;
    d->ie = (int *)malloc(sizeof(int) * nb);
    for (int q = 1; q <= nb; ++q) d->ie[q - 1] = (q * hh) / nb + 1;
    size_t msz = (size_t)mw * mw;
    d->rinv = (double *)calloc(msz * nb, 8);
    d->rinv1 = (double *)calloc(msz * (nb > 1 ? nb - 1 : 1), 8);
    float *cw = malloc(sizeof(float) * mw * hh * 5);
    float *cax = cw, *cay = cw + mw * hh, *cbb = cw + 2 * mw * hh, *ccx = cw + 3 * mw * hh,
          *ccy = cw + 4 * mw * hh;
    tile_coeffs(al, nx, d->i0, d->j0, mw, hh, cax);
    tile_coeffs(ab, nx, d->i0, d->j0, mw, hh, cay);
    tile_coeffs(ac, nx, d->i0, d->j0, mw, hh, cbb);
    tile_coeffs(ar, nx, d->i0, d->j0, mw, hh, ccx);
    tile_coeffs(at, nx, d->i0, d->j0, mw, hh, ccy);
    double *H = calloc((size_t)(mw + 2) * (hh + 2), 8);
    pre_t p = {cax, cay, cbb, ccx, ccy, mw, d->rinv, d->rinv1, mw, H, mw + 2, mw + 2, 0, mw + 2,
               d->ie, nb, 1};
    st |= pre_core(&p);
    free(H);
    free(cw);
  }
  if (status) *status = st;
  return pc;
}

void or_tile_free(tile_pc_t *pc) {
  if (!pc) return;
  for (int t = 0; t < pc->ntiles; ++t) {
    free(pc->td[t].rinv), free(pc->td[t].rinv1), free(pc->td[t].ie);
  }
  free((void *)pc->T.tile_nb);
  free(pc->td);
  free(pc);
}

int or_tile_count(const tile_pc_t *pc) { return pc->ntiles; }

/* Copies tile t's influence data out: rinv (mw*mw*nb), rinv1 (mw*mw*(nb-1)). */
void or_tile_get(const tile_pc_t *pc, int t, int *geom, double *rinv, double *rinv1) {
  const tile_data_t *d = &pc->td[t];
  geom[0] = d->i0, geom[1] = d->j0, geom[2] = d->mw, geom[3] = d->hh, geom[4] = d->nb;
  size_t msz = (size_t)d->mw * d->mw;
  if (rinv) memcpy(rinv, d->rinv, msz * d->nb * 8);
  if (rinv1 && d->nb > 1) memcpy(rinv1, d->rinv1, msz * (d->nb - 1) * 8);
}

/* z = M^{-1} r: each tile solved with zero Dirichlet data on its boundary. */
void or_tile_apply(const tile_pc_t *pc, const float *al, const float *ab, const float *ac,
                   const float *ar, const float *at, const double *r, double *z) {
  int nx = pc->T.nx;
#pragma omp parallel for schedule(dynamic)
  for (int t = 0; t < pc->ntiles; ++t) {
    const tile_data_t *d = &pc->td[t];
    int mw = d->mw, hh = d->hh, nb = d->nb;
    float *cw = malloc(sizeof(float) * mw * hh * 5);
    float *cax = cw, *cay = cw + mw * hh, *cbb = cw + 2 * mw * hh, *ccx = cw + 3 * mw * hh,
          *ccy = cw + 4 * mw * hh;
    tile_coeffs(al, nx, d->i0, d->j0, mw, hh, cax);
    tile_coeffs(ab, nx, d->i0, d->j0, mw, hh, cay);
    tile_coeffs(ac, nx, d->i0, d->j0, mw, hh, cbb);
    tile_coeffs(ar, nx, d->i0, d->j0, mw, hh, ccx);
    tile_coeffs(at, nx, d->i0, d->j0, mw, hh, ccy);
    double *F = malloc(sizeof(double) * mw * hh);
    for (int k = 0; k < hh; ++k)
      for (int i = 0; i < mw; ++i) F[(size_t)k * mw + i] = r[(size_t)(d->j0 + k) * nx + d->i0 + i];
    int I0 = mw + 2;
    double *X = calloc((size_t)I0 * (hh + 2), 8);
    double *H = calloc((size_t)I0 * (hh + 2), 8);
    double *D0 = calloc((size_t)mw * (nb > 1 ? nb - 1 : 1), 8);
    double *D1 = calloc((size_t)mw, 8), *D2 = calloc((size_t)mw, 8);
    rep_f64(cax, cay, cbb, ccx, ccy, mw, d->rinv, d->rinv1, D0, D1, D2, F, mw, H, X, d->ie, I0, mw,
            nb);
    for (int k = 0; k < hh; ++k)
      for (int i = 0; i < mw; ++i)
        z[(size_t)(d->j0 + k) * nx + d->i0 + i] = X[IX(I0, i + 2, k + 2)];
    free(cw), free(F), free(X), free(H), free(D0), free(D1), free(D2);
  }
}

/* y = A x on unpadded vectors; zero outside the domain except periodic x. */
void or_apply(const float *al, const float *ab, const float *ac, const float *ar,
              const float *at, int nx, int ny, int periodic, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      size_t c = (size_t)j * nx + i;
      double xs = j > 0 ? x[c - nx] : 0.0;
      double xn = j < ny - 1 ? x[c + nx] : 0.0;
      double xw = i > 0 ? x[c - 1] : (periodic ? x[c + nx - 1] : 0.0);
      double xe = i < nx - 1 ? x[c + 1] : (periodic ? x[c - nx + 1] : 0.0);
      double t = (double)ab[c] * xs;
      t = t + (double)al[c] * xw;
      t = t + (double)ac[c] * x[c];
      t = t + (double)ar[c] * xe;
      t = t + (double)at[c] * xn;
      y[c] = t;
    }
}

/* Deterministic dot product: per-row partial sums, then rows in order. */
double or_dot(const double *a, const double *b, int nx, int ny) {
  double *rows = malloc(sizeof(double) * ny);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; ++j) {
    double s = 0.0;
    for (int i = 0; i < nx; ++i) s += a[(size_t)j * nx + i] * b[(size_t)j * nx + i];
    rows[j] = s;
  }
  double s = 0.0;
  for (int j = 0; j < ny; ++j) s += rows[j];
  free(rows);
  return s;
}

/* Preconditioned CG to ||b - A x|| <= tol ||b|| (true FP64 residual, checked
 * on exit of the recursive loop; restarts from the true residual if the
 * recursive residual drifted).  x holds the initial guess on entry.
 * Returns iterations; *relres gets the final true relative residual. */
int or_pcg(const tile_pc_t *pc, const float *al, const float *ab, const float *ac, const float *ar,
           const float *at, int periodic, const double *b, double *x, double tol, int maxit,
           double *relres) {
  int nx = pc->T.nx, ny = pc->T.ny;
  size_t n = (size_t)nx * ny;
  double *r = malloc(n * 8), *z = malloc(n * 8), *p = malloc(n * 8), *q = malloc(n * 8);
  double bn = sqrt(or_dot(b, b, nx, ny));
  if (bn == 0.0) bn = 1.0;
  int it = 0;
  double rel = 0.0;
  for (int restart = 0; restart < 8; ++restart) {
    or_apply(al, ab, ac, ar, at, nx, ny, periodic, x, q);
    for (size_t k = 0; k < n; ++k) r[k] = b[k] - q[k];
    rel = sqrt(or_dot(r, r, nx, ny)) / bn;
    if (rel <= tol || it >= maxit || !isfinite(rel)) break;
    or_tile_apply(pc, al, ab, ac, ar, at, r, z);
    memcpy(p, z, n * 8);
    double rz = or_dot(r, z, nx, ny);
    while (it < maxit) {
      or_apply(al, ab, ac, ar, at, nx, ny, periodic, p, q);
      double pq = or_dot(p, q, nx, ny);
      if (!isfinite(pq) || pq == 0.0) {
        it = maxit;
        break;
      }
      double alpha = rz / pq;
      for (size_t k = 0; k < n; ++k) {
        x[k] += alpha * p[k];
        r[k] -= alpha * q[k];
      }
      ++it;
      double rr = or_dot(r, r, nx, ny);
      if (!isfinite(rr)) {
        it = maxit;
        break;
      }
      if (sqrt(rr) / bn <= tol) break;
      or_tile_apply(pc, al, ab, ac, ar, at, r, z);
      double rz2 = or_dot(r, z, nx, ny);
      double beta = rz2 / rz;
      rz = rz2;
      for (size_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
    }
  }
  if (relres) *relres = rel;
  free(r), free(z), free(p), free(q);
  return it;
}

/* Preconditioned Chebyshev iteration: the new method's second outer
 * iteration around the tile SEVP preconditioner (the reference's P-CSI,
 * M/sevp.f90:553-616, is the unpreconditioned form with bounds from
 * lanczos/ratqr).  Bounds lmin, lmax of the spectrum of M^-1 A:
 *   theta = (lmax + lmin) / 2, delta = (lmax - lmin) / 2, sigma = theta / delta;
 *   r = b - A x; d = M^-1 r / theta; rho = 1 / sigma;
 *   repeat: x += d; r -= A d; rho' = 1 / (2 sigma - rho);
 *           d = rho' rho d + (2 rho' / delta) M^-1 r; rho = rho'
 * until ||r|| <= tol ||b|| on the recursive residual; the true residual is
 * then recomputed and the iteration restarts from it if it is not yet
 * below the tolerance.  Returns the x updates made; *relres gets the final
 * true relative residual. */
int or_cheb(const tile_pc_t *pc, const float *al, const float *ab, const float *ac,
            const float *ar, const float *at, int periodic, const double *b, double *x,
            double lmin, double lmax, double tol, int maxit, double *relres) {
  int nx = pc->T.nx, ny = pc->T.ny;
  size_t n = (size_t)nx * ny;
  double *r = malloc(n * 8), *z = malloc(n * 8), *d = malloc(n * 8), *q = malloc(n * 8);
  double bn = sqrt(or_dot(b, b, nx, ny));
  if (bn == 0.0) bn = 1.0;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  int it = 0;
  double rel = 0.0;
  for (int restart = 0; restart < 8; ++restart) {
    or_apply(al, ab, ac, ar, at, nx, ny, periodic, x, q);
    for (size_t k = 0; k < n; ++k) r[k] = b[k] - q[k];
    rel = sqrt(or_dot(r, r, nx, ny)) / bn;
    if (rel <= tol || it >= maxit || !isfinite(rel)) break;
    or_tile_apply(pc, al, ab, ac, ar, at, r, z);
    for (size_t k = 0; k < n; ++k) d[k] = z[k] / theta;
    double rho = 1.0 / sigma;
    while (it < maxit) {
      or_apply(al, ab, ac, ar, at, nx, ny, periodic, d, q);
      for (size_t k = 0; k < n; ++k) {
        x[k] += d[k];
        r[k] -= q[k];
      }
      ++it;
      double rr = or_dot(r, r, nx, ny);
      if (!isfinite(rr)) {
        it = maxit;
        break;
      }
      if (sqrt(rr) / bn <= tol) break;
      or_tile_apply(pc, al, ab, ac, ar, at, r, z);
      const double rho1 = 1.0 / (2.0 * sigma - rho);
      const double c1 = rho1 * rho, c2 = 2.0 * rho1 / delta;
      for (size_t k = 0; k < n; ++k) d[k] = c1 * d[k] + c2 * z[k];
      rho = rho1;
    }
  }
  if (relres) *relres = rel;
  free(r), free(z), free(d), free(q);
  return it;
}

/* ---------------------------------------------------------------------
 * Barotropic pressure correction of FS (M/fs_GLOBAL.f90:1156-1283), the
 * ITMASK loop around the elliptic solve.  Arrays column-major with the
 * reference's shapes: U (I0,J0,K1), V (I0,J1,K1), IU0 / IV0 (I0,J0) and
 * IU (I0,J0,K1) / IV (I0,J1,K1) INTEGER*2, ODX / ODY / OCS (J0), CSV / ODYV
 * (J1), ODZ (K1), S (I2,J2), X / P0 (I0,J0), SCR (I0,J0,4); I1 = I0-1,
 * I2 = I0-2, J1 = J0-1, J2 = J0-2, K1 = K0-1.  REAL*4 arithmetic is done in
 * float, REAL*8 in double, in the Fortran evaluation order.
 */
#define U3(i, j, k) u[IX3(i0, j0, i, j, k)]
#define V3(i, j, k) v[IX3(i0, j0 - 1, i, j, k)]

/* Zero the top-layer advection velocity over land
 * (M/fs_GLOBAL.f90:1158-1171; the periodic faces under LOPENW == 1). */
void or_fs_mask(int i0, int j0, float *u, float *v, const int16_t *iu0, const int16_t *iv0,
                int periodic) {
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, j2 = j0 - 2;
  for (int j = 2; j <= j1; ++j) {
    for (int i = 2; i <= i2; ++i) U3(i, j, 1) = (float)iu0[IX(i0, i, j)] * U3(i, j, 1);
    if (periodic) {
      U3(1, j, 1) = (float)iu0[IX(i0, 1, j)] * U3(1, j, 1);
      U3(i1, j, 1) = (float)iu0[IX(i0, i1, j)] * U3(i1, j, 1);
    }
  }
  for (int j = 2; j <= j2; ++j)
    for (int i = 2; i <= i1; ++i) V3(i, j, 1) = (float)iv0[IX(i0, i, j)] * V3(i, j, 1);
}

/* Free-surface right-hand side from continuity (FLAG_FS branch,
 * M/fs_GLOBAL.f90:1177-1192): W integrated from W(:,:,K0) = 0 upwards,
 *   W(I,J,K) = W(I,J,K+1) + ((U(I,J,K)-U(I-1,J,K))*ODX(J)
 *              + (CSV(J)*V(I,J,K)-CSV(J-1)*V(I,J-1,K))*OCS(J)*ODY(J)) / ODZ(K),
 * and S(I-1,J-1) = W(I,J,1). */
void or_fs_rhs(int i0, int j0, int k0, const float *u, const float *v, const float *odx,
               const float *ody, const float *ocs, const float *csv, const float *odz, float *s) {
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, k1 = k0 - 1;
  for (int j = 2; j <= j1; ++j)
    for (int i = 2; i <= i1; ++i) {
      float w = 0.f;
      for (int k = k1; k >= 1; --k) {
        const float temp1 = 1.f / odz[k - 1];
        const float temp = ocs[j - 1] * ody[j - 1];
        const float a = (U3(i, j, k) - U3(i - 1, j, k)) * odx[j - 1];
        const float b = csv[j - 1] * V3(i, j, k) - csv[j - 2] * V3(i, j - 1, k);
        w = w + (a + b * temp) * temp1;
      }
      s[IX(i2, i - 1, j - 1)] = w;
    }
}

/* After the solve (M/fs_GLOBAL.f90:1216-1280): P0 += ODT*X; the current
 * corrections SCR(:,:,1) (U faces, periodic under FLAG_PERIODIC_WE) and
 * SCR(:,:,2) (V faces) from the gradients of X, added to every layer
 * (IU / IV below the top) and accumulated in SCR(:,:,3) / SCR(:,:,4).
 * Returns the largest top-layer velocity on land faces (the loop's test). */
float or_fs_correct(int i0, int j0, int k0, const double *x, float odt, const float *odx,
                    const float *odyv, const int16_t *iu, const int16_t *iv, const int16_t *iu0,
                    const int16_t *iv0, float *p0, float *u, float *v, float *scr, int periodic) {
  const int i1 = i0 - 1, i2 = i0 - 2, j1 = j0 - 1, j2 = j0 - 2, k1 = k0 - 1;
  float *s1 = scr, *s2 = scr + (size_t)i0 * j0, *s3 = scr + 2 * (size_t)i0 * j0,
        *s4 = scr + 3 * (size_t)i0 * j0;
  for (int j = 2; j <= j1; ++j)
    for (int i = 2; i <= i1; ++i)
      p0[IX(i0, i, j)] = (float)((double)p0[IX(i0, i, j)] + (double)odt * x[IX(i0, i, j)]);
  for (int j = 2; j <= j1; ++j) {
    for (int i = 2; i <= i2; ++i)
      s1[IX(i0, i, j)] = (float)(-((x[IX(i0, i + 1, j)] - x[IX(i0, i, j)]) * (double)odx[j - 1]));
    s1[IX(i0, 1, j)] = 0.f;
    s1[IX(i0, i1, j)] = 0.f;
    if (periodic) {
      s1[IX(i0, 1, j)] = (float)(-((x[IX(i0, 2, j)] - x[IX(i0, i1, j)]) * (double)odx[j - 1]));
      s1[IX(i0, i1, j)] = s1[IX(i0, 1, j)];
    }
    for (int i = 1; i <= i1; ++i) {
      const float c = s1[IX(i0, i, j)];
      s3[IX(i0, i, j)] = s3[IX(i0, i, j)] + c;
      U3(i, j, 1) = U3(i, j, 1) + c;
      for (int k = 2; k <= k1; ++k) U3(i, j, k) = U3(i, j, k) + c * (float)iu[IX3(i0, j0, i, j, k)];
    }
  }
  for (int j = 2; j <= j2; ++j)
    for (int i = 2; i <= i1; ++i)
      s2[IX(i0, i, j)] = (float)(-((x[IX(i0, i, j + 1)] - x[IX(i0, i, j)]) * (double)odyv[j - 1]));
  for (int i = 2; i <= i1; ++i) {
    s2[IX(i0, i, 1)] = 0.f;
    s2[IX(i0, i, j1)] = 0.f;
  }
  for (int j = 1; j <= j1; ++j)
    for (int i = 2; i <= i1; ++i) {
      s4[IX(i0, i, j)] = s4[IX(i0, i, j)] + s2[IX(i0, i, j)];
      V3(i, j, 1) = V3(i, j, 1) + s2[IX(i0, i, j)];
    }
  for (int k = 2; k <= k1; ++k)
    for (int j = 1; j <= j1; ++j)
      for (int i = 2; i <= i1; ++i)
        V3(i, j, k) = V3(i, j, k) + s2[IX(i0, i, j)] * (float)iv[IX3(i0, j0 - 1, i, j, k)];
  float tmp = 0.f;
  for (int j = 2; j <= j1; ++j)
    for (int i = 2; i <= i2; ++i) {
      const float t = (float)(1 - iu0[IX(i0, i, j)]) * fabsf(U3(i, j, 1));
      tmp = tmp > t ? tmp : t;
    }
  for (int j = 2; j <= j2; ++j)
    for (int i = 2; i <= i1; ++i) {
      const float t = (float)(1 - iv0[IX(i0, i, j)]) * fabsf(V3(i, j, 1));
      tmp = tmp > t ? tmp : t;
    }
  return tmp;
}
#undef U3
#undef V3
