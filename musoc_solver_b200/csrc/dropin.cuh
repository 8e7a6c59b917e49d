// Device-side argument blocks and launchers of the reference-faithful
// drop-in routines (full-width SEVP, influence precompute, Krylov).
#pragma once
#include "common.cuh"

namespace sevp {

// The drop-in cache (sevp_dropin_cache, capi.cu): whether it is on, and the
// release of the Krylov work buffers kept while it is (krylov.cu).
bool dropin_cache_on();
void release_kept_work();

// Arguments of the marching solve; every pointer is a device pointer and
// every array keeps the reference's column-major layout and leading
// dimension (see M/sevp.f90:11-438).
struct MarchArgs {
  const float *ax, *ay, *bb, *cx, *cy;
  int ldc;
  const float *f;
  int ldf;
  const double *rinv, *rinv1;
  int m2;
  double *dum0, *dum1, *dum2;
  double *h;
  int ldh, hzero;
  double *x;
  int ldx;
  int periodic, gi0;
  const int *ie;
  int nblk;
};

struct PreArgs {
  const float *ax, *ay, *bb, *cx, *cy;
  int ldc;
  double *rinv, *rinv1;
  int m2;
  double *hwork;  // m2 slices of (ldh x rows) for the unit responses
  int ldh, hzero;
  int periodic, gi0;
  const int *ie;       // device
  const int *ie_host;  // host copy (block loop runs on the host)
  int nblk;
  double *b1, *b2;     // MATINV scratch, n + 1 each
};

struct StripArgs {
  const float *s, *al, *ab, *ac, *ar, *at;
  double *x, *xx;
  float *src, *cl, *cb, *cc, *cr, *ct;
  int i2, j2, ibir;
  int side_rows;  // rows of the wrapped strip's side boundaries copied: J2 (reference) or J2+2
};

int dev_march_solve(const MarchArgs &a, cudaStream_t st);
int dev_matinv(double *B, int n, double *b1, double *b2, int *bad, cudaStream_t st);
int dev_pre(const PreArgs &p, double *hfinal, int *bad, cudaStream_t st);
int dev_strip_extract(const StripArgs &s, int il, int mode, cudaStream_t st);
int dev_strip_scatter(const StripArgs &s, int il, int periodic, cudaStream_t st);

// Krylov drop-ins on padded (i2+2, j2+2) FP64 arrays.
int dev_sqprod(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
               const double *x, double *r, int i2, int j2, int transpose, cudaStream_t st);
int dev_inprod(const double *r, const double *p, int i2, int j2, double *result_host,
               cudaStream_t st);
int dev_boundary(double *x, int i2, int j2, cudaStream_t st);
int dev_bicgstab(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const float *b, double *x, int i2, int j2, int periodic,
                 int *iters, double *final_res, cudaStream_t st);
int dev_csi(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
            double mineig, double maxeig, const float *b, double *x, int i2, int j2, int periodic,
            int *iters, double *final_res, cudaStream_t st);
int dev_lanczos(const float *al, const float *ab, const float *ac, const float *ar,
                const float *at, int i2, int j2, double *mineig, double *maxeig, cudaStream_t st);

// Host restatements of the 10x10 tridiagonal eigen steps (M/sevp.f90:838-1006).
int host_figi(int n, const double *t, double *d, double *e, double *e2);
int host_ratqr(int n, double eps1, const double *d, const double *e, double *mineig);

}  // namespace sevp
