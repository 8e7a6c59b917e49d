// Fortran-compatible C entry points (include/sevp_b200.h, first layer).
//
// Each routine takes the reference's argument list by reference with
// column-major host arrays, copies the array spans the reference routine
// touches to the GPU, runs the drop-in kernels and copies the outputs back.
// The reference stops the program on errors; these record a status instead
// (sevp_last_status) and leave the outputs unchanged when they fail.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "dropin.cuh"

using namespace sevp;

namespace {
thread_local int g_status = SEVP_OK;
int g_periodic_we = 1;
bool g_cache_on = false;

// Device blocks of finished calls, kept for the next calls while caching is
// on (sevp_dropin_cache), so that a call's workspaces cost no cudaMalloc /
// cudaFree: (bytes, device, block).  A block goes back to the pool when its
// call ends; before blocks are handed out again the device is synchronised
// once (a call that failed half-way may have left a kernel running).
struct PoolBlock {
  size_t bytes;
  int device;
  void *p;
};
std::vector<PoolBlock> g_pool;
bool g_pool_released = false;

void *pool_get(size_t bytes, size_t *cap) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return nullptr;
  if (g_pool_released) {
    if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
    g_pool_released = false;
  }
  int best = -1;
  for (size_t k = 0; k < g_pool.size(); ++k)
    if (g_pool[k].device == device && g_pool[k].bytes >= bytes &&
        (best < 0 || g_pool[k].bytes < g_pool[(size_t)best].bytes))
      best = (int)k;
  if (best >= 0) {
    void *p = g_pool[(size_t)best].p;
    *cap = g_pool[(size_t)best].bytes;
    g_pool.erase(g_pool.begin() + best);
    return p;
  }
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  *cap = bytes;
  return p;
}
void pool_put(void *p, size_t cap) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return;
  g_pool.push_back(PoolBlock{cap, device, p});
  g_pool_released = true;
}

// Device copy of a host span, released on scope exit (to the pool while
// caching is on, else freed).
template <typename T>
struct DBuf {
  T *d = nullptr;
  size_t n = 0;
  size_t cap = 0;  // bytes of a pooled block (0: owned, freed on exit)
  int err = 0;
  explicit DBuf(size_t count) : n(count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (g_cache_on) {
      d = static_cast<T *>(pool_get(bytes, &cap));
      if (!d) err = 1, cap = 0;
    } else if (cudaMalloc((void **)&d, bytes) != cudaSuccess) {
      err = 1, d = nullptr;
    }
  }
  DBuf(const T *h, size_t count) : DBuf(count) {
    if (!err && h && count && cudaMemcpy(d, h, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
      err = 1;
  }
  ~DBuf() {
    if (d && cap)
      pool_put(d, cap);
    else if (d)
      cudaFree(d);
  }
  int zero() { return (!err && cudaMemset(d, 0, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess) ? 0 : 1; }
  int to_host(T *h) const {
    return (h && n && cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) ? 1 : 0;
  }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
};

// Device copies of read-only drop-in inputs (coefficients, RINV, RINV1, IE)
// kept between calls when the caller opts in (sevp_dropin_cache): keyed by
// the host address, the byte count and the device.  The caller promises that
// the arrays at those addresses keep their values until it calls
// sevp_dropin_cache(0), which frees the copies.
struct CacheEntry {
  const void *host;
  size_t bytes;
  int device;
  void *dev;
};
std::vector<CacheEntry> g_cache;

const void *cached_upload(const void *host, size_t bytes, int *err) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return *err = 1, nullptr;
  for (const CacheEntry &e : g_cache)
    if (e.host == host && e.bytes == bytes && e.device == device) return e.dev;
  void *d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return *err = 1, nullptr;
  if (cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return *err = 1, nullptr;
  }
  g_cache.push_back(CacheEntry{host, bytes, device, d});
  return d;
}

// A read-only input: the cached device copy when caching is on, else a copy
// owned by this call.
template <typename T>
struct RoBuf {
  std::unique_ptr<DBuf<T>> own;
  const T *d = nullptr;
  int err = 0;
  RoBuf(const T *h, size_t n) {
    if (g_cache_on && h && n) {
      d = static_cast<const T *>(cached_upload(h, n * sizeof(T), &err));
    } else {
      own.reset(new DBuf<T>(h, n));
      d = own->d;
      err = own->err;
    }
  }
};

// elements of a column-major (ld, rows) array accessed for `cols` columns
inline size_t span(int ld, int rows, int cols) {
  return rows <= 0 ? 0 : (size_t)(rows - 1) * (size_t)ld + (size_t)cols;
}

int finish(int s) {
  if (s == SEVP_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      sevp_internal_set_error(e, "drop-in kernel", __FILE__, __LINE__);
      s = SEVP_CUDA_ERROR;
    }
  }
  g_status = s;
  return s;
}

#define ANYERR(...) any_err({__VA_ARGS__})
inline bool any_err(std::initializer_list<int> l) {
  for (int v : l)
    if (v) return true;
  return false;
}

bool valid_ie(const int *ie, int nblk, int jmax) {
  if (!ie || nblk < 1) return false;
  int prev = 1;
  for (int k = 0; k < nblk; ++k) {
    if (ie[k] < prev || ie[k] > jmax) return false;
    prev = ie[k];
  }
  return ie[0] >= 2;
}

// REP family: forward to the one-CTA marching solve.
void march_dropin(const float *ax, const float *ay, const float *bb, const float *cx,
                  const float *cy, const double *rinv, const double *rinv1, double *dum0,
                  double *dum1, double *dum2, const float *f, double *h, double *x, const int *ie,
                  int i0, int i2, int m0, int m2, int nblk, int periodic, int ldf, int ldh,
                  int hzero) {
  if (!ax || !ay || !bb || !cx || !cy || !rinv || !f || !h || !x || !ie || nblk < 1 || m2 < 1 ||
      i2 < 1 || i0 < m2 + 2 || (nblk > 1 && !rinv1) || m0 < m2 + 2) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int je = ie[nblk - 1];
  if (!valid_ie(ie, nblk, 1 << 30)) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int crows = je - 1;  // equation rows 1..IE(NBLK)-1
  const size_t msz = (size_t)m2 * m2;
  RoBuf<float> dax(ax, span(i2, crows, m2)), day(ay, span(i2, crows, m2)), dbb(bb, span(i2, crows, m2)),
      dcx(cx, span(i2, crows, m2)), dcy(cy, span(i2, crows, m2));
  DBuf<float> df(f, span(ldf, crows, m2));
  RoBuf<double> dr(rinv, msz * nblk), dr1(rinv1, msz * std::max(nblk - 1, 0));
  DBuf<double> d0(dum0, (size_t)m2 * std::max(nblk - 1, 1)), d1(dum1, m2), d2(dum2, m2);
  DBuf<double> dh(h, span(ldh, je, hzero)), dx(x, span(i0, je + 1, m2 + 2));
  RoBuf<int> die(ie, nblk);
  if (ANYERR(dax.err, day.err, dbb.err, dcx.err, dcy.err, df.err, dr.err, dr1.err, d0.err, d1.err,
             d2.err, dh.err, dx.err, die.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  MarchArgs a{dax.d, day.d, dbb.d, dcx.d, dcy.d, i2, df.d, ldf, dr.d, dr1.d, m2, d0.d, d1.d, d2.d,
              dh.d, ldh, hzero, dx.d, i0, periodic, i0, die.d, nblk};
  int s = dev_march_solve(a, 0);
  if (finish(s) != SEVP_OK) return;
  if (dx.to_host(x) || dh.to_host(h) || d1.to_host(dum1) || d2.to_host(dum2) ||
      (nblk > 1 && dum0 && d0.to_host(dum0)))
    g_status = SEVP_CUDA_ERROR;
}

void pre_dropin(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
                double *rinv, double *rinv1, double *h, const int *ie, int ldc, int m0, int m2,
                int nblk, int periodic, int gi0) {
  if (!ax || !ay || !bb || !cx || !cy || !rinv || !h || !ie || nblk < 1 || m2 < 1 ||
      m0 < m2 + 2 || ldc < m2 || (nblk > 1 && !rinv1) || !valid_ie(ie, nblk, 1 << 30)) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int je = ie[nblk - 1];
  const int crows = je - 1;
  const size_t msz = (size_t)m2 * m2;
  int maxrows = 0, jl = 1;
  for (int nb = 0; nb < nblk; ++nb) {
    maxrows = std::max(maxrows, ie[nb] + 1 - jl + 1);
    jl = ie[nb];
  }
  DBuf<float> dax(ax, span(ldc, crows, m2)), day(ay, span(ldc, crows, m2)), dbb(bb, span(ldc, crows, m2)),
      dcx(cx, span(ldc, crows, m2)), dcy(cy, span(ldc, crows, m2));
  DBuf<double> dr(msz * nblk), dr1(msz * std::max(nblk - 1, 1));
  DBuf<double> dh(h, span(m0, je + 1, m0));
  DBuf<double> hw((size_t)m2 * m0 * maxrows), b1(m2 + 1), b2(m2 + 1);
  DBuf<int> die(ie, nblk), bad(1);
  if (ANYERR(dax.err, day.err, dbb.err, dcx.err, dcy.err, dr.err, dr1.err, dh.err, hw.err, b1.err,
             b2.err, die.err, bad.err, bad.zero(), dr.zero(), dr1.zero())) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  PreArgs p{dax.d, day.d, dbb.d, dcx.d, dcy.d, ldc, dr.d, dr1.d, m2, hw.d, m0, m0, periodic, gi0,
            die.d, ie, nblk, b1.d, b2.d};
  int s = dev_pre(p, dh.d, bad.d, 0);
  if (finish(s) != SEVP_OK) return;
  int hbad = 0;
  cudaMemcpy(&hbad, bad.d, sizeof(int), cudaMemcpyDeviceToHost);
  if (dr.to_host(rinv) || (nblk > 1 && dr1.to_host(rinv1)) || dh.to_host(h)) {
    g_status = SEVP_CUDA_ERROR;
    return;
  }
  g_status = hbad ? SEVP_SINGULAR : SEVP_OK;
}

}  // namespace

bool sevp::dropin_cache_on() { return g_cache_on; }

void sevp_internal_set_status(int s) { g_status = s; }

extern "C" {

int sevp_last_status(void) { return g_status; }

int sevp_dropin_cache(int enable) {
  for (const CacheEntry &e : g_cache) cudaFree(e.dev);
  g_cache.clear();
  release_kept_work();
  for (const PoolBlock &b : g_pool) cudaFree(b.p);
  g_pool.clear();
  g_pool_released = false;
  g_cache_on = enable != 0;
  return SEVP_OK;
}
void sevp_set_periodic_we(int p) { g_periodic_we = p ? 1 : 0; }
int sevp_get_periodic_we(void) { return g_periodic_we; }

void rep1_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
           const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
           const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
           const int *nblk) {
  if (!i0 || !i2 || !nblk) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  march_dropin(ax, ay, bb, cx, cy, rinv, rinv1, dum0, dum1, dum2, f, h, x, ie, *i0, *i2, *i0, *i2,
               *nblk, 1, *i2, *i0, *i0);
}

void rep_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
          const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
          const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
          const int *nblk) {
  if (!i0 || !i2 || !nblk) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  march_dropin(ax, ay, bb, cx, cy, rinv, rinv1, dum0, dum1, dum2, f, h, x, ie, *i0, *i2, *i0, *i2,
               *nblk, 0, *i2, *i0, *i0);
}

void repbir_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
             const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
             const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
             const int *m0, const int *m2, const int *nblk) {
  if (!i0 || !i2 || !m0 || !m2 || !nblk) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  march_dropin(ax, ay, bb, cx, cy, rinv, rinv1, dum0, dum1, dum2, f, h, x, ie, *i0, *i2, *m0, *m2,
               *nblk, 0, *m2, *m0, *m0);
}

void repbir_period_(const float *ax, const float *ay, const float *bb, const float *cx,
                    const float *cy, const double *rinv, const double *rinv1, double *dum0,
                    double *dum1, double *dum2, const float *f, double *h, double *x,
                    const int *ie, const int *i0, const int *i2, const int *m0, const int *m2,
                    const int *nblk) {
  if (!i0 || !i2 || !m0 || !m2 || !nblk || *m0 != *i0) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  march_dropin(ax, ay, bb, cx, cy, rinv, rinv1, dum0, dum1, dum2, f, h, x, ie, *i0, *i2, *m0, *m2,
               *nblk, 1, *m2, *m0, *m0);
}

void pre1_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
           double *rinv, double *rinv1, double *h, const int *ie, const int *i0, const int *i2,
           const int *nblk) {
  if (!i0 || !i2 || !nblk || *i0 != *i2 + 2) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  pre_dropin(ax, ay, bb, cx, cy, rinv, rinv1, h, ie, *i2, *i0, *i2, *nblk, 1, *i0);
}

void pre_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
          double *rinv, double *rinv1, double *h, const int *ie, const int *i2, const int *m0,
          const int *m2, const int *nblk) {
  if (!i2 || !m0 || !m2 || !nblk) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  pre_dropin(ax, ay, bb, cx, cy, rinv, rinv1, h, ie, *i2, *m0, *m2, *nblk, 0, *m0);
}

void matinv_(double *b, const int *n) {
  if (!b || !n || *n < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int N = *n;
  DBuf<double> db(b, (size_t)N * N), b1(N + 1), b2(N + 1);
  DBuf<int> bad(1);
  if (ANYERR(db.err, b1.err, b2.err, bad.err, bad.zero())) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  int s = dev_matinv(db.d, N, b1.d, b2.d, bad.d, 0);
  if (finish(s) != SEVP_OK) return;
  int hbad = 0;
  cudaMemcpy(&hbad, bad.d, sizeof(int), cudaMemcpyDeviceToHost);
  if (db.to_host(b)) {
    g_status = SEVP_CUDA_ERROR;
    return;
  }
  g_status = hbad ? SEVP_SINGULAR : SEVP_OK;
}

static void sqprod_common(const float *al, const float *ab, const float *ac, const float *ar,
                          const float *at, const double *x, double *r, const int *i2,
                          const int *j2, int transpose) {
  if (!al || !ab || !ac || !ar || !at || !x || !r || !i2 || !j2 || *i2 < 1 || *j2 < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const size_t nc = (size_t)*i2 * *j2, nx = (size_t)(*i2 + 2) * (*j2 + 2);
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc);
  DBuf<double> dx(x, nx), dr(r, nx);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err, dx.err, dr.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  int s = dev_sqprod(a1.d, a2.d, a3.d, a4.d, a5.d, dx.d, dr.d, *i2, *j2, transpose, 0);
  if (finish(s) != SEVP_OK) return;
  if (dr.to_host(r)) g_status = SEVP_CUDA_ERROR;
}

void p_sqprod_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
               const double *x, double *r, const int *i2, const int *j2) {
  sqprod_common(al, ab, ac, ar, at, x, r, i2, j2, 0);
}

void p_sqprod_t_(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const double *x, double *r, const int *i2, const int *j2) {
  sqprod_common(al, ab, ac, ar, at, x, r, i2, j2, 1);
}

void p_inprod_(const double *r, const double *p, double *tp, const int *i2, const int *j2) {
  if (!r || !p || !tp || !i2 || !j2 || *i2 < 1 || *j2 < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const size_t nx = (size_t)(*i2 + 2) * (*j2 + 2);
  DBuf<double> dr(r, nx), dp(p, nx);
  if (ANYERR(dr.err, dp.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  double v = 0.0;
  int s = dev_inprod(dr.d, dp.d, *i2, *j2, &v, 0);
  if (finish(s) == SEVP_OK) *tp = v;
}

void solver_boundary_update_(double *x, const int *i2, const int *j2) {
  if (!x || !i2 || !j2 || *i2 < 1 || *j2 < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  if (!g_periodic_we) {
    g_status = SEVP_OK;
    return;
  }
  const size_t nx = (size_t)(*i2 + 2) * (*j2 + 2);
  DBuf<double> dx(x, nx);
  if (dx.err) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  int s = dev_boundary(dx.d, *i2, *j2, 0);
  if (finish(s) != SEVP_OK) return;
  if (dx.to_host(x)) g_status = SEVP_CUDA_ERROR;
}

void p_bicgstab_le_(const float *al, const float *ab, const float *ac, const float *ar,
                    const float *at, const float *b, double *x, const float *, const float *,
                    const float *, const float *, const float *, const int *i2, const int *j2) {
  if (!al || !ab || !ac || !ar || !at || !b || !x || !i2 || !j2 || *i2 < 1 || *j2 < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const size_t nc = (size_t)*i2 * *j2, nx = (size_t)(*i2 + 2) * (*j2 + 2);
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc), db(b, nc);
  DBuf<double> dx(x, nx);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err, db.err, dx.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  int it = 0;
  double res = 0.0;
  const int s = dev_bicgstab(a1.d, a2.d, a3.d, a4.d, a5.d, db.d, dx.d, *i2, *j2, g_periodic_we,
                             &it, &res, 0);
  const bool ran = (s == SEVP_OK || s == SEVP_MAXITER || s == SEVP_NONFINITE);
  if (finish(ran ? SEVP_OK : s) != SEVP_OK) return;
  g_status = s;
  if (dx.to_host(x)) g_status = SEVP_CUDA_ERROR;
}

void p_csi_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
            const double *mineig, const double *maxeig, const float *b, double *x, const float *,
            const float *, const float *, const float *, const float *, const int *i2,
            const int *j2) {
  if (!al || !ab || !ac || !ar || !at || !b || !x || !mineig || !maxeig || !i2 || !j2 || *i2 < 1 ||
      *j2 < 1 || !(*maxeig != *mineig)) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const size_t nc = (size_t)*i2 * *j2, nx = (size_t)(*i2 + 2) * (*j2 + 2);
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc), db(b, nc);
  DBuf<double> dx(x, nx);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err, db.err, dx.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  int it = 0;
  double res = 0.0;
  const int s = dev_csi(a1.d, a2.d, a3.d, a4.d, a5.d, *mineig, *maxeig, db.d, dx.d, *i2, *j2,
                        g_periodic_we, &it, &res, 0);
  const bool ran = (s == SEVP_OK || s == SEVP_MAXITER || s == SEVP_NONFINITE);
  if (finish(ran ? SEVP_OK : s) != SEVP_OK) return;
  g_status = s;
  if (dx.to_host(x)) g_status = SEVP_CUDA_ERROR;
}

void lanczos_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
              double *mineig, double *maxeig, const int *i2, const int *j2) {
  if (!al || !ab || !ac || !ar || !at || !mineig || !maxeig || !i2 || !j2 || *i2 < 1 || *j2 < 1) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const size_t nc = (size_t)*i2 * *j2;
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err)) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  double mn = 0.0, mx = 0.0;
  const int s = dev_lanczos(a1.d, a2.d, a3.d, a4.d, a5.d, *i2, *j2, &mn, &mx, 0);
  if (finish(s == SEVP_BREAKDOWN ? SEVP_OK : s) != SEVP_OK) return;
  g_status = s;
  *mineig = mn;
  *maxeig = mx;
}

void sevp_bir_sweeps_(const float *al, const float *ab, const float *ac, const float *ar,
                      const float *at, const float *sr, const double *rinv, const double *rinv1,
                      double *x, double *xx, const int *ie, const int *i2p, const int *j2p,
                      const int *nb0p, const int *nbirp, const int *niterp, const int *fix_wrap) {
  if (!al || !ab || !ac || !ar || !at || !sr || !rinv || !x || !xx || !ie || !i2p || !j2p ||
      !nb0p || !nbirp || !niterp || !fix_wrap) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int i2 = *i2p, j2 = *j2p, nb0 = *nb0p, nbir = *nbirp, niter = *niterp;
  if (i2 < 2 || j2 < 2 || nb0 < 1 || nbir < 2 || niter < 0 || (2 * i2) % nbir != 0 ||
      ((2 * i2 / nbir) % 2) != 0 || (nb0 > 1 && !rinv1) || !valid_ie(ie, nb0, j2 + 1)) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int ibir = 2 * i2 / nbir, inc = ibir / 2, i0 = i2 + 2, j0 = j2 + 2;
  const size_t nc = (size_t)i2 * j2, ibr2 = (size_t)ibir * ibir;
  const size_t rst = ibr2 * nb0, r1st = ibr2 * std::max(nb0 - 1, 1);
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc), ds(sr, nc);
  DBuf<double> dr(rinv, rst * nbir), dr1(rinv1, nb0 > 1 ? r1st * nbir : 0);
  DBuf<double> dx(x, (size_t)i0 * j0), dxx(xx, (size_t)(ibir + 2) * j0);
  DBuf<float> src((size_t)ibir * j2), cl((size_t)ibir * j2), cb((size_t)ibir * j2),
      cc((size_t)ibir * j2), cr((size_t)ibir * j2), ct((size_t)ibir * j2);
  DBuf<double> h((size_t)(ibir + 2) * j0), d0((size_t)ibir * std::max(nb0 - 1, 1)), d1(ibir), d2(ibir);
  DBuf<int> die(ie, nb0);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err, ds.err, dr.err, dr1.err, dx.err, dxx.err,
             src.err, cl.err, cb.err, cc.err, cr.err, ct.err, h.err, d0.err, d1.err, d2.err, die.err,
             h.zero())) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  StripArgs sa{ds.d, a1.d, a2.d, a3.d, a4.d, a5.d, dx.d, dxx.d, src.d, cl.d, cb.d, cc.d, cr.d, ct.d,
               i2, j2, ibir, *fix_wrap ? j2 + 2 : j2};
  int s = SEVP_OK;
  for (int it = 0; it < niter && !s; ++it)
    for (int n = 1; n <= nbir && !s; ++n) {
      const int il = (n - 1) * inc + 1;
      const double *R = dr.d + (size_t)(n - 1) * rst;
      const double *R1 = nb0 > 1 ? dr1.d + (size_t)(n - 1) * r1st : nullptr;
      if (n != nbir) {
        s = dev_strip_extract(sa, il, 0, 0);
        if (s) break;
        MarchArgs m{a1.d + (il - 1), a2.d + (il - 1), a3.d + (il - 1), a4.d + (il - 1),
                    a5.d + (il - 1), i2, src.d, ibir, R, R1, ibir, d0.d, d1.d, d2.d, h.d, ibir + 2,
                    ibir + 2, dx.d + (il - 1), i0, 0, i0, die.d, nb0};
        s = dev_march_solve(m, 0);
      } else {
        s = dev_strip_extract(sa, il, 1, 0);
        if (s) break;
        MarchArgs m{cl.d, cb.d, cc.d, cr.d, ct.d, ibir, src.d, ibir, R, R1, ibir, d0.d, d1.d, d2.d,
                    h.d, ibir + 2, ibir + 2, dxx.d, ibir + 2, 0, ibir + 2, die.d, nb0};
        s = dev_march_solve(m, 0);
        if (s) break;
        s = dev_strip_scatter(sa, il, g_periodic_we, 0);
      }
    }
  if (finish(s) != SEVP_OK) return;
  if (dx.to_host(x) || dxx.to_host(xx)) g_status = SEVP_CUDA_ERROR;
}

void sevp_pre_strips_(const float *al, const float *ab, const float *ac, const float *ar,
                      const float *at, double *rinv, double *rinv1, const int *ie, const int *i2p,
                      const int *j2p, const int *nb0p, const int *nbirp) {
  if (!al || !ab || !ac || !ar || !at || !rinv || !ie || !i2p || !j2p || !nb0p || !nbirp) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int i2 = *i2p, j2 = *j2p, nb0 = *nb0p, nbir = *nbirp;
  if (i2 < 2 || j2 < 2 || nb0 < 1 || nbir < 1 || (2 * i2) % nbir != 0 || (nb0 > 1 && !rinv1) ||
      !valid_ie(ie, nb0, j2 + 1)) {
    g_status = SEVP_BAD_ARG;
    return;
  }
  const int ibir = 2 * i2 / nbir, inc = ibir / 2, j0 = j2 + 2;
  const size_t nc = (size_t)i2 * j2, ibr2 = (size_t)ibir * ibir;
  const size_t rst = ibr2 * nb0, r1st = ibr2 * std::max(nb0 - 1, 1);
  int maxrows = 0, jl = 1;
  for (int nb = 0; nb < nb0; ++nb) {
    maxrows = std::max(maxrows, ie[nb] + 1 - jl + 1);
    jl = ie[nb];
  }
  DBuf<float> a1(al, nc), a2(ab, nc), a3(ac, nc), a4(ar, nc), a5(at, nc);
  DBuf<float> cl((size_t)ibir * j2), cb((size_t)ibir * j2), cc((size_t)ibir * j2),
      cr((size_t)ibir * j2), ct((size_t)ibir * j2);
  DBuf<double> dr(rst * nbir), dr1(r1st * nbir), hw((size_t)ibir * (ibir + 2) * maxrows),
      b1(ibir + 1), b2(ibir + 1);
  DBuf<int> die(ie, nb0), bad(1);
  if (ANYERR(a1.err, a2.err, a3.err, a4.err, a5.err, cl.err, cb.err, cc.err, cr.err, ct.err,
             dr.err, dr1.err, hw.err, b1.err, b2.err, die.err, bad.err, bad.zero(), dr.zero(),
             dr1.zero())) {
    finish(SEVP_CUDA_ERROR);
    return;
  }
  StripArgs sa{nullptr, a1.d, a2.d, a3.d, a4.d, a5.d, nullptr, nullptr, nullptr, cl.d, cb.d, cc.d,
               cr.d, ct.d, i2, j2, ibir, j2};
  int s = SEVP_OK;
  for (int n = 1; n <= nbir && !s; ++n) {
    const int il = (n - 1) * inc + 1;
    PreArgs p{};
    if (nbir == 1 || n != nbir) {
      p = PreArgs{a1.d + (il - 1), a2.d + (il - 1), a3.d + (il - 1), a4.d + (il - 1),
                  a5.d + (il - 1), i2, dr.d + (size_t)(n - 1) * rst,
                  dr1.d + (size_t)(n - 1) * r1st, ibir, hw.d, ibir + 2, ibir + 2, 0, ibir + 2,
                  die.d, ie, nb0, b1.d, b2.d};
    } else {
      s = dev_strip_extract(sa, il, 1, 0);
      if (s) break;
      p = PreArgs{cl.d, cb.d, cc.d, cr.d, ct.d, ibir, dr.d + (size_t)(n - 1) * rst,
                  dr1.d + (size_t)(n - 1) * r1st, ibir, hw.d, ibir + 2, ibir + 2, 0, ibir + 2,
                  die.d, ie, nb0, b1.d, b2.d};
    }
    s = dev_pre(p, nullptr, bad.d, 0);
  }
  if (finish(s) != SEVP_OK) return;
  int hbad = 0;
  cudaMemcpy(&hbad, bad.d, sizeof(int), cudaMemcpyDeviceToHost);
  if (dr.to_host(rinv) || (nb0 > 1 && dr1.to_host(rinv1))) {
    g_status = SEVP_CUDA_ERROR;
    return;
  }
  g_status = hbad ? SEVP_SINGULAR : SEVP_OK;
}

}  // extern "C"
