// Device structures and tile-SEVP march routines shared by the solver
// kernels (solver.cu) and the fused one-launch iterations (fused.cu).
#pragma once
#include <type_traits>

#include "common.cuh"
#include "tile_sevp.cuh"

namespace sevp {

// ------------------------------------------------------------------ state
struct SolveState {
  double rz;      // current r.z
  double pq;      // current p.(A p)
  double rr;      // current ||r||^2 (recursive residual)
  double bb;      // reference norm^2 for the stopping test
  double alpha, beta;
  double tol2;    // stop when rr <= tol2 * bb
  double rr64;    // FP64 true residual ||b - A x||^2 (residual kernel)
  double bb64;    // ||b||^2 (residual kernel)
  // the same with every row scaled by the residual operator's row weight
  // (equal to rr64, bb64 when the context has no row weights); the PCG
  // recursion works on the scaled residual
  double rr64w, bb64w;
  // Chebyshev scalars of the fused iteration (sevp_set_chebyshev_bounds)
  double cheb_theta, cheb_delta, cheb_sigma, cheb_rho;
  int iter, max_iter, done, status;
  // 1: the next tile pass continues the previous search direction after a
  // residual replacement (beta = new r.z / old r.z instead of a restart)
  int keep_dir;
  // r.z of the last tile pass, also when that pass ended the run (rz keeps
  // the one before): a run resumed on a replaced residual takes its next
  // beta from the two
  double rz_next;
  // 1 when the last residual pass resumed the stopped run (its recursive
  // residual was close to the replaced one); 0 when the run restarts its
  // preconditioned residual from the replaced residual
  int resumed;
  unsigned ticket[4];
  // optional record of the PCG coefficients: alpha_j at hist[2 (j-1)],
  // beta_j at hist[2 (j-1) + 1] for iterations j = 1..hist_cap
  double *hist;
  int hist_cap;
};

struct Coeffs {
  const float *al, *ab, *ac, *ar, *at;
};

struct GridDims {
  int nx, ny, periodic;
};

// ------------------------------------------------ five-point stencil row
// Explicitly rounded multiply and fused multiply-add: the compiler may not
// pick which product of a sum it fuses, so every kernel that applies the
// operator forms the same value bit for bit.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// A x at one point: south, west, centre, east, north, accumulated in that
// order in the vector type T.
template <typename T>
__device__ __forceinline__ T stencil5(float cb, T vb, float cw, T vw, float cc, T vc, float ce,
                                      T ve, float cn, T va) {
  T av = mul_rn(T(cb), vb);
  av = fma_rn(T(cw), vw, av);
  av = fma_rn(T(cc), vc, av);
  av = fma_rn(T(ce), ve, av);
  return fma_rn(T(cn), va, av);
}

// ------------------------------------------------- reductions / finisher
// Writes this CTA's NV partial sums, and lets the last CTA to arrive sum all
// partials in block order and call fin(sums) once.
template <int NV, class Fin>
__device__ __forceinline__ void reduce_and_finish(double (&v)[NV], double *partials,
                                                  unsigned *ticket, Fin &fin) {
  __shared__ double red[NV * 32];
  __shared__ int s_last;
  const int nblk = gridDim.x * gridDim.y;
  const int bid = blockIdx.y * gridDim.x + blockIdx.x;
  block_sum<NV>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)bid * NV + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    s_last = (t == (unsigned)nblk - 1u);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(size_t)b * NV + k]);
    __syncthreads();
    block_sum<NV>(acc, red);
    if (threadIdx.x == 0) {
      fin(acc);
      *ticket = 0u;
      __threadfence();
    }
  }
}

// --------------------------------------------------- tile march routines
constexpr int kTileWarps = 8;
// FP32-vector tiles up to this height use k_tile_short (measured faster
// there; the FP64 kernel and taller tiles keep k_tile_apply)
constexpr int kShortTileRows = 6;


// Shared memory per warp: the tile's rows of z (FP64 marching state, 32
// lanes per row), the last-equation residual of each sub-block (stored at
// the sub-block's last row), and the mat-vec broadcast vector.
__host__ __device__ inline size_t tile_smem_per_warp(int hmax) {
  return (size_t)hmax * 32 * 8 * 2 + 32 * 8;
}

// Element of influence data whose precision is chosen per warp group: every
// matrix keeps the slot (and offset) of its FP64 layout, and a group stored
// as FP32 holds each matrix's mw * mw floats in the first half of its slot.
// A tile's base pointer carries the choice in its bit 2 (kMixF32Tag, set by
// tile_mats); offsets added to it in MixMat units (8 bytes) keep the tag,
// and seg_matvec removes it before reading.
struct alignas(4) MixMat {
  float lo, hi;
};
constexpr uintptr_t kMixF32Tag = 4;

// out(n) = sum_k dv[seg + k] * M[k * mw + n].  All loads of the column are
// issued before the first multiply-add, so a mat-vec costs one memory round
// trip instead of one per group of rows.  MT is the stored matrix type.
template <int WMAX, typename MT>
__device__ __forceinline__ double seg_matvec_w(const double *dv, int segbase, const MT *M, int mw,
                                               int n) {
  MT m[WMAX];
#pragma unroll
  for (int k = 0; k < WMAX; ++k) m[k] = (k < mw) ? __ldg(M + (size_t)k * mw + n) : MT(0);
  if (sizeof(MT) == 4) {
    // FP32 influence data: multiply-add in FP32 (the mixed-precision mode)
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < WMAX; ++k)
      if (k < mw) s += (float)dv[segbase + k] * (float)m[k];
    return (double)s;
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < WMAX; ++k)
    if (k < mw) s += dv[segbase + k] * (double)m[k];
  return s;
}
template <typename MT>
__device__ __forceinline__ double seg_matvec_t(const double *dv, int segbase, const MT *M, int mw,
                                               int n) {
  if (mw <= 8) return seg_matvec_w<8, MT>(dv, segbase, M, mw, n);
  if (mw <= 16) return seg_matvec_w<16, MT>(dv, segbase, M, mw, n);
  return seg_matvec_w<32, MT>(dv, segbase, M, mw, n);
}
template <typename MT>
__device__ __forceinline__ double seg_matvec(const double *dv, int segbase, const MT *M, int mw,
                                             int n) {
  if constexpr (std::is_same<MT, MixMat>::value) {
    const uintptr_t u = reinterpret_cast<uintptr_t>(M);
    if (u & kMixF32Tag)
      return seg_matvec_t<float>(dv, segbase, reinterpret_cast<const float *>(u - kMixF32Tag), mw,
                                 n);
    return seg_matvec_t<double>(dv, segbase, reinterpret_cast<const double *>(u), mw, n);
  } else {
    return seg_matvec_t<MT>(dv, segbase, M, mw, n);
  }
}

// Asynchronous copy of one 4- or 8-byte element from global to shared
// memory (zero-filled, with no global read, when pred is false).
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem, bool pred) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? BYTES : 0;
  if constexpr (BYTES == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(gmem), "r"(n)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(gmem), "r"(n)
                 : "memory");
}

// Influence data of tile (a, b) of warp group grp (mw: the tile's width;
// empty lanes get the buffer start), tagged for FP32 reads when the group
// is stored as FP32 in a MixMat buffer.
template <typename MT>
__device__ __forceinline__ const MT *tile_mats(const MT *mats, const TileGeom &tg, int b, int grp,
                                               int a, int mw) {
  const MT *m = mats + (mw > 0 ? tg.moff[(size_t)b * tg.tx + a] : 0);
  if constexpr (std::is_same<MT, MixMat>::value) {
    if (tg.grp_f32 && tg.grp_f32[(size_t)b * tg.txg + grp])
      m = reinterpret_cast<const MT *>(reinterpret_cast<uintptr_t>(m) + kMixF32Tag);
  }
  return m;
}

// 1/a for the marching rows: the hardware's approximate FP64 reciprocal
// refined by two Newton-Raphson steps r <- r + r (1 - a r), each of which
// squares the relative error (a few ulp at most from the rounded quotient).
// It is formed off the row recurrence's dependency chain.
__device__ __forceinline__ double march_rcp(double a) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
  double e = fma(-a, r, 1.0);
  r = fma(r, e, r);
  e = fma(-a, r, 1.0);
  return fma(r, e, r);
}

// Finishes a PCG iteration after pass B: r.z and r.r are complete.
struct TileFin {
  SolveState *st;
  __device__ void operator()(double (&s)[2]) {
    double rz = s[0], rr = s[1];
    int first = (st->beta == 0.0 && st->iter == 0 && !st->keep_dir);
    st->keep_dir = 0;
    st->rr = rr;
    st->rz_next = rz;
    if (!isfinite(rz) || !isfinite(rr)) {
      st->status = SEVP_NONFINITE;
      st->done = 1;
      return;
    }
    // a finished run keeps the previous r.z: a continuation after a
    // residual replacement takes beta = (new r.z) / (that r.z), the step
    // this run would have taken next
    if (rr <= st->tol2 * st->bb) {
      st->done = 1;
      st->status = SEVP_OK;
      return;
    }
    if (st->iter >= st->max_iter) {
      st->done = 1;
      st->status = SEVP_MAXITER;
      return;
    }
    if (rz == 0.0) {
      st->status = SEVP_BREAKDOWN;
      st->done = 1;
      return;
    }
    st->beta = first ? 0.0 : rz / st->rz;
    if (st->hist && st->iter >= 1 && st->iter <= st->hist_cap)
      st->hist[2 * (st->iter - 1) + 1] = st->beta;
    st->rz = rz;
  }
};

// The march of march_task_regs for a full-height task with one sub-block
// (hh == HM, nb == 1, the common case): the same operations in straight-line
// code, without the sub-block bookkeeping.  RCP: the FP32-vector march
// keeps the reciprocals of AT from the forward sweep for the backward sweep
// (the same rows) instead of forming them again; chosen per kernel, since
// the registers it takes pay off in some and not in others.  mv() gives an
// active lane its entry of the influence mat-vec of dv (filled by the
// forward sweep); post() runs on every lane once all lanes have it.
template <bool SYM, bool kChain, int HM, bool RCP, class Rhs, class Emit, class Mv, class Post>
__device__ __forceinline__ void march_task_full_mv(const float (&cc_)[HM], const float (&ce_)[HM],
                                                   const float (&cn_)[HM],
                                                   const float (&cw_)[SYM ? 1 : HM],
                                                   const float (&cs_)[SYM ? 1 : HM], int n, int mw,
                                                   bool active, int lane, double *dv, Rhs &&rhs,
                                                   Emit &&emit, Mv &&mv, Post &&post) {
  double zs[HM], rcp[RCP ? HM : 1];
  double zb = 0.0, zc = 0.0, rho = 0.0;
  float cn_prev = 0.f;
#pragma unroll
  for (int k = 0; k < HM; ++k) {
    double cw, cs;
    if (SYM) {
      const float arw = __shfl_up_sync(0xffffffffu, ce_[k], 1);
      cw = (n == 0) ? 0.0 : (double)arw;
      cs = (double)cn_prev;
      cn_prev = cn_[k];
    } else {
      cw = cw_[k];
      cs = cs_[k];
    }
    const double cc = cc_[k], ce = ce_[k];
    const double cn = active ? (double)cn_[k] : 1.0;
    const double rk = rhs(k);
    const double part = (kChain && active) ? (rk - cs * zb) - cc * zc : 0.0;
    double zw = __shfl_up_sync(0xffffffffu, zc, 1);
    double ze = __shfl_down_sync(0xffffffffu, zc, 1);
    if (n == 0) zw = 0.0;
    if (n >= mw - 1) ze = 0.0;
    zs[k] = zc;
    const double res = (kChain && active) ? (part - cw * zw) - ce * ze : 0.0;
    if (k < HM - 1) {
      double zn;
      if constexpr (kChain && RCP) {
        rcp[k] = march_rcp(cn);
        zn = res * rcp[k];
      } else if constexpr (kChain) {
        zn = res * march_rcp(cn);
      }
      else
        zn = active ? ((((rk - cw * zw) - cs * zb) - cc * zc) - ce * ze) / cn : 0.0;
      zb = zc;
      zc = zn;
    } else {
      if constexpr (kChain)
        rho = res;
      else
        rho = active ? (((rk - cw * zw) - cs * zb) - cc * zc) - ce * ze : 0.0;
    }
  }
  dv[lane] = rho;
  __syncwarp();
  const double v = active ? mv() : 0.0;
  __syncwarp();
  post();
  zs[0] += v;
  double hb = 0.0, hc = v;
  float cn_prev_b = 0.f;
#pragma unroll
  for (int k = 0; k < HM - 1; ++k) {
    const float ncc = active ? cc_[k] : 0.f, nce = active ? ce_[k] : 0.f;
    const float ncn = active ? cn_[k] : 1.f;
    double cw, cs;
    if (SYM) {
      const float arw = __shfl_up_sync(0xffffffffu, nce, 1);
      cw = (n == 0) ? 0.0 : (double)arw;
      cs = (double)cn_prev_b;
      cn_prev_b = ncn;
    } else {
      cw = active ? cw_[k] : 0.f;
      cs = active ? cs_[k] : 0.f;
    }
    const double cc = ncc, ce = nce, cn = ncn;
    const double part = kChain ? -(cs * hb) - cc * hc : 0.0;
    double hw = __shfl_up_sync(0xffffffffu, hc, 1);
    double he = __shfl_down_sync(0xffffffffu, hc, 1);
    if (n == 0) hw = 0.0;
    if (n >= mw - 1) he = 0.0;
    double hn;
    if constexpr (kChain)
      hn = active ? ((part - cw * hw) - ce * he) * (RCP ? rcp[k] : march_rcp(cn)) : 0.0;
    else
      hn = active ? ((((-(cw * hw)) - cs * hb) - cc * hc) - ce * he) / cn : 0.0;
    zs[k + 1] += hn;
    hb = hc;
    hc = hn;
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < HM; ++k) emit(k, zs[k]);
  }
}

template <typename MT, bool SYM, bool kChain, int HM, bool RCP, class Rhs, class Emit>
__device__ __forceinline__ void march_task_full(const float (&cc_)[HM], const float (&ce_)[HM],
                                                const float (&cn_)[HM],
                                                const float (&cw_)[SYM ? 1 : HM],
                                                const float (&cs_)[SYM ? 1 : HM], int n, int mw,
                                                bool active, int lane, int segbase, double *dv,
                                                const MT *mt, Rhs &&rhs, Emit &&emit) {
  march_task_full_mv<SYM, kChain, HM, RCP>(
      cc_, ce_, cn_, cw_, cs_, n, mw, active, lane, dv, rhs, emit,
      [&]() { return seg_matvec<MT>(dv, segbase, mt, mw, n); }, []() {});
}

// SEVP march of one task with every row in registers: the forward sweep
// (particular solution with zero guess rows and block-top corrections) and
// the backward sweep (guess-row values and homogeneous corrections) of
// k_tile_apply, operation for operation.  rhs(k) gives row k's right-hand
// side (0 for inactive lanes; called once per row k < hh, in order, by all
// lanes of the warp); emit(k, z) receives the solution of row k of an
// active lane as soon as its sub-block is final.  hh, nb and the sub-block bounds are the same for all
// lanes of a warp, so the predicated rows keep the warp converged for the
// shuffles and mat-vecs.
template <typename MT, bool SYM, bool kChain, int HM, bool RCP, class Rhs, class Emit>
__device__ __forceinline__ void march_task_regs(const float (&cc_)[HM], const float (&ce_)[HM],
                                                const float (&cn_)[HM],
                                                const float (&cw_)[SYM ? 1 : HM],
                                                const float (&cs_)[SYM ? 1 : HM], int hh, int nb,
                                                int n, int mw, bool active, int lane, int segbase,
                                                double *dv, const MT *mt, Rhs &&rhs, Emit &&emit) {
  if (nb == 1 && hh == HM) {
    march_task_full<MT, SYM, kChain, HM, RCP>(cc_, ce_, cn_, cw_, cs_, n, mw, active, lane,
                                              segbase, dv, mt, rhs, emit);
    return;
  }
  const size_t msz = (size_t)mw * mw;
  // ---- forward sweep
  double zs[HM], rho[HM];
  double zb = 0.0, zc = 0.0;
  float cn_prev = 0.f;
  int t = 0, kb = 0, ke = sub_start(1, hh, nb) - 1;
#pragma unroll
  for (int k = 0; k < HM; ++k) {
    zs[k] = 0.0;
    rho[k] = 0.0;
    if (k < hh) {
      double cw, cs;
      if (SYM) {
        const float arw = __shfl_up_sync(0xffffffffu, ce_[k], 1);
        cw = (n == 0) ? 0.0 : (double)arw;
        cs = (double)cn_prev;
        cn_prev = cn_[k];
      } else {
        cw = cw_[k];
        cs = cs_[k];
      }
      const double cc = cc_[k], ce = ce_[k];
      const double cn = active ? (double)cn_[k] : 1.0;
      const double rcp_k = kChain ? march_rcp(cn) : 0.0;
      const double rk = rhs(k);
      if (k == kb) zc = 0.0;
      const double part = (kChain && active) ? (rk - cs * zb) - cc * zc : 0.0;
      double zw = __shfl_up_sync(0xffffffffu, zc, 1);
      double ze = __shfl_down_sync(0xffffffffu, zc, 1);
      if (n == 0) zw = 0.0;
      if (n >= mw - 1) ze = 0.0;
      zs[k] = zc;
      const double res = (kChain && active) ? (part - cw * zw) - ce * ze : 0.0;
      if (k < ke) {
        double zn;
        if constexpr (kChain)
          zn = res * rcp_k;
        else
          zn = active ? ((((rk - cw * zw) - cs * zb) - cc * zc) - ce * ze) / cn : 0.0;
        zb = zc;
        zc = zn;
      } else {
        double rh;
        if constexpr (kChain)
          rh = res;
        else
          rh = active ? (((rk - cw * zw) - cs * zb) - cc * zc) - ce * ze : 0.0;
        rho[k] = rh;
        if (t < nb - 1) {
          dv[lane] = rh;
          __syncwarp();
          double sc = active ? seg_matvec<MT>(dv, segbase, mt + (size_t)(nb + t) * msz, mw, n) : 0.0;
          __syncwarp();
          zc = zc - sc;
        }
        zb = zc;
        ++t;
        kb = k + 1;
        ke = sub_start(t + 1, hh, nb) - 1;
      }
    }
  }
  // ---- backward sweep
  double vnext = 0.0;
  for (t = nb - 1; t >= 0; --t) {
    kb = sub_start(t, hh, nb);
    ke = sub_start(t + 1, hh, nb) - 1;
    double rho_ke = 0.0;
    float cn_ke = 0.f, cnb = 0.f;
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      if (k == ke) rho_ke = rho[k], cn_ke = cn_[k];
      if (k == kb - 1) cnb = cn_[k];
    }
    const double cnk = active ? (double)cn_ke : 0.0;
    dv[lane] = rho_ke - cnk * vnext;
    __syncwarp();
    double v = active ? seg_matvec<MT>(dv, segbase, mt + (size_t)t * msz, mw, n) : 0.0;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < HM; ++k)
      if (k == kb) zs[k] += v;
    double hb = 0.0, hc = v;
    if (!active) cnb = 0.f;
    if (t > 0) {
      dv[lane] = v * (double)cnb;
      __syncwarp();
      hb = active ? seg_matvec<MT>(dv, segbase, mt + (size_t)(nb + t - 1) * msz, mw, n) : 0.0;
      __syncwarp();
    }
    float cn_prev_b = cnb;
#pragma unroll
    for (int k = 0; k < HM - 1; ++k) {
      if (k >= kb && k < ke) {
        const float ncc = active ? cc_[k] : 0.f, nce = active ? ce_[k] : 0.f;
        const float ncn = active ? cn_[k] : 1.f;
        double cw, cs;
        if (SYM) {
          const float arw = __shfl_up_sync(0xffffffffu, nce, 1);
          cw = (n == 0) ? 0.0 : (double)arw;
          cs = (double)cn_prev_b;
          cn_prev_b = ncn;
        } else {
          cw = active ? cw_[k] : 0.f;
          cs = active ? cs_[k] : 0.f;
        }
        const double cc = ncc, ce = nce, cn = ncn;
        const double rcp_k = kChain ? march_rcp(cn) : 0.0;
        const double part = kChain ? -(cs * hb) - cc * hc : 0.0;
        double hw = __shfl_up_sync(0xffffffffu, hc, 1);
        double he = __shfl_down_sync(0xffffffffu, hc, 1);
        if (n == 0) hw = 0.0;
        if (n >= mw - 1) he = 0.0;
        double hn;
        if constexpr (kChain)
          hn = active ? ((part - cw * hw) - ce * he) * rcp_k : 0.0;
        else
          hn = active ? ((((-(cw * hw)) - cs * hb) - cc * hc) - ce * he) / cn : 0.0;
        zs[k + 1] += hn;
        hb = hc;
        hc = hn;
      }
    }
    if (active) {
#pragma unroll
      for (int k = 0; k < HM; ++k)
        if (k >= kb && k <= ke) emit(k, zs[k]);
    }
    vnext = v;
  }
}

// Coefficient rows of one task into registers.
template <bool SYM, int HM>
__device__ __forceinline__ void load_task_coeffs(const Coeffs &c, size_t idx0, int nx, int hh,
                                                 bool active, float (&cc_)[HM], float (&ce_)[HM],
                                                 float (&cn_)[HM], float (&cw_)[SYM ? 1 : HM],
                                                 float (&cs_)[SYM ? 1 : HM]) {
#pragma unroll
  for (int k = 0; k < HM; ++k) {
    const bool ok = active && k < hh;
    const size_t id = ok ? idx0 + (size_t)k * nx : 0;
    cc_[k] = ok ? __ldg(c.ac + id) : 0.f;
    ce_[k] = ok ? __ldg(c.ar + id) : 0.f;
    cn_[k] = ok ? __ldg(c.at + id) : 0.f;
    if (!SYM) {
      cw_[k] = ok ? __ldg(c.al + id) : 0.f;
      cs_[k] = ok ? __ldg(c.ab + id) : 0.f;
    }
  }
}

// ----------------------------------------- one-launch Chebyshev iteration
// (fused.cu): one grid pass per iteration, the operator applied inside the
// tile kernel to the previous launch's direction.
constexpr int kChebMaxRows = 8;  // tile rows held in registers

template <typename V>
struct ChebLaunch {
  int sym;            // the operator is symmetric: 3-plane reads
  int mats_fp32;      // mats holds FP32 influence data (1), or MixMat data (2)
  TileGeom tg;
  Coeffs c;
  int periodic;
  const void *mats;
  const V *din;       // d_k
  V *dout, *x, *r;    // d_{k+1}; x and r in place
  SolveState *st;
  double *partials;
  unsigned *ticket;
  cudaStream_t stream;
};
template <typename V>
int cheb_launch(const ChebLaunch<V> &L);

// ------------------------------------------------------- PCG pass A
// Finisher of pass A: p.q is complete; alpha = r.z / p.q.
struct PassAFin {
  SolveState *st;
  __device__ void operator()(double (&s)[1]) {
    st->pq = s[0];
    st->iter += 1;
    if (!isfinite(s[0])) {
      st->status = SEVP_NONFINITE;
      st->done = 1;
    } else if (s[0] == 0.0) {
      st->status = SEVP_BREAKDOWN;
      st->done = 1;
    } else {
      st->alpha = st->rz / s[0];
      if (st->hist && st->iter <= st->hist_cap) st->hist[2 * (st->iter - 1)] = st->alpha;
    }
  }
};

// Pass A on TMA-staged tiles (stencil_tma.cu): p = z + beta p_old (z alone
// when beta = 0), q = A p, alpha = r.z / p.q.
template <typename V>
struct PassALaunch {
  GridDims g;
  Coeffs c;
  int sym;
  const V *z, *pold;
  V *pnew, *q;
  SolveState *st;
  double *partials;
  size_t partials_n;  // doubles in partials
  unsigned *ticket;
  cudaStream_t stream;
};
// Whether the grid and the buffers meet the tensor copy's alignment rules;
// the launch returns SEVP_BAD_ARG (nothing launched) when they do not.
template <typename V>
bool pass_a_tma_eligible(const PassALaunch<V> &L);
template <typename V>
int pass_a_tma_launch(const PassALaunch<V> &L);

// PCG pass B on FP32 vectors with the task rows and influence matrices
// brought in by the tensor memory accelerator (tile_tma.cu): x += alpha p,
// r -= alpha q, z = M^-1 r on the block-Jacobi tiles (symmetric operator,
// FP64 influence data), r.z and r.r, and the finish of the iteration.
struct PassBLaunch {
  TileGeom tg;
  Coeffs c;
  const double *mats;
  float *x;
  const float *p;
  float *r;
  const float *q;
  float *z;
  SolveState *st;
  double *partials;
  size_t partials_n;  // doubles in partials (three per CTA are used)
  unsigned *ticket;
  unsigned blocks;  // grid size (the register kernel's, so the sums run in its order)
  cudaStream_t stream;
};
// Whether the tiling and the buffers suit the kernel (tile columns of 8, 16
// or 32 lanes, unshifted, at most kShortTileRows rows; rows of a multiple
// of 16 bytes; 16-byte aligned buffers; tensor maps the driver accepts).
bool pass_b_tma_eligible(const PassBLaunch &L);
// SEVP_BAD_ARG (nothing launched) when not eligible.
int pass_b_tma_launch(const PassBLaunch &L);

}  // namespace sevp
