// Native SEVP-PCG solver for sm_100a: operator apply, tile SEVP
// preconditioners (block-Jacobi tiles, and the overlapping Schwarz sweep over
// a second, shifted tiling; precompute and apply), the FP64 /
// mixed-precision preconditioned conjugate-gradient drivers, and the time
// stepping calls that keep the solution history on the device.
//
// The reference solves the barotropic pressure equation with SEVP marching
// alone (M/sevp.f90:11-438) or with an unpreconditioned BiCGSTAB / Chebyshev
// iteration (M/sevp.f90:443-616).  This file implements the method the
// library adds: SEVP as the preconditioner of an outer CG iteration, with the
// domain cut into tiles that are solved by SEVP independently.
//
// Per PCG iteration two grid passes are made (the two global reductions of CG
// force two synchronisation points):
//   pass A (stencil kernel):  p = z + beta p_old ; q = A p ; partial p.q
//   pass B (tile kernel):     x += alpha p ; r -= alpha q ; z = M^{-1} r ;
//                             partial r.z and r.r
// (with the Schwarz preconditioner, pass B is three tile passes: the update
// with the first tiling's solve, then k_tile_couple on the shifted tiling
// and again on the first, the last one forming r.z and r.r)
// Scalars (alpha, beta, convergence) are formed on the device by the last CTA
// of each pass from the per-CTA partial sums, in a fixed order, so results
// are deterministic and the host only polls a "done" flag between chunks of
// iterations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "solver_core.cuh"

namespace sevp {

// ------------------------------------------------------ stencil kernels
// Column-walking 5-point stencil.  A CTA of 256 threads covers 32 columns;
// its 8 warps are stacked in y, each walking `rpw` rows.  The field value at
// a point is produced by op.value(idx) (fused producers: z + beta p, x + d);
// east/west neighbours come from warp shuffles, except at the warp's edge
// lanes, which evaluate the neighbour column directly (periodic wrap in x).
constexpr int kStencilThreads = 256;
constexpr int kStencilCols = 30;  // output columns per warp (32 loaded)
// Launch shape, chosen by measurement at 3600x2400 on a B200: the minimum
// resident CTAs cap the registers (64 for the stencil, 85 for the tile
// kernel) so that enough warps keep memory requests in flight; FP32 fields
// load 4 rows per step, FP64 fields 2.
#ifndef SEVP_STENCIL_UNROLL
#define SEVP_STENCIL_UNROLL 0
#endif
#ifndef SEVP_STENCIL_MINB
#define SEVP_STENCIL_MINB 6
#endif
#ifndef SEVP_TILE_MINB
#define SEVP_TILE_MINB 3
#endif

// SYM: the operator is symmetric (AL(i,j) = AR(i-1,j), AB(i,j) = AT(i,j-1)),
// so only AC, AR and AT are read; AL comes from the west lane's AR and AB
// from the previous row's AT.
template <class Op, bool SYM>
__global__ void __launch_bounds__(kStencilThreads, SEVP_STENCIL_MINB)
    k_stencil(GridDims g, Coeffs c, Op op, int rpw, double *partials, unsigned *ticket,
              SolveState *st) {
  using T = typename Op::T;
  // rows per step: all their loads are issued together
  constexpr int U = SEVP_STENCIL_UNROLL > 0 ? SEVP_STENCIL_UNROLL : (sizeof(T) == 4 ? 4 : 2);
  if (Op::kUsesState && st->done) return;
  op.prepare(st);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nx = g.nx, ny = g.ny;
  // Overlapping warps: a warp loads 32 consecutive columns and writes the
  // inner kStencilCols; lanes 0 and 31 only supply the west and east
  // neighbours, so every neighbour value arrives by shuffle from the same
  // coalesced row load.  The warps of a CTA sit side by side.
  const int raw = (blockIdx.x * (kStencilThreads / 32) + w) * kStencilCols + lane - 1;
  const bool out = lane >= 1 && lane <= kStencilCols && raw >= 0 && raw < nx;
  int i = raw;
  bool col_ok = raw >= 0 && raw < nx;
  if (g.periodic && raw == -1) i = nx - 1, col_ok = true;
  if (g.periodic && raw == nx) i = 0, col_ok = true;
  const int j0 = blockIdx.y * rpw;
  const int j1 = min(j0 + rpw, ny);
  double acc[Op::NV];
#pragma unroll
  for (int k = 0; k < Op::NV; ++k) acc[k] = 0.0;
  if (j0 < ny) {
    T vb = (j0 > 0 && col_ok) ? op.value((size_t)(j0 - 1) * nx + i) : T(0);
    T vc = col_ok ? op.value((size_t)j0 * nx + i) : T(0);
    float at_prev = (SYM && j0 > 0 && col_ok) ? __ldg(c.at + (size_t)(j0 - 1) * nx + i) : 0.f;
    for (int jb = j0; jb < j1; jb += U) {
      // loads: the next U rows of the field and U rows of coefficients
      T va[U];
      float cb[U], cw[U], ccn[U], ce[U], cn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = jb + u;
        const size_t idx = (size_t)j * nx + i;
        const bool rok = (j < j1) && col_ok;
        va[u] = (rok && j + 1 < ny) ? op.value(idx + nx) : T(0);
        ccn[u] = rok ? __ldg(c.ac + idx) : 0.f;
        ce[u] = rok ? __ldg(c.ar + idx) : 0.f;
        cn[u] = rok ? __ldg(c.at + idx) : 0.f;
        if (SYM) {
          cw[u] = 0.f;
          cb[u] = 0.f;
        } else {
          cb[u] = rok ? __ldg(c.ab + idx) : 0.f;
          cw[u] = rok ? __ldg(c.al + idx) : 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = jb + u;
        if (j >= j1) break;
        const T vw = __shfl_up_sync(0xffffffffu, vc, 1);
        const T ve = __shfl_down_sync(0xffffffffu, vc, 1);
        float cwu = cw[u], cbu = cb[u];
        if (SYM) {
          cwu = __shfl_up_sync(0xffffffffu, ce[u], 1);  // AL = AR of the west point
          cbu = (u == 0) ? at_prev : cn[u - 1];          // AB = AT of the south point
        }
        if (out) {
          const T av = stencil5(cbu, vb, cwu, vw, ccn[u], vc, ce[u], ve, cn[u], va[u]);
          op.emit((size_t)j * nx + i, j, vc, av, acc);
        }
        vb = vc;
        vc = va[u];
      }
      if (SYM) at_prev = cn[U - 1];
    }
  }
  reduce_and_finish<Op::NV>(acc, partials, ticket, op);
}

// Exact symmetry test of the five planes: AR(i,j) == AL(i+1,j) (with the
// periodic wrap) and AT(i,j) == AB(i,j+1).  Coefficients that multiply
// values outside the domain are not compared.
__global__ void k_check_symmetry(Coeffs c, int nx, int ny, int periodic, int *asym) {
  const size_t n = (size_t)nx * ny;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx), j = (int)(e / nx);
    bool bad = false;
    if (i < nx - 1) bad |= c.ar[e] != c.al[e + 1];
    else if (periodic) bad |= c.ar[e] != c.al[e + 1 - nx];
    if (j < ny - 1) bad |= c.at[e] != c.ab[e + nx];
    if (bad) atomicOr(asym, 1);
  }
}

// y = A x
template <typename TT>
struct OpApply {
  using T = TT;
  static constexpr int NV = 1;
  static constexpr bool kUsesState = false;
  const T *x;
  T *y;
  __device__ void prepare(SolveState *) {}
  __device__ T value(size_t idx) const { return x[idx]; }
  __device__ void emit(size_t idx, int, T, T av, double (&acc)[NV]) const { y[idx] = av; }
  __device__ void operator()(double (&)[NV]) {}
};

// PCG pass A: p = z + beta p_old ; q = A p ; p.q  -> alpha = r.z / p.q
template <typename V>
struct OpPassA {
  using T = V;
  static constexpr int NV = 1;
  static constexpr bool kUsesState = true;
  const V *z, *pold;
  V *pnew, *q;
  SolveState *st;
  V beta;
  bool first;
  __device__ void prepare(SolveState *s) {
    beta = (V)s->beta;
    first = (s->beta == 0.0);
  }
  __device__ V value(size_t idx) const {
    V zv = z[idx];
    return first ? zv : fma_rn(beta, pold[idx], zv);
  }
  __device__ void emit(size_t idx, int, V vc, V av, double (&acc)[NV]) const {
    pnew[idx] = vc;
    q[idx] = av;
    acc[0] += (double)vc * (double)av;
  }
  __device__ void operator()(double (&s)[NV]) { PassAFin{st}(s); }
};

// FP64 residual: x_out = x + d (d optional, FP32 correction); ru = b - A x_out
// with the residual operator; r = w_j ru (w_j the row weight of row j, 1
// without weights) written as R (double or float, optional).  Sums ||r||^2,
// ||w b||^2 (the scaled system the PCG recursion works on) and ||ru||^2,
// ||b||^2 (the stopping test).
template <typename R>
struct OpResidual {
  using T = double;
  // ||r||^2, ||w b||^2, ||ru||^2, ||b||^2, and for a resumed run ||r - r_old||^2
  static constexpr int NV = 5;
  static constexpr bool kUsesState = false;
  const double *x;
  const float *d;
  double *xout;
  const double *b;
  R *r;
  SolveState *st;
  double tol2;
  // (safety * outer tolerance)^2: the inner solve need not go below it; a
  // relative tolerance (of ||b||) unless abs_mode
  double outer2;
  // 1: also initialise the inner FP32 solve state; 2: the same for a PCG run
  // that resumes on this residual (beta from the stopped run's last two r.z)
  // when the stopped run's recursive residual, still in r, is within
  // resume_dev of the replaced one (relative)
  int set_inner;
  double resume_dev;
  const double *roww;  // row weights (ny) or null
  int abs_mode;        // the outer test is absolute: ||b - A x|| <= tol
  __device__ void prepare(SolveState *) {}
  __device__ double value(size_t idx) const {
    double v = x[idx];
    if (d) v += (double)d[idx];
    return v;
  }
  __device__ void emit(size_t idx, int j, double vc, double av, double (&acc)[NV]) const {
    if (xout) xout[idx] = vc;
    const double bv = b[idx];
    const double ru = bv - av;
    double rv = ru, bw = bv;
    if (roww) {
      const double w = roww[j];
      rv = w * ru;
      bw = w * bv;
    }
    if (set_inner == 2 && r) {
      const double dr = rv - (double)r[idx];
      acc[4] += dr * dr;
    }
    if (r) r[idx] = (R)rv;
    acc[0] += rv * rv;
    acc[1] += bw * bw;
    acc[2] += ru * ru;
    acc[3] += bv * bv;
  }
  __device__ void operator()(double (&s)[NV]) {
    st->rr64w = s[0];
    st->bb64w = s[1];
    st->rr64 = s[2];
    st->bb64 = s[3];
    if (set_inner) {
      // inner solve starts from zero: its reference norm is ||r||^2
      st->bb = s[0];
      st->rr = s[0];
      // reduce ||r|| by inner_tol, or only as far as the outer test needs
      const double target = abs_mode ? outer2 : outer2 * s[3];
      st->tol2 = s[2] > 0.0 ? fmax(tol2, fmin(target / s[2], 0.25)) : tol2;
      st->iter = 0;
      st->done = 0;
      st->beta = 0.0;
      st->status = SEVP_OK;
      // the step the stopped run would have taken next, now on the replaced
      // residual: z of its last pass stays (one step behind r).  Sound only
      // while the recursive residual still tracks the true one; a run that
      // reduced its residual down to FP32 rounding (a nearly exact
      // preconditioner) leaves a z unrelated to the replaced residual, and
      // the caller then preconditions the replaced residual afresh
      st->resumed = 0;
      if (set_inner == 2 && st->rz != 0.0 && s[4] <= resume_dev * resume_dev * s[0]) {
        st->beta = st->rz_next / st->rz;
        st->rz = st->rz_next;
        st->resumed = 1;
      }
    }
    if (!isfinite(s[0]) || !isfinite(s[2]) || !isfinite(s[3])) st->status = SEVP_NONFINITE;
  }
};

// --------------------------------------------------- tile apply kernel
// Inputs of one tile row for one lane (prefetched one row ahead).
template <typename V>
struct RowIn {
  V x, p, r, q;
  float cw, cs, cc, ce, cn;
};

template <typename V, bool UPDATE, bool SYM>
__device__ __forceinline__ void load_row(RowIn<V> &in, const Coeffs &c, const V *x, const V *p,
                                         const V *r, const V *q, size_t idx) {
  if (UPDATE) {
    in.x = x[idx];
    in.p = p[idx];
    in.q = q[idx];
  }
  in.r = r[idx];
  if (!SYM) {
    in.cw = __ldg(c.al + idx);
    in.cs = __ldg(c.ab + idx);
  }
  in.cc = __ldg(c.ac + idx);
  in.ce = __ldg(c.ar + idx);
  in.cn = __ldg(c.at + idx);
}

// UPDATE: fused x += alpha p, r -= alpha q before preconditioning (pass B).
// DOTS:   accumulate r.z and r.r and finish the iteration on the device.
// SYM:    symmetric operator: AL and AB are taken from the west lane's AR and
//         the previous row's AT (inside a tile the couplings that cross the
//         tile edge are dropped, so the edge values are never needed).
// MT:     stored type of the influence matrices (double, or float for the
//         FP32 inner solve).
template <typename V, typename MT, bool UPDATE, bool DOTS, bool SYM>
__global__ void __launch_bounds__(kTileWarps * 32, SEVP_TILE_MINB)
    k_tile_apply(TileGeom tg, Coeffs c, const MT *__restrict__ mats, V *x, const V *p, V *r,
                 const V *q, V *z, SolveState *st, double *partials, unsigned *ticket) {
  if ((DOTS || UPDATE) && st->done) return;
  constexpr bool kChain = sizeof(V) == 4;
  extern __shared__ __align__(16) unsigned char tsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char *base = tsm + tile_smem_per_warp(tg.hmax) * wib;
  double *zs = (double *)base;                       // [hmax][32]
  double *rho_s = zs + (size_t)tg.hmax * 32;         // [hmax][32]
  double *dv = rho_s + (size_t)tg.hmax * 32;         // [32]

  double acc_rz = 0.0, acc_rr = 0.0;
  // warps loop over the tile tasks with a grid-wide stride, so the grid can
  // be capped at the resident CTAs (no partial last wave)
  const int ntasks = tg.ty * tg.txg;
  for (int gw = blockIdx.x * kTileWarps + wib; gw < ntasks; gw += gridDim.x * kTileWarps) {
    const int b = gw / tg.txg;
    const int grp = gw - b * tg.txg;
    const int seg = lane / tg.wseg, n = lane - seg * tg.wseg, segbase = seg * tg.wseg;
    const int a = grp * tg.tpw + seg;
    const int mw = (a < tg.tx) ? tile_width(tg, a) : 0;
    const bool active = n < mw;
    const int nx = tg.nx;
    const int j0 = b * tg.th, hh = tile_height(tg, b), nb = tg.grp_nb[(size_t)b * tg.txg + grp];
    const int i = tile_col(tg, a, n);
    const MT *mt = tile_mats(mats, tg, b, grp, a, mw);
    const size_t msz = (size_t)mw * mw;
    double alpha = 0.0;
    if (UPDATE) alpha = st->alpha;

    // ---- forward sweep: particular solution with zero guess rows and
    //      block-top corrections (the elimination of the SEVP system).
    //      zs keeps each sub-block's top row before its correction.
    double zb = 0.0, zc = 0.0;
    float cn_prev = 0.f;  // AT of the previous row (AB of this row when SYM)
    int t = 0, kb = 0, ke = sub_start(1, hh, nb) - 1;
    RowIn<V> cur{}, nxt{};
    const size_t idx0 = (size_t)j0 * nx + i;
    if (active) load_row<V, UPDATE, SYM>(cur, c, x, p, r, q, idx0);
    for (int k = 0; k < hh; ++k) {
      const size_t idx = idx0 + (size_t)k * nx;
      if (active && k + 1 < hh) load_row<V, UPDATE, SYM>(nxt, c, x, p, r, q, idx + nx);
      double rv = 0.0;
      double cw, cs;
      if (SYM) {
        const float arw = __shfl_up_sync(0xffffffffu, cur.ce, 1);
        cw = (n == 0) ? 0.0 : (double)arw;
        cs = (double)cn_prev;
        cn_prev = cur.cn;
      } else {
        cw = cur.cw;
        cs = cur.cs;
      }
      const double cc = cur.cc, ce = cur.ce;
      const double cn = active ? (double)cur.cn : 1.0;
      // FP32 vectors (the inner solve): the row equation is evaluated as
      // ((r - AB z_s - AC z_c) - AL z_w - AR z_e) * (1 / AT), so only two
      // multiply-adds and a multiply wait on the neighbour shuffles; FP64
      // vectors keep the reference's order and division (faster there)
      const double rcp_k = kChain ? march_rcp(cn) : 0.0;
      if (active) {
        if (UPDATE) {
          V xn = cur.x + (V)alpha * cur.p;
          V rn = cur.r - (V)alpha * cur.q;
          x[idx] = xn;
          r[idx] = rn;
          rv = (double)rn;
        } else {
          rv = (double)cur.r;
        }
        acc_rr += rv * rv;
      }
      if (k == kb) zc = 0.0;
      const double part = (kChain && active) ? (rv - cs * zb) - cc * zc : 0.0;
      double zw = __shfl_up_sync(0xffffffffu, zc, 1);
      double ze = __shfl_down_sync(0xffffffffu, zc, 1);
      if (n == 0) zw = 0.0;
      if (n >= mw - 1) ze = 0.0;
      zs[k * 32 + lane] = zc;
      const double res = (kChain && active) ? (part - cw * zw) - ce * ze : 0.0;
      if (k < ke) {
        double zn;
        if constexpr (kChain)
          zn = res * rcp_k;
        else
          zn = active ? ((((rv - cw * zw) - cs * zb) - cc * zc) - ce * ze) / cn : 0.0;
        zb = zc;
        zc = zn;
      } else {
        double rho;
        if constexpr (kChain)
          rho = res;
        else
          rho = active ? (((rv - cw * zw) - cs * zb) - cc * zc) - ce * ze : 0.0;
        rho_s[k * 32 + lane] = rho;
        if (t < nb - 1) {
          dv[lane] = rho;
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
      cur = nxt;
    }
    // ---- backward sweep: guess-row values and homogeneous corrections
    double vnext = 0.0;
    for (t = nb - 1; t >= 0; --t) {
      kb = sub_start(t, hh, nb);
      ke = sub_start(t + 1, hh, nb) - 1;
      const double cnk = active ? (double)__ldg(c.at + idx0 + (size_t)ke * nx) : 0.0;
      dv[lane] = rho_s[ke * 32 + lane] - cnk * vnext;
      __syncwarp();
      double v = active ? seg_matvec<MT>(dv, segbase, mt + (size_t)t * msz, mw, n) : 0.0;
      __syncwarp();
      zs[kb * 32 + lane] += v;
      double hb = 0.0, hc = v;
      float cnb = 0.f;  // AT of row kb-1
      if (t > 0) {
        cnb = active ? __ldg(c.at + idx0 + (size_t)(kb - 1) * nx) : 0.f;
        dv[lane] = v * (double)cnb;
        __syncwarp();
        hb = active ? seg_matvec<MT>(dv, segbase, mt + (size_t)(nb + t - 1) * msz, mw, n) : 0.0;
        __syncwarp();
      }
      float ncw = 0.f, ncs = 0.f, ncc = 0.f, nce = 0.f, ncn = 1.f;
      if (active && kb < ke) {
        const size_t id = idx0 + (size_t)kb * nx;
        if (!SYM) ncw = __ldg(c.al + id), ncs = __ldg(c.ab + id);
        ncc = __ldg(c.ac + id), nce = __ldg(c.ar + id), ncn = __ldg(c.at + id);
      }
      float cn_prev_b = cnb;
      for (int k = kb; k < ke; ++k) {
        double cw, cs;
        const double cc = ncc, ce = nce, cn = ncn;
        if (SYM) {
          const float arw = __shfl_up_sync(0xffffffffu, nce, 1);
          cw = (n == 0) ? 0.0 : (double)arw;
          cs = (double)cn_prev_b;
          cn_prev_b = ncn;
        } else {
          cw = ncw;
          cs = ncs;
        }
        if (active && k + 1 < ke) {
          const size_t id = idx0 + (size_t)(k + 1) * nx;
          if (!SYM) ncw = __ldg(c.al + id), ncs = __ldg(c.ab + id);
          ncc = __ldg(c.ac + id), nce = __ldg(c.ar + id), ncn = __ldg(c.at + id);
        }
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
        zs[(k + 1) * 32 + lane] += hn;
        hb = hc;
        hc = hn;
      }
      if (active) {
#pragma unroll 4
        for (int k = kb; k <= ke; ++k) {
          const size_t idx = idx0 + (size_t)k * nx;
          V zv = (V)zs[k * 32 + lane];
          z[idx] = zv;
          if (DOTS) acc_rz += (double)r[idx] * (double)zv;
        }
      }
      vnext = v;
    }
  }
  if (DOTS) {
    double v2[2] = {acc_rz, acc_rr};
    TileFin fin{st};
    reduce_and_finish<2>(v2, partials, ticket, fin);
  }
}

// Tiles of at most HM rows (the short tiles the autotuner prefers): the same
// algorithm as k_tile_apply, with every row of a task loaded into registers
// at once (one memory round trip per task instead of one per row) and the
// rows unrolled.
template <typename V, typename MT, bool UPDATE, bool DOTS, bool SYM, int HM>
__global__ void __launch_bounds__(kTileWarps * 32, 2)
    k_tile_short(TileGeom tg, Coeffs c, const MT *__restrict__ mats, V *x, const V *p, V *r,
                 const V *q, V *z, SolveState *st, double *partials, unsigned *ticket) {
  if ((DOTS || UPDATE) && st->done) return;
  constexpr bool kChain = sizeof(V) == 4;
  __shared__ double dv_all[kTileWarps * 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *dv = dv_all + wib * 32;
  double acc_rz = 0.0, acc_rr = 0.0;
  double alpha = 0.0;
  if (UPDATE) alpha = st->alpha;
  const int ntasks = tg.ty * tg.txg;
  for (int gw = blockIdx.x * kTileWarps + wib; gw < ntasks; gw += gridDim.x * kTileWarps) {
    const int b = gw / tg.txg;
    const int grp = gw - b * tg.txg;
    const int seg = lane / tg.wseg, n = lane - seg * tg.wseg, segbase = seg * tg.wseg;
    const int a = grp * tg.tpw + seg;
    const int mw = (a < tg.tx) ? tile_width(tg, a) : 0;
    const bool active = n < mw;
    const int nx = tg.nx;
    const int j0 = b * tg.th, hh = tile_height(tg, b), nb = tg.grp_nb[(size_t)b * tg.txg + grp];
    const int i = tile_col(tg, a, n);
    const MT *mt = tile_mats(mats, tg, b, grp, a, mw);
    const size_t idx0 = (size_t)j0 * nx + i;

    // ---- all loads of the task
    V rr[HM], xx[UPDATE ? HM : 1], pp[UPDATE ? HM : 1], qq[UPDATE ? HM : 1];
    float cc_[HM], ce_[HM], cn_[HM], cw_[SYM ? 1 : HM], cs_[SYM ? 1 : HM];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      const size_t id = ok ? idx0 + (size_t)k * nx : 0;
      rr[k] = ok ? r[id] : V(0);
      if (UPDATE) {
        xx[k] = ok ? x[id] : V(0);
        pp[k] = ok ? p[id] : V(0);
        qq[k] = ok ? q[id] : V(0);
      }
    }
    load_task_coeffs<SYM, HM>(c, idx0, nx, hh, active, cc_, ce_, cn_, cw_, cs_);

    // row k's right-hand side: the residual, after the fused update
    // x += alpha p, r -= alpha q
    auto rhs = [&](int k) -> double {
      if (!active) return 0.0;
      if (UPDATE) {
        const size_t idx = idx0 + (size_t)k * nx;
        const V xn = xx[k] + (V)alpha * pp[k];
        const V rn = rr[k] - (V)alpha * qq[k];
        x[idx] = xn;
        r[idx] = rn;
        rr[k] = rn;
      }
      const double rv = (double)rr[k];
      acc_rr += rv * rv;
      return rv;
    };
    auto emit = [&](int k, double zk) {
      const V zv = (V)zk;
      z[idx0 + (size_t)k * nx] = zv;
      if (DOTS) acc_rz += (double)rr[k] * (double)zv;
    };
    march_task_regs<MT, SYM, kChain, HM, UPDATE && !DOTS>(cc_, ce_, cn_, cw_, cs_, hh, nb, n, mw,
                                                          active, lane, segbase, dv, mt, rhs, emit);
  }
  if (DOTS) {
    double v2[2] = {acc_rz, acc_rr};
    TileFin fin{st};
    reduce_and_finish<2>(v2, partials, ticket, fin);
  }
}

// One stage of the overlapping (two-tiling, symmetric multiplicative)
// Schwarz preconditioner on the tiling tg.  The stage's right-hand side is
// the residual left by the previous stage, r - A z_prev; because the
// previous stage solved its own tiles exactly, that residual is minus the
// couplings of its correction w across the boundaries of the previous
// stage's tiling (column shift xo): west/east neighbours inside this tile
// come by shuffle (the two tilings' column boundaries never coincide), and
// the tile rows' halo neighbours south and north are loaded.  The tile
// solves then run as in k_tile_short.
// MODE 0: out = M rhs.  MODE 1: out = base + w + M rhs.  MODE 2: as 1,
// plus r.z and r.r and the finish of the PCG iteration (TileFin).
// st may be null outside a PCG loop (MODE 0 and 1); in the loop a finished
// solve skips the stage.
template <typename V, typename MT, bool SYM, int HM, int MODE>
__global__ void __launch_bounds__(kTileWarps * 32, 2)
    k_tile_couple(TileGeom tg, int xo, int periodic, Coeffs c, const MT *__restrict__ mats,
                  const V *w, const V *base, const V *r, V *out, SolveState *st,
                  double *partials, unsigned *ticket) {
  if (st && st->done) return;
  constexpr bool kChain = sizeof(V) == 4;
  // base and residual rows of the final stage, staged by cp.async (one
  // slot per lane and row, read back only by the lane that copied it)
  constexpr int kStage = MODE == 2 ? 2 : (MODE == 1 ? 1 : 0);
  __shared__ double dv_all[kTileWarps * 32];
  __shared__ __align__(16) V stg_all[kStage ? kTileWarps * kStage * HM * 32 : 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *dv = dv_all + wib * 32;
  V *stg = stg_all + (kStage ? wib * kStage * HM * 32 : 0);
  double acc_rz = 0.0, acc_rr = 0.0;
  const int ntasks = tg.ty * tg.txg;
  for (int gw = blockIdx.x * kTileWarps + wib; gw < ntasks; gw += gridDim.x * kTileWarps) {
    const int b = gw / tg.txg;
    const int grp = gw - b * tg.txg;
    const int seg = lane / tg.wseg, n = lane - seg * tg.wseg, segbase = seg * tg.wseg;
    const int a = grp * tg.tpw + seg;
    const int mw = (a < tg.tx) ? tile_width(tg, a) : 0;
    const bool active = n < mw;
    const int nx = tg.nx;
    const int j0 = b * tg.th, hh = tile_height(tg, b), nb = tg.grp_nb[(size_t)b * tg.txg + grp];
    const int i = tile_col(tg, a, n);
    const MT *mt = tile_mats(mats, tg, b, grp, a, mw);
    const size_t idx0 = (size_t)j0 * nx + i;
    if constexpr (kStage > 0) {
#pragma unroll
      for (int k = 0; k < HM; ++k) {
        const bool ok = active && k < hh;
        const size_t id = ok ? idx0 + (size_t)k * nx : 0;
        cp_async_elem<sizeof(V)>(stg + k * 32 + lane, base + id, ok);
        if constexpr (kStage == 2) cp_async_elem<sizeof(V)>(stg + (HM + k) * 32 + lane, r + id, ok);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // boundaries of the previous stage's tiling at this column
    int qc = i - xo;
    if (qc < 0) qc += nx;
    bool wb = active && qc % tg.tm == 0;
    bool eb = active && ((qc + 1) % tg.tm == 0 || qc == nx - 1);
    if (!periodic && i == 0) wb = false;
    if (!periodic && i == nx - 1) eb = false;
    const bool has_s = active && j0 > 0, has_n = active && j0 + hh < tg.ny;

    // ---- loads: w rows and halo rows, coefficients
    V wv[HM];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      wv[k] = ok ? w[idx0 + (size_t)k * nx] : V(0);
    }
    const V ws = has_s ? w[idx0 - nx] : V(0);
    const V wn = has_n ? w[idx0 + (size_t)hh * nx] : V(0);
    float cc_[HM], ce_[HM], cn_[HM], cw_[SYM ? 1 : HM], cs_[SYM ? 1 : HM];
    load_task_coeffs<SYM, HM>(c, idx0, nx, hh, active, cc_, ce_, cn_, cw_, cs_);
    // AB of the tile's first row: the row below's AT when symmetric
    float ab0;
    if constexpr (SYM)
      ab0 = has_s ? __ldg(c.at + idx0 - nx) : 0.f;
    else
      ab0 = cs_[0];

    // row k's right-hand side: minus the couplings of w across the previous
    // tiling's boundaries (the shuffles run on all lanes)
    auto rhs = [&](int k) -> double {
      const double wwv = __shfl_up_sync(0xffffffffu, (double)wv[k], 1);
      const double wev = __shfl_down_sync(0xffffffffu, (double)wv[k], 1);
      float alv;
      if constexpr (SYM)
        alv = __shfl_up_sync(0xffffffffu, ce_[k], 1);
      else
        alv = cw_[k];
      double v = 0.0;
      if (wb) v -= (double)alv * wwv;
      if (eb) v -= (double)ce_[k] * wev;
      if (k == 0 && has_s) v -= (double)ab0 * (double)ws;
      if (k == hh - 1 && has_n) v -= (double)cn_[k] * (double)wn;
      return active ? v : 0.0;
    };
    if constexpr (kStage > 0) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    auto emit = [&](int k, double zk) {
      const size_t id = idx0 + (size_t)k * nx;
      if constexpr (MODE == 0) {
        out[id] = (V)zk;
      } else {
        const V zv = (V)(((double)stg[k * 32 + lane] + (double)wv[k]) + zk);
        out[id] = zv;
        if constexpr (MODE == 2) {
          const double rr = (double)stg[(HM + k) * 32 + lane];
          acc_rz += rr * (double)zv;
          acc_rr += rr * rr;
        }
      }
    };
    march_task_regs<MT, SYM, kChain, HM, MODE == 0>(cc_, ce_, cn_, cw_, cs_, hh, nb, n, mw, active,
                                                    lane, segbase, dv, mt, rhs, emit);
  }
  if constexpr (MODE == 2) {
    double v2[2] = {acc_rz, acc_rr};
    TileFin fin{st};
    reduce_and_finish<2>(v2, partials, ticket, fin);
  }
}

__global__ void k_to_float(const double *a, float *b, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    b[k] = (float)a[k];
}

// Per-tile marching growth: the smallest sub-block height s_max such that
// z^s <= growth, with z + 1/z = max over the tile's marched rows of
// (|AC| + |AL| + |AR|) / |AT|.  One warp per tile; writes s per tile, and
// log z per tile when lz is given (infinity where a marched AT is zero).
__global__ void k_tile_growth(TileGeom tg, Coeffs c, double log_growth, int *s_tile,
                              float *lz = nullptr) {
  const int lane = threadIdx.x & 31;
  const int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (tile >= tg.tx * tg.ty) return;
  const int a = tile % tg.tx, b = tile / tg.tx;
  const int mw = tile_width(tg, a), hh = tile_height(tg, b);
  double cmax = 2.0;
  bool bad = false;
  for (int e = lane; e < mw * (hh - 1); e += 32) {
    const int k = e / mw, n = e % mw;
    const size_t idx = (size_t)(b * tg.th + k) * tg.nx + tile_col(tg, a, n);
    double at = fabs((double)c.at[idx]);
    double num = fabs((double)c.ac[idx]) + fabs((double)c.al[idx]) + fabs((double)c.ar[idx]);
    if (at == 0.0) bad = true;
    else cmax = fmax(cmax, num / at);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    bad |= __shfl_xor_sync(0xffffffffu, (int)bad, o);
  }
  if (lane == 0) {
    int s = tg.th;
    if (bad) {
      s = 1;
    } else {
      const double zz = 0.5 * (cmax + sqrt(fmax(cmax * cmax - 4.0, 0.0)));
      if (zz > 1.0) s = (int)floor(log_growth / log(zz));
      if (lz) lz[tile] = (float)log(zz);
    }
    if (lz && bad) lz[tile] = INFINITY;
    s_tile[tile] = s < 1 ? 1 : (s > tg.th ? tg.th : s);
  }
}

// Influence data with the precision chosen per warp group (MixMat layout):
// a group flagged in tg.grp_f32 gets each matrix rounded to FP32 in the
// first half of its FP64 slot, the others an FP64 copy.  One CTA per tile.
__global__ void k_mix_influence(TileGeom tg, const double *mats, double *mix) {
  const int tile = blockIdx.x;
  const int a = tile % tg.tx, b = tile / tg.tx;
  const int grp = a / tg.tpw, mw = tile_width(tg, a);
  const int nb = tg.grp_nb[(size_t)b * tg.txg + grp];
  const bool f32 = tg.grp_f32[(size_t)b * tg.txg + grp] != 0;
  const size_t msz = (size_t)mw * mw, base = (size_t)tg.moff[tile];
  for (int t = 0; t < 2 * nb - 1; ++t) {
    const double *src = mats + base + t * msz;
    double *dst = mix + base + t * msz;
    for (size_t e = threadIdx.x; e < msz; e += blockDim.x) {
      if (f32)
        reinterpret_cast<float *>(dst)[e] = (float)src[e];
      else
        dst[e] = src[e];
    }
  }
}

// -------------------------------------------------- tile precompute
// One CTA per tile, 32 warps; warp g marches the response to a unit guess
// value in column g.  Coefficients are staged in shared memory.  The
// guess-row -> last-equation map of each sub-block is inverted by
// Gauss-Jordan elimination with partial pivoting.
__global__ void __launch_bounds__(1024)
    k_tile_precompute(TileGeom tg, Coeffs c, double *mats, int *status) {
  extern __shared__ __align__(16) unsigned char psm[];
  const int tile = blockIdx.x;
  const int a = tile % tg.tx, b = tile / tg.tx;
  const int mw = tile_width(tg, a), hh = tile_height(tg, b);
  const int nb = tg.grp_nb[(size_t)b * tg.txg + a / tg.tpw];
  const int j0 = b * tg.th;
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int TM = 32;
  float *cf = (float *)psm;  // [5][hmax][32]
  const int hm = tg.hmax;
  double *S = (double *)(psm + (size_t)5 * hm * TM * sizeof(float));  // [32][32]
  double *P = S + TM * TM;
  double *Aug = P + TM * TM;   // [32][64]
  double *R1p = Aug + TM * 2 * TM;
  double *fac = R1p + TM * TM;  // [32]
  __shared__ int s_piv;
  __shared__ double s_pval;
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  for (int e = threadIdx.x; e < hh * TM; e += blockDim.x) {
    int k = e / TM, n = e % TM;
    float w = 0.f, s = 0.f, cc = 0.f, ee = 0.f, nn = 0.f;
    if (n < mw) {
      const int col = tile_col(tg, a, n);
      size_t idx = (size_t)(j0 + k) * tg.nx + col;
      w = c.al[idx], s = c.ab[idx], cc = c.ac[idx], ee = c.ar[idx], nn = c.at[idx];
    }
    cf[(0 * hm + k) * TM + n] = w;
    cf[(1 * hm + k) * TM + n] = s;
    cf[(2 * hm + k) * TM + n] = cc;
    cf[(3 * hm + k) * TM + n] = ee;
    cf[(4 * hm + k) * TM + n] = nn;
  }
  __syncthreads();
  const size_t msz = (size_t)mw * mw;
  double *mt = mats + tg.moff[(size_t)b * tg.tx + a];
#define CF(q, k, n) ((double)cf[((q) * hm + (k)) * TM + (n)])
  for (int t = 0; t < nb; ++t) {
    const int kb = sub_start(t, hh, nb), ke = sub_start(t + 1, hh, nb) - 1;
    if (g < mw) {
      const int n = lane;
      double hb = (t > 0 && n < mw) ? R1p[g * TM + n] * CF(4, kb - 1, g) : 0.0;
      double hc = (n == g) ? 1.0 : 0.0;
      for (int k = kb; k < ke; ++k) {
        double hw = __shfl_up_sync(0xffffffffu, hc, 1);
        double he = __shfl_down_sync(0xffffffffu, hc, 1);
        if (n == 0) hw = 0.0;
        if (n >= mw - 1) he = 0.0;
        double hn = 0.0;
        if (n < mw)
          hn = -((((CF(0, k, n) * hw) + CF(1, k, n) * hb) + CF(2, k, n) * hc) + CF(3, k, n) * he) /
               CF(4, k, n);
        hb = hc;
        hc = hn;
      }
      double hw = __shfl_up_sync(0xffffffffu, hc, 1);
      double he = __shfl_down_sync(0xffffffffu, hc, 1);
      if (n == 0) hw = 0.0;
      if (n >= mw - 1) he = 0.0;
      if (n < mw) {
        S[g * TM + n] =
            (((CF(0, ke, n) * hw) + CF(1, ke, n) * hb) + CF(2, ke, n) * hc) + CF(3, ke, n) * he;
        P[g * TM + n] = hc;
      }
    }
    __syncthreads();
    // Gauss-Jordan on [S | I]
    for (int e = threadIdx.x; e < TM * 2 * TM; e += blockDim.x) {
      int r = e / (2 * TM), cix = e % (2 * TM);
      double v = 0.0;
      if (r < mw) {
        if (cix < mw) v = S[r * TM + cix];
        else if (cix >= TM && cix - TM < mw) v = (cix - TM == r) ? 1.0 : 0.0;
      }
      Aug[r * 2 * TM + cix] = v;
    }
    __syncthreads();
    for (int k = 0; k < mw; ++k) {
      if (g == 0) {
        double av = (lane >= k && lane < mw) ? fabs(Aug[lane * 2 * TM + k]) : -1.0;
        int ai = lane;
        for (int o = 16; o > 0; o >>= 1) {
          double ov = __shfl_down_sync(0xffffffffu, av, o);
          int oi = __shfl_down_sync(0xffffffffu, ai, o);
          if (ov > av || (ov == av && oi < ai)) av = ov, ai = oi;
        }
        if (lane == 0) {
          s_piv = ai;
          s_pval = av;
        }
      }
      __syncthreads();
      const int piv = s_piv;
      if (!(s_pval > 0.0) || !isfinite(s_pval)) {
        if (threadIdx.x == 0) s_bad = 1;
      }
      if (piv != k) {
        for (int cix = threadIdx.x; cix < 2 * TM; cix += blockDim.x) {
          double t0 = Aug[k * 2 * TM + cix];
          Aug[k * 2 * TM + cix] = Aug[piv * 2 * TM + cix];
          Aug[piv * 2 * TM + cix] = t0;
        }
      }
      __syncthreads();
      double pv = Aug[k * 2 * TM + k];
      double inv = (pv != 0.0) ? 1.0 / pv : 0.0;
      if (threadIdx.x < TM) fac[threadIdx.x] = Aug[threadIdx.x * 2 * TM + k];
      __syncthreads();
      for (int cix = threadIdx.x; cix < 2 * TM; cix += blockDim.x) Aug[k * 2 * TM + cix] *= inv;
      __syncthreads();
      for (int e = threadIdx.x; e < mw * 2 * TM; e += blockDim.x) {
        int r = e / (2 * TM), cix = e % (2 * TM);
        if (r != k) {
          double f = fac[r];
          if (f != 0.0) Aug[r * 2 * TM + cix] -= f * Aug[k * 2 * TM + cix];
        }
      }
      __syncthreads();
    }
    // Sinv_t -> global; R1_t = -Sinv_t P -> global and shared (next sub-block)
    for (int e = threadIdx.x; e < mw * mw; e += blockDim.x) {
      int r = e / mw, cix = e % mw;
      mt[(size_t)t * msz + e] = Aug[r * 2 * TM + TM + cix];
    }
    if (t < nb - 1) {
      for (int e = threadIdx.x; e < mw * mw; e += blockDim.x) {
        int r = e / mw, cix = e % mw;
        double s = 0.0;
        for (int k = 0; k < mw; ++k) s = s - Aug[r * 2 * TM + TM + k] * P[k * TM + cix];
        mt[(size_t)(nb + t) * msz + e] = s;
        R1p[r * TM + cix] = s;
      }
    }
    __syncthreads();
  }
#undef CF
  if (threadIdx.x == 0 && s_bad) atomicOr(status, 1);
}

}  // namespace sevp

// ======================================================================
// context
// ======================================================================
using namespace sevp;

// One tile set of the preconditioner: geometry, sub-block counts per warp
// group and per tile, and the influence data (FP64, plus an FP32 copy built
// on demand for the mixed solve's inner iterations).
struct Tiling {
  TileGeom tg{};
  Coeffs c{};                   // the planes its kernels read
  float *d_al = nullptr, *d_ar = nullptr;  // seam-cut AL/AR copies (closed grids, shifted tiling)
  int *d_grp_nb = nullptr;
  long long *d_moff = nullptr;
  double *d_mats = nullptr;
  float *d_mats32 = nullptr;
  // per-group-precision copy (MixMat layout) and its group flags
  // (sevp_set_influence_fp32)
  double *d_matsmix = nullptr;
  unsigned char *d_grp_f32 = nullptr;
  int f32_groups = 0;
  long long mix_bytes_per_pass = 0;
  long long mats_elems = 0;
  std::vector<int> grp_nb;   // per warp group (ty * txg)
  std::vector<int> tile_nb;  // effective sub-blocks per tile (ty * tx)
  bool built = false;
  void release() {
    for (void *p : {(void *)d_grp_nb, (void *)d_moff, (void *)d_mats, (void *)d_mats32,
                    (void *)d_al, (void *)d_ar, (void *)d_matsmix, (void *)d_grp_f32})
      if (p) cudaFree(p);
    d_grp_nb = nullptr, d_moff = nullptr, d_mats = nullptr, d_mats32 = nullptr;
    d_al = nullptr, d_ar = nullptr, d_matsmix = nullptr, d_grp_f32 = nullptr;
    tg.grp_f32 = nullptr;
    f32_groups = 0;
    mix_bytes_per_pass = 0;
    mats_elems = 0;
    built = false;
  }
};

struct sevp_ctx {
  int nx = 0, ny = 0, periodic = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  Coeffs c{};
  bool have_op = false;
  // tiles: ta is the block-Jacobi tiling; tb the shifted second tiling of
  // the overlapping Schwarz preconditioner (built when schwarz_req != 0)
  Tiling ta, tb;
  int sym = 0;                  // operator exactly symmetric: 3-plane kernels
  int asym = 0;                 // the operator is not symmetric: CG solves are refused
  int force_full = 0;           // use the 5-plane kernels regardless
  // operator of the FP64 residual passes when it is not the PCG operator c
  // (sevp_set_residual_operator): the caller's planes, with row weights w_j
  // such that c is (up to FP32 rounding) the symmetric W A
  Coeffs cres{};
  int res_sym = 0;
  bool have_res = false;
  const double *roww = nullptr;
  bool infl32_active = false;   // current solve uses the FP32 influence copies
  // growth limit of the per-group FP32 influence data of the FP32-vector
  // tile passes (sevp_set_influence_fp32; <= 1: off)
  double mix_limit = 0.0;
  // largest ||r_true - r_recursive|| / ||r_true|| at which a mixed PCG run
  // resumes on a replaced residual (sevp_set_resume_check)
  double resume_dev = 0.3;
  // the tiling request of the last sevp_set_operator (the second tiling is
  // built from it)
  sevp_tiling treq{};
  std::vector<int> treq_rows, treq_tiles;
  int schwarz_req = 0;  // requested column shift of tb: 0 off, -1 automatic
  // PCG coefficient record of FP64 solves (sevp_record_coefficients)
  double *hist = nullptr;
  int hist_cap = 0;
  // Schwarz work vectors: first-stage z and second-stage correction
  double *s1_64 = nullptr, *s2_64 = nullptr;
  float *s1_32 = nullptr, *s2_32 = nullptr;
  // work vectors
  size_t n = 0;
  double *r64 = nullptr, *z64 = nullptr, *p64[2] = {nullptr, nullptr}, *q64 = nullptr;
  double *x64s = nullptr;  // ping-pong partner for the refinement update
  float *r32 = nullptr, *z32 = nullptr, *p32[2] = {nullptr, nullptr}, *q32 = nullptr,
        *d32 = nullptr;
  // spectrum bounds of M^-1 A for the Chebyshev iteration (0: not set)
  double cheb_lmin = 0.0, cheb_lmax = 0.0;
  double *bh = nullptr;  // device staging for host solves
  double *xh = nullptr;
  double *e1h = nullptr, *e2h = nullptr;
  // time stepping with the history held on the device (sevp_step_host):
  // three rotating buffers, the last two solutions and the next output
  double *step_buf[3] = {nullptr, nullptr, nullptr};
  int step_e1 = 0, step_e2 = 1, step_hist = 0;
  // asynchronous stepping: b staged on a copy-in stream (two buffers), x
  // copied out on a copy-out stream; events order the reuse of the buffers
  cudaStream_t cp_in = nullptr, cp_out = nullptr;
  double *bstage[2] = {nullptr, nullptr};
  const double *bstage_src[2] = {nullptr, nullptr};
  int bstage_next = 0;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_out[3] = {nullptr, nullptr, nullptr};
  bool ev_out_set[3] = {false, false, false};
  cudaEvent_t ev_solved = nullptr;
  // coarse-grid feature averages of the learned warm start (3 planes)
  float *nn_avg = nullptr;
  size_t nn_avg_n = 0;
  // learned warm start (bound by the network module)
  sevp_warmstart_fn warm_fn = nullptr;
  void *warm_user = nullptr;
  int warm_launches_per_call = 0;
  const double *cur_b = nullptr;
  // device scalars
  SolveState *st = nullptr;
  SolveState *h_st = nullptr;  // pinned mirror
  double *partials = nullptr;
  size_t partials_n = 0;
  unsigned *tickets = nullptr;
  long long launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // CUDA graph of a check interval of the FP32 inner PCG loop (captured on a
  // private stream, replayed on the context stream); valid for the buffers
  // and influence-data choice it was captured with
  int use_graphs = 1;
  int stencil_rpw = 0;  // rows per CTA of the stencil kernels (0: not chosen yet)
  int pass_a_kernel = SEVP_PASS_A_TILES;
  int pass_b_kernel = SEVP_PASS_B_REGISTERS;
  int pass_b_used = -1;  // kernel of the last FP32 pass B launch
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t inner_graph = nullptr;
  int inner_graph_ce = 0;
  const void *inner_graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // optional per-kernel-class timing (CUDA events on the context stream)
  int prof = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  size_t ev_used = 0;
  std::vector<int> ev_class;  // 0 tile apply (pass B / precondition), 1 stencil
  double prof_ms[4] = {0, 0, 0, 0};
  long long prof_n[4] = {0, 0, 0, 0};
};

namespace {
// Brackets one launch with a pair of events when profiling is on.
struct ProfScope {
  sevp_ctx *c;
  int cls;
  cudaEvent_t e1 = nullptr;
  ProfScope(sevp_ctx *ctx, int k) : c(ctx), cls(k) {
    if (!c->prof) return;
    if (c->ev_used == c->ev_pool.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      c->ev_pool.push_back({a, b});
    }
    auto &pr = c->ev_pool[c->ev_used++];
    c->ev_class.push_back(cls);
    cudaEventRecord(pr.first, c->stream);
    e1 = pr.second;
  }
  ~ProfScope() {
    if (e1) cudaEventRecord(e1, c->stream);
  }
};
}  // namespace

namespace {
thread_local char g_err[512] = {0};
}
void sevp_internal_set_error(cudaError_t e, const char *what, const char *file, int line) {
  snprintf(g_err, sizeof g_err, "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
}
void sevp_internal_set_message(const char *msg) { snprintf(g_err, sizeof g_err, "%s", msg); }
extern "C" const char *sevp_last_error(void) { return g_err; }

extern "C" const char *sevp_status_string(int s) {
  switch (s) {
    case SEVP_OK: return "ok";
    case SEVP_MAXITER: return "iteration cap reached";
    case SEVP_BREAKDOWN: return "Krylov breakdown";
    case SEVP_NONFINITE: return "non-finite value";
    case SEVP_TIMEOUT: return "device wait timed out";
    case SEVP_BAD_ARG: return "bad argument";
    case SEVP_CUDA_ERROR: return "CUDA error";
    case SEVP_SINGULAR: return "singular influence matrix";
    case SEVP_NONSYMMETRIC: return "operator is not symmetric";
    default: return "unknown status";
  }
}

// Rows per CTA of the stencil kernels, chosen once per context: a CTA loads
// rpw + 2 rows, and the grid runs in ceil(CTAs / slots) waves, so pick the
// rpw in [8, 32] that minimises waves x (rpw + 2) (ties: more rows).
static int stencil_rpw(sevp_ctx *ctx) {
  if (ctx->stencil_rpw > 0) return ctx->stencil_rpw;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long slots = (long long)sms * SEVP_STENCIL_MINB;
  const long long gx = ceil_div(ceil_div(ctx->nx, kStencilCols), kStencilThreads / 32);
  int best = 8;
  long long best_cost = -1;
  for (int rpw = 8; rpw <= 32; ++rpw) {
    const long long ctas = gx * ceil_div(ctx->ny, rpw);
    const long long cost = ((ctas + slots - 1) / slots) * (rpw + 2);
    if (best_cost < 0 || cost <= best_cost) best = rpw, best_cost = cost;
  }
  ctx->stencil_rpw = std::max(1, std::min(best, ctx->ny));
  return ctx->stencil_rpw;
}

static dim3 stencil_grid(const sevp_ctx *ctx, int rpw) {
  const int groups = ceil_div(ctx->nx, kStencilCols);
  return dim3((unsigned)ceil_div(groups, kStencilThreads / 32), (unsigned)ceil_div(ctx->ny, rpw));
}

static size_t tile_warps(const TileGeom &tg) { return (size_t)tg.ty * tg.txg; }

template <class Op>
static int launch_stencil_c(sevp_ctx *ctx, const Op &op, int ticket_slot, const Coeffs &c,
                            int sym) {
  int rpw = stencil_rpw(ctx);
  dim3 grid = stencil_grid(ctx, rpw);
  GridDims gd{ctx->nx, ctx->ny, ctx->periodic};
  ProfScope ps(ctx, 1);
  if (sym)
    k_stencil<Op, true><<<grid, kStencilThreads, 0, ctx->stream>>>(
        gd, c, op, rpw, ctx->partials, ctx->tickets + ticket_slot, ctx->st);
  else
    k_stencil<Op, false><<<grid, kStencilThreads, 0, ctx->stream>>>(
        gd, c, op, rpw, ctx->partials, ctx->tickets + ticket_slot, ctx->st);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}
template <class Op>
static int launch_stencil(sevp_ctx *ctx, const Op &op, int ticket_slot) {
  return launch_stencil_c(ctx, op, ticket_slot, ctx->c, ctx->sym);
}

// Resident CTAs of a kernel on the current device at the given shared
// memory (queried once per kernel and size; one device per process is
// assumed).
template <typename K>
static int resident_ctas(K kern, size_t smem, size_t &set_smem, int &slots) {
  if (slots > 0 && set_smem == smem) return SEVP_OK;
  // static plus dynamic shared memory above 48 KB needs the opt-in
  if (smem > 0)
    SEVP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, dev = 0, sms = 0;
  SEVP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileWarps * 32, smem));
  SEVP_CUDA_TRY(cudaGetDevice(&dev));
  SEVP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  slots = std::max(1, per_sm) * sms;
  set_smem = smem;
  return SEVP_OK;
}

template <typename V, typename MT, bool UPDATE, bool DOTS, bool SYM>
static int launch_tile_k(sevp_ctx *ctx, const Tiling &T, const MT *mats, V *x, const V *p, V *r,
                         const V *q, V *z, int ticket_slot) {
  const size_t warps = tile_warps(T.tg);
  const bool short_tiles = sizeof(V) == 4 && T.tg.hmax <= kShortTileRows;
  const size_t smem = short_tiles ? 0 : tile_smem_per_warp(T.tg.hmax) * kTileWarps;
  auto kern = short_tiles ? k_tile_short<V, MT, UPDATE, DOTS, SYM, kShortTileRows>
                          : k_tile_apply<V, MT, UPDATE, DOTS, SYM>;
  // per instantiation and kernel choice
  static size_t set_smem[2] = {0, 0};
  static int slots[2] = {0, 0};
  int s = resident_ctas(kern, smem, set_smem[short_tiles], slots[short_tiles]);
  if (s) return s;
  const unsigned blocks = (unsigned)std::min<size_t>((warps + kTileWarps - 1) / kTileWarps,
                                                     (size_t)slots[short_tiles]);
  if constexpr (sizeof(V) == 4 && std::is_same<MT, double>::value && UPDATE && DOTS && SYM) {
    // PCG pass B with tensor-copied task stages, on the same grid
    if (short_tiles && ctx->pass_b_kernel == SEVP_PASS_B_STAGED) {
      const PassBLaunch L{T.tg, T.c, mats, x, p, r, q, z, ctx->st, ctx->partials,
                          ctx->partials_n, ctx->tickets + ticket_slot, blocks, ctx->stream};
      if (pass_b_tma_eligible(L)) {
        ProfScope ps(ctx, 0);
        const int s2 = pass_b_tma_launch(L);
        ctx->launches++;
        ctx->pass_b_used = SEVP_PASS_B_STAGED;
        return s2;
      }
    }
    ctx->pass_b_used = SEVP_PASS_B_REGISTERS;
  }
  ProfScope ps(ctx, UPDATE ? 0 : 2);
  kern<<<blocks, kTileWarps * 32, smem, ctx->stream>>>(T.tg, T.c, mats, x, p, r, q, z, ctx->st,
                                                      ctx->partials, ctx->tickets + ticket_slot);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

// Dispatch: symmetric-coefficient variant when the operator is symmetric;
// FP32 influence matrices only for FP32 vectors when the solve asks for them.
template <typename V, bool UPDATE, bool DOTS>
static int launch_tile(sevp_ctx *ctx, const Tiling &T, V *x, const V *p, V *r, const V *q, V *z,
                       int ticket_slot) {
  if constexpr (sizeof(V) == 4) {
    if (ctx->infl32_active && T.d_mats32) {
      if (ctx->sym)
        return launch_tile_k<V, float, UPDATE, DOTS, true>(ctx, T, T.d_mats32, x, p, r, q, z, ticket_slot);
      return launch_tile_k<V, float, UPDATE, DOTS, false>(ctx, T, T.d_mats32, x, p, r, q, z, ticket_slot);
    }
    if (T.d_matsmix) {
      const MixMat *mm = reinterpret_cast<const MixMat *>(T.d_matsmix);
      if (ctx->sym)
        return launch_tile_k<V, MixMat, UPDATE, DOTS, true>(ctx, T, mm, x, p, r, q, z, ticket_slot);
      return launch_tile_k<V, MixMat, UPDATE, DOTS, false>(ctx, T, mm, x, p, r, q, z, ticket_slot);
    }
  }
  if (ctx->sym)
    return launch_tile_k<V, double, UPDATE, DOTS, true>(ctx, T, T.d_mats, x, p, r, q, z, ticket_slot);
  return launch_tile_k<V, double, UPDATE, DOTS, false>(ctx, T, T.d_mats, x, p, r, q, z, ticket_slot);
}

// Tile rows the Schwarz stage kernel holds in registers.
constexpr int kCoupleMaxRows = 8;

template <typename V, typename MT, bool SYM, int HM, int MODE>
static int launch_couple_k(sevp_ctx *ctx, const Tiling &T, int xo, const MT *mats, const V *w,
                           const V *base, const V *r, V *out, SolveState *st, int ticket_slot) {
  auto kern = k_tile_couple<V, MT, SYM, HM, MODE>;
  static size_t set_smem = 0;
  static int slots = 0;
  int s = resident_ctas(kern, 0, set_smem, slots);
  if (s) return s;
  const size_t warps = tile_warps(T.tg);
  const unsigned blocks =
      (unsigned)std::min<size_t>((warps + kTileWarps - 1) / kTileWarps, (size_t)slots);
  ProfScope ps(ctx, 3);
  kern<<<blocks, kTileWarps * 32, 0, ctx->stream>>>(T.tg, xo, ctx->periodic, T.c, mats, w, base,
                                                   r, out, st, ctx->partials,
                                                   ctx->tickets + ticket_slot);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

template <typename V, typename MT, bool SYM, int MODE>
static int launch_couple_h(sevp_ctx *ctx, const Tiling &T, int xo, const MT *mats, const V *w,
                           const V *base, const V *r, V *out, SolveState *st, int ticket_slot) {
  if (T.tg.hmax <= 6)
    return launch_couple_k<V, MT, SYM, 6, MODE>(ctx, T, xo, mats, w, base, r, out, st, ticket_slot);
  return launch_couple_k<V, MT, SYM, kCoupleMaxRows, MODE>(ctx, T, xo, mats, w, base, r, out, st,
                                                           ticket_slot);
}

// One Schwarz stage on tiling T after a stage on the tiling with column
// shift xo (see k_tile_couple for MODE).
template <typename V, int MODE>
static int launch_couple(sevp_ctx *ctx, const Tiling &T, int xo, const V *w, const V *base,
                         const V *r, V *out, SolveState *st, int ticket_slot) {
  if constexpr (sizeof(V) == 4) {
    if (ctx->infl32_active && T.d_mats32) {
      if (ctx->sym)
        return launch_couple_h<V, float, true, MODE>(ctx, T, xo, T.d_mats32, w, base, r, out, st, ticket_slot);
      return launch_couple_h<V, float, false, MODE>(ctx, T, xo, T.d_mats32, w, base, r, out, st, ticket_slot);
    }
  }
  if (ctx->sym)
    return launch_couple_h<V, double, true, MODE>(ctx, T, xo, T.d_mats, w, base, r, out, st, ticket_slot);
  return launch_couple_h<V, double, false, MODE>(ctx, T, xo, T.d_mats, w, base, r, out, st, ticket_slot);
}

static bool schwarz_on(const sevp_ctx *ctx) { return ctx->schwarz_req != 0 && ctx->tb.built; }

template <typename V>
static void schwarz_bufs(sevp_ctx *ctx, V *&s1, V *&s2) {
  if constexpr (sizeof(V) == 4)
    s1 = ctx->s1_32, s2 = ctx->s2_32;
  else
    s1 = ctx->s1_64, s2 = ctx->s2_64;
}

// z = M^-1 r with the preconditioner the context is set to.  UPDATE fuses
// x += alpha p, r -= alpha q before it (PCG pass B); DOTS accumulates r.z
// and r.r and finishes the iteration on the device.  With the Schwarz
// preconditioner: z1 = M_a r, z2 = M_b (r - A z1), z = z1 + z2 + M_a (r -
// A (z1 + z2)), the residuals formed from the tile-boundary couplings.
template <typename V, bool UPDATE, bool DOTS>
static int precondition_pass(sevp_ctx *ctx, V *x, const V *p, V *r, const V *q, V *z) {
  if (!schwarz_on(ctx)) return launch_tile<V, UPDATE, DOTS>(ctx, ctx->ta, x, p, r, q, z, 4);
  V *s1, *s2;
  schwarz_bufs(ctx, s1, s2);
  int s = launch_tile<V, UPDATE, false>(ctx, ctx->ta, x, p, r, q, s1, 4);
  if (s) return s;
  SolveState *st = DOTS ? ctx->st : nullptr;
  s = launch_couple<V, 0>(ctx, ctx->tb, ctx->ta.tg.xs, s1, nullptr, nullptr, s2, st, 4);
  if (s) return s;
  if (DOTS) return launch_couple<V, 2>(ctx, ctx->ta, ctx->tb.tg.xs, s2, s1, r, z, ctx->st, 4);
  return launch_couple<V, 1>(ctx, ctx->ta, ctx->tb.tg.xs, s2, s1, nullptr, z, nullptr, 4);
}

// Folds recorded event pairs into per-class totals (synchronises the stream).
// iters >= 0: the recorded launches are one check interval of PCG
// iterations, of which iters ran; the launches after the run finished
// return at once and are not counted (the first iters pass-A and pass-B
// launches, and the first 2 iters Schwarz stages, are the ones that ran).
static void prof_collect(sevp_ctx *ctx, int iters = -1) {
  if (!ctx->ev_used) return;
  cudaStreamSynchronize(ctx->stream);
  int seen[4] = {0, 0, 0, 0};
  for (size_t k = 0; k < ctx->ev_used; ++k) {
    const int cls = ctx->ev_class[k];
    if (iters >= 0 && cls != 2 && seen[cls]++ >= (cls == 3 ? 2 * iters : iters)) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_pool[k].first, ctx->ev_pool[k].second) == cudaSuccess) {
      ctx->prof_ms[ctx->ev_class[k]] += ms;
      ctx->prof_n[ctx->ev_class[k]] += 1;
    }
  }
  ctx->ev_used = 0;
  ctx->ev_class.clear();
}

extern "C" int sevp_profile(sevp_ctx *ctx, int enable) {
  if (!ctx) return SEVP_BAD_ARG;
  prof_collect(ctx);
  ctx->prof = enable ? 1 : 0;
  for (int k = 0; k < 4; ++k) ctx->prof_ms[k] = 0.0, ctx->prof_n[k] = 0;
  return SEVP_OK;
}

extern "C" int sevp_profile_read(sevp_ctx *ctx, double *ms, long long *count) {
  if (!ctx || !ms || !count) return SEVP_BAD_ARG;
  prof_collect(ctx);
  for (int k = 0; k < 4; ++k) ms[k] = ctx->prof_ms[k], count[k] = ctx->prof_n[k];
  return SEVP_OK;
}

static void free_work(sevp_ctx *ctx) {
  void *ptrs[] = {ctx->r64, ctx->z64, ctx->p64[0], ctx->p64[1], ctx->q64, ctx->x64s, ctx->r32,
                  ctx->z32, ctx->p32[0], ctx->p32[1], ctx->q32, ctx->d32, ctx->bh, ctx->xh,
                  ctx->e1h, ctx->e2h, ctx->st, ctx->partials, ctx->tickets,
                  ctx->step_buf[0], ctx->step_buf[1], ctx->step_buf[2], ctx->bstage[0],
                  ctx->bstage[1], ctx->nn_avg,
                  ctx->s1_64, ctx->s2_64, ctx->s1_32, ctx->s2_32, ctx->hist};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  ctx->ta.release();
  ctx->tb.release();
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  for (cudaEvent_t e : {ctx->ev_in[0], ctx->ev_in[1], ctx->ev_out[0], ctx->ev_out[1],
                        ctx->ev_out[2], ctx->ev_solved})
    if (e) cudaEventDestroy(e);
  for (cudaStream_t st : {ctx->cp_in, ctx->cp_out})
    if (st) cudaStreamDestroy(st);
  for (auto &pr : ctx->ev_pool) cudaEventDestroy(pr.first), cudaEventDestroy(pr.second);
  ctx->ev_pool.clear();
}

extern "C" int sevp_create(sevp_ctx **out, int nx, int ny, int periodic, void *stream) {
  if (!out || nx < 1 || ny < 1) return SEVP_BAD_ARG;
  *out = nullptr;
  sevp_ctx *ctx = new sevp_ctx();
  ctx->nx = nx, ctx->ny = ny, ctx->periodic = periodic ? 1 : 0;
  ctx->stream = (cudaStream_t)stream;
  ctx->n = (size_t)nx * ny;
  cudaGetDevice(&ctx->device);
  size_t n = ctx->n;
  auto fail = [&](cudaError_t e, const char *w) {
    sevp_internal_set_error(e, w, __FILE__, __LINE__);
    free_work(ctx);
    delete ctx;
    return SEVP_CUDA_ERROR;
  };
  cudaError_t e;
#define ALLOC(ptr, bytes)                                          \
  e = cudaMalloc((void **)&(ptr), (bytes));                        \
  if (e != cudaSuccess) return fail(e, "cudaMalloc " #ptr);        \
  e = cudaMemsetAsync((ptr), 0, (bytes), ctx->stream);             \
  if (e != cudaSuccess) return fail(e, "cudaMemset " #ptr);
  ALLOC(ctx->r64, n * 8);
  ALLOC(ctx->z64, n * 8);
  ALLOC(ctx->p64[0], n * 8);
  ALLOC(ctx->p64[1], n * 8);
  ALLOC(ctx->q64, n * 8);
  ALLOC(ctx->x64s, n * 8);
  ALLOC(ctx->r32, n * 4);
  ALLOC(ctx->z32, n * 4);
  ALLOC(ctx->p32[0], n * 4);
  ALLOC(ctx->p32[1], n * 4);
  ALLOC(ctx->q32, n * 4);
  ALLOC(ctx->d32, n * 4);
  ALLOC(ctx->st, sizeof(SolveState));
  ALLOC(ctx->tickets, 16 * sizeof(unsigned));
  // partial sums: enough for the larger of the stencil and tile grids
  // stencil grid: ceil(nx / 256) x ceil(ny / rpw), rpw >= 8
  size_t sgrid = (size_t)ceil_div(ceil_div(nx, kStencilCols), kStencilThreads / 32) * ceil_div(ny, 8);
  size_t tgrid = (size_t)ceil_div(nx, 1) * ceil_div(ny, 1) / (kTileWarps) + 1024;
  ctx->partials_n = std::max(sgrid, tgrid) * 2 + 64;
  ALLOC(ctx->partials, ctx->partials_n * 8);
#undef ALLOC
  e = cudaMallocHost((void **)&ctx->h_st, sizeof(SolveState));
  if (e != cudaSuccess) return fail(e, "cudaMallocHost");
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(e, "sync");
  *out = ctx;
  return SEVP_OK;
}

extern "C" int sevp_destroy(sevp_ctx *ctx) {
  if (!ctx) return SEVP_OK;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->inner_graph) cudaGraphExecDestroy(ctx->inner_graph);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  free_work(ctx);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  delete ctx;
  return SEVP_OK;
}

extern "C" long long sevp_kernel_launches(const sevp_ctx *ctx) { return ctx ? ctx->launches : 0; }

extern "C" int sevp_operator_symmetric(const sevp_ctx *ctx) { return ctx ? ctx->sym : 0; }

// Drops the captured inner-loop graph (the operator or buffers changed).
static void drop_inner_graph(sevp_ctx *ctx) {
  if (ctx->inner_graph) cudaGraphExecDestroy(ctx->inner_graph);
  ctx->inner_graph = nullptr;
  ctx->inner_graph_ce = 0;
}

extern "C" int sevp_set_graphs(sevp_ctx *ctx, int enable) {
  if (!ctx) return SEVP_BAD_ARG;
  ctx->use_graphs = enable ? 1 : 0;
  if (!enable) drop_inner_graph(ctx);
  return SEVP_OK;
}

extern "C" int sevp_set_pass_a_kernel(sevp_ctx *ctx, int kind) {
  if (!ctx || (kind != SEVP_PASS_A_TILES && kind != SEVP_PASS_A_COLUMNS)) return SEVP_BAD_ARG;
  ctx->pass_a_kernel = kind;
  drop_inner_graph(ctx);
  return SEVP_OK;
}

extern "C" int sevp_set_pass_b_kernel(sevp_ctx *ctx, int kind) {
  if (!ctx || (kind != SEVP_PASS_B_REGISTERS && kind != SEVP_PASS_B_STAGED)) return SEVP_BAD_ARG;
  ctx->pass_b_kernel = kind;
  drop_inner_graph(ctx);
  return SEVP_OK;
}

extern "C" int sevp_set_resume_check(sevp_ctx *ctx, double max_rel_dev) {
  if (!ctx || !(max_rel_dev == max_rel_dev)) return SEVP_BAD_ARG;
  ctx->resume_dev = max_rel_dev;
  return SEVP_OK;
}

extern "C" int sevp_pass_b_kernel_used(const sevp_ctx *ctx) { return ctx ? ctx->pass_b_used : -1; }

extern "C" int sevp_set_full_coefficients(sevp_ctx *ctx, int force) {
  if (!ctx) return SEVP_BAD_ARG;
  ctx->force_full = force ? 1 : 0;
  if (force) ctx->sym = 0;
  drop_inner_graph(ctx);
  return SEVP_OK;
}

extern "C" int sevp_tile_layout(const sevp_ctx *ctx, int *tiles_x, int *tiles_y, int *nb_per_tile) {
  if (!ctx || !ctx->have_op || !tiles_x || !tiles_y) return SEVP_BAD_ARG;
  *tiles_x = ctx->ta.tg.tx;
  *tiles_y = ctx->ta.tg.ty;
  if (nb_per_tile)
    for (size_t t = 0; t < ctx->ta.tile_nb.size(); ++t) nb_per_tile[t] = ctx->ta.tile_nb[t];
  return SEVP_OK;
}
extern "C" long long sevp_influence_bytes(const sevp_ctx *ctx) {
  return ctx ? ctx->ta.mats_elems * 8 : 0;
}

// Builds tile set T with column shift xs from the context's tiling request:
// sub-block heights per tile (explicit, per tile row, or from the marching
// growth bound measured on the device), warp-group counts, the influence
// data layout, and the influence data (k_tile_precompute).
static int build_tiling(sevp_ctx *ctx, Tiling &T, int xs) {
  const sevp_tiling *tl = &ctx->treq;
  const int tm = tl->tile_m, th = tl->tile_h;
  T.release();
  TileGeom &tg = T.tg;
  tg = TileGeom{};
  tg.nx = ctx->nx, tg.ny = ctx->ny, tg.tm = tm, tg.th = th;
  tg.tx = ceil_div(ctx->nx, tm);
  tg.ty = ceil_div(ctx->ny, th);
  tg.wseg = tm <= 8 ? 8 : (tm <= 16 ? 16 : 32);
  tg.tpw = 32 / tg.wseg;
  tg.txg = ceil_div(tg.tx, tg.tpw);
  tg.hmax = th;
  tg.xs = xs;
  T.c = ctx->c;
  if (xs != 0 && !ctx->periodic) {
    // closed grid: the shifted tiling's wrapped tile must not couple
    // column nx-1 to column 0
    const size_t bytes = ctx->n * sizeof(float);
    SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_al, bytes));
    SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_ar, bytes));
    SEVP_CUDA_TRY(cudaMemcpyAsync(T.d_al, ctx->c.al, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    SEVP_CUDA_TRY(cudaMemcpyAsync(T.d_ar, ctx->c.ar, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    const size_t pitch = (size_t)ctx->nx * sizeof(float);
    SEVP_CUDA_TRY(cudaMemset2DAsync(T.d_al, pitch, 0, sizeof(float), ctx->ny, ctx->stream));
    SEVP_CUDA_TRY(cudaMemset2DAsync(T.d_ar + (ctx->nx - 1), pitch, 0, sizeof(float), ctx->ny,
                                    ctx->stream));
    T.c.al = T.d_al;
    T.c.ar = T.d_ar;
  }
  // sub-block height per tile
  const int ntiles = tg.tx * tg.ty;
  std::vector<int> s_tile(ntiles, std::max(1, tl->sub_rows));
  if (!ctx->treq_tiles.empty()) {
    // given per tile of the unshifted tiling: a shifted tile takes the
    // smallest height of the unshifted tiles it overlaps
    for (int t = 0; t < ntiles; ++t) {
      const int a = t % tg.tx, b = t / tg.tx;
      int v = INT32_MAX;
      for (int n = 0; n < tile_width(tg, a); ++n)
        v = std::min(v, ctx->treq_tiles[(size_t)b * tg.tx + tile_col(tg, a, n) / tm]);
      s_tile[t] = v;
    }
  } else if (!ctx->treq_rows.empty()) {
    for (int t = 0; t < ntiles; ++t) s_tile[t] = ctx->treq_rows[t / tg.tx];
  } else if (tl->growth_limit > 1.0) {
    int *d_s = nullptr;
    SEVP_CUDA_TRY(cudaMalloc((void **)&d_s, sizeof(int) * ntiles));
    k_tile_growth<<<(ntiles + 7) / 8, 256, 0, ctx->stream>>>(tg, T.c, log(tl->growth_limit), d_s);
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s_tile.data(), d_s, sizeof(int) * ntiles, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_s);
    if (e != cudaSuccess) {
      sevp_internal_set_error(e, "tile growth", __FILE__, __LINE__);
      return SEVP_CUDA_ERROR;
    }
  }
  T.grp_nb.assign((size_t)tg.ty * tg.txg, 1);
  for (int t = 0; t < ntiles; ++t) {
    const int a = t % tg.tx, b = t / tg.tx;
    if (s_tile[t] < 1) return SEVP_BAD_ARG;
    const int nb = ceil_div(tile_height(tg, b), std::min(s_tile[t], tile_height(tg, b)));
    int &g = T.grp_nb[(size_t)b * tg.txg + a / tg.tpw];
    g = std::max(g, nb);
  }
  int nbmax = 1;
  for (int v : T.grp_nb) nbmax = std::max(nbmax, v);
  tg.nbmax = nbmax;
  T.tile_nb.assign(ntiles, 1);
  std::vector<long long> moff((size_t)ntiles);
  long long off = 0;
  for (int b = 0; b < tg.ty; ++b)
    for (int a = 0; a < tg.tx; ++a) {
      const int mw = tile_width(tg, a), nb = T.grp_nb[(size_t)b * tg.txg + a / tg.tpw];
      T.tile_nb[(size_t)b * tg.tx + a] = nb;
      moff[(size_t)b * tg.tx + a] = off;
      off += (long long)(2 * nb - 1) * mw * mw;
      off = (off + 1) & ~1LL;  // 16-byte aligned start for every tile
    }
  T.mats_elems = off;
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_grp_nb, sizeof(int) * T.grp_nb.size()));
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_moff, sizeof(long long) * moff.size()));
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_mats, sizeof(double) * std::max<long long>(off, 1)));
  SEVP_CUDA_TRY(cudaMemcpyAsync(T.d_grp_nb, T.grp_nb.data(), sizeof(int) * T.grp_nb.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
  SEVP_CUDA_TRY(cudaMemcpyAsync(T.d_moff, moff.data(), sizeof(long long) * moff.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
  tg.grp_nb = T.d_grp_nb;
  tg.moff = T.d_moff;
  // partial-sum capacity for the tile grid
  size_t tblocks = (tile_warps(tg) + kTileWarps - 1) / kTileWarps;
  if (tblocks * 2 + 64 > ctx->partials_n) {
    SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->partials);
    ctx->partials_n = tblocks * 2 + 64;
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->partials, ctx->partials_n * 8));
  }
  // tile-apply shared memory must fit
  if (tile_smem_per_warp(tg.hmax) * kTileWarps > 220 * 1024) return SEVP_BAD_ARG;
  // precompute
  int *d_status = nullptr;
  SEVP_CUDA_TRY(cudaMalloc((void **)&d_status, sizeof(int)));
  SEVP_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), ctx->stream));
  size_t psmem = (size_t)5 * tg.hmax * 32 * sizeof(float) + (size_t)(32 * 32 * 3 + 32 * 64 + 32) * 8;
  SEVP_CUDA_TRY(cudaFuncSetAttribute(k_tile_precompute, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)psmem));
  k_tile_precompute<<<tg.ty * tg.tx, 1024, psmem, ctx->stream>>>(tg, T.c, T.d_mats, d_status);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  int h_status = 0;
  SEVP_CUDA_TRY(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  cudaFree(d_status);
  if (h_status) return SEVP_SINGULAR;
  T.built = true;
  return SEVP_OK;
}

// Per-group FP32 influence data of tiling T for ctx->mix_limit (see
// sevp_set_influence_fp32): a group reads FP32 matrices when every tile in
// it has z^s <= mix_limit, s its sub-block height and z its row growth
// (k_tile_growth).  Drops the previous copy first; nothing more when off.
static int build_mix(sevp_ctx *ctx, Tiling &T) {
  if (T.d_matsmix) cudaFree(T.d_matsmix);
  if (T.d_grp_f32) cudaFree(T.d_grp_f32);
  T.d_matsmix = nullptr;
  T.d_grp_f32 = nullptr;
  T.tg.grp_f32 = nullptr;
  T.f32_groups = 0;
  T.mix_bytes_per_pass = 0;
  if (ctx->mix_limit <= 1.0 || !T.built) return SEVP_OK;
  TileGeom &tg = T.tg;
  const int ntiles = tg.tx * tg.ty;
  std::vector<float> lz((size_t)ntiles, 0.f);
  {
    int *d_s = nullptr;
    float *d_lz = nullptr;
    SEVP_CUDA_TRY(cudaMalloc((void **)&d_s, sizeof(int) * ntiles));
    cudaError_t e = cudaMalloc((void **)&d_lz, sizeof(float) * ntiles);
    if (e == cudaSuccess) {
      k_tile_growth<<<(ntiles + 7) / 8, 256, 0, ctx->stream>>>(tg, T.c, log(2.0), d_s, d_lz);
      ctx->launches++;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(lz.data(), d_lz, sizeof(float) * ntiles, cudaMemcpyDeviceToHost,
                          ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_s);
    if (d_lz) cudaFree(d_lz);
    if (e != cudaSuccess) {
      sevp_internal_set_error(e, "influence precision", __FILE__, __LINE__);
      return SEVP_CUDA_ERROR;
    }
  }
  const double lim = log(ctx->mix_limit);
  std::vector<unsigned char> f32(T.grp_nb.size(), 1);
  for (int t = 0; t < ntiles; ++t) {
    const int a = t % tg.tx, b = t / tg.tx;
    const size_t g = (size_t)b * tg.txg + a / tg.tpw;
    const int hs = ceil_div(tile_height(tg, b), T.grp_nb[g]);
    if (!((double)hs * (double)lz[t] <= lim)) f32[g] = 0;
  }
  long long bytes = 0;
  for (int t = 0; t < ntiles; ++t) {
    const int a = t % tg.tx, b = t / tg.tx;
    const size_t g = (size_t)b * tg.txg + a / tg.tpw;
    const long long mw = tile_width(tg, a);
    bytes += (2LL * T.grp_nb[g] - 1) * mw * mw * (f32[g] ? 4 : 8);
  }
  for (unsigned char v : f32) T.f32_groups += v;
  T.mix_bytes_per_pass = bytes;
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_grp_f32, f32.size()));
  SEVP_CUDA_TRY(cudaMemcpyAsync(T.d_grp_f32, f32.data(), f32.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
  const size_t n = (size_t)std::max<long long>(T.mats_elems, 1);
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_matsmix, n * sizeof(double)));
  SEVP_CUDA_TRY(cudaMemsetAsync(T.d_matsmix, 0, n * sizeof(double), ctx->stream));
  tg.grp_f32 = T.d_grp_f32;
  k_mix_influence<<<ntiles, 256, 0, ctx->stream>>>(tg, T.d_mats, T.d_matsmix);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  // the host vector f32 must outlive the copy above
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return SEVP_OK;
}

// Column cuts of the tiling with shift xs: the first column of every tile.
static std::vector<char> tiling_cuts(const sevp_ctx *ctx, int xs) {
  std::vector<char> cut((size_t)ctx->nx, 0);
  const int tm = ctx->treq.tile_m;
  for (int a = 0; a < ceil_div(ctx->nx, tm); ++a) cut[(size_t)((a * tm + xs) % ctx->nx)] = 1;
  return cut;
}

// Column shift of the second Schwarz tiling: the requested one, or for
// shift < 0 the one nearest tile_m / 2 whose tile edges all lie strictly
// inside tiles of the unshifted tiling (and the other way round), so that
// every coupling a stage needs is between two lanes of one tile.  0: none.
static int schwarz_shift(const sevp_ctx *ctx, int req) {
  const int tm = ctx->treq.tile_m;
  if (tm < 2 || ctx->nx < 2) return 0;
  const std::vector<char> ca = tiling_cuts(ctx, 0);
  auto ok = [&](int xs) {
    if (xs < 1 || xs >= tm || xs >= ctx->nx) return false;
    const std::vector<char> cb = tiling_cuts(ctx, xs);
    for (int c = 0; c < ctx->nx; ++c)
      if (ca[c] && cb[c]) return false;
    return true;
  };
  if (req > 0) return ok(req) ? req : 0;
  for (int d = 0; d < tm; ++d) {
    if (ok(tm / 2 - d)) return tm / 2 - d;
    if (ok(tm / 2 + d)) return tm / 2 + d;
  }
  return 0;
}

// (Re)builds the second tiling and the Schwarz work vectors.
static int build_schwarz(sevp_ctx *ctx) {
  ctx->tb.release();
  if (!ctx->schwarz_req) return SEVP_OK;
  if (ctx->treq.tile_h > kCoupleMaxRows) return SEVP_BAD_ARG;
  const int xs = schwarz_shift(ctx, ctx->schwarz_req);
  if (!xs) return SEVP_BAD_ARG;
  const size_t n = ctx->n;
  if (!ctx->s1_64) {
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->s1_64, n * 8));
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->s2_64, n * 8));
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->s1_32, n * 4));
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->s2_32, n * 4));
  }
  int s = build_tiling(ctx, ctx->tb, xs);
  if (s) ctx->tb.release();
  return s;
}

// Exact symmetry test of five planes on the device (k_check_symmetry).
static int check_symmetry(sevp_ctx *ctx, const Coeffs &c, int *asym) {
  int *d_asym = nullptr;
  SEVP_CUDA_TRY(cudaMalloc((void **)&d_asym, sizeof(int)));
  SEVP_CUDA_TRY(cudaMemsetAsync(d_asym, 0, sizeof(int), ctx->stream));
  const size_t n = (size_t)ctx->nx * ctx->ny;
  k_check_symmetry<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 32), 256, 0, ctx->stream>>>(
      c, ctx->nx, ctx->ny, ctx->periodic, d_asym);
  ctx->launches++;
  *asym = 1;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(asym, d_asym, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_asym);
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "symmetry check", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  return SEVP_OK;
}

extern "C" int sevp_set_residual_operator(sevp_ctx *ctx, const float *al, const float *ab,
                                          const float *ac, const float *ar, const float *at,
                                          const double *row_weight) {
  if (!ctx) return SEVP_BAD_ARG;
  ctx->have_res = false;
  ctx->roww = nullptr;
  if (!al) return SEVP_OK;
  if (!ab || !ac || !ar || !at) return SEVP_BAD_ARG;
  ctx->cres = Coeffs{al, ab, ac, ar, at};
  int asym = 1;
  int s = check_symmetry(ctx, ctx->cres, &asym);
  if (s) return s;
  ctx->res_sym = asym ? 0 : 1;
  ctx->roww = row_weight;
  ctx->have_res = true;
  return SEVP_OK;
}

extern "C" int sevp_set_operator(sevp_ctx *ctx, const float *al, const float *ab, const float *ac,
                                 const float *ar, const float *at, const sevp_tiling *tl) {
  if (!ctx || !al || !ab || !ac || !ar || !at || !tl) return SEVP_BAD_ARG;
  drop_inner_graph(ctx);
  const int tm = tl->tile_m, th = tl->tile_h;
  if (tm < 1 || tm > 32 || th < 1 || th > 32 || tl->sub_rows < 1) return SEVP_BAD_ARG;
  ctx->have_op = false;
  ctx->c = Coeffs{al, ab, ac, ar, at};
  {
    int h_asym = 1;
    int s = check_symmetry(ctx, ctx->c, &h_asym);
    if (s) return s;
    ctx->sym = (!h_asym && !ctx->force_full) ? 1 : 0;
    ctx->asym = h_asym ? 1 : 0;
    if (h_asym)
      sevp_internal_set_message(
          "sevp_set_operator: the operator is not symmetric; apply and precondition work, "
          "sevp_solve returns SEVP_NONSYMMETRIC");
  }
  // keep the request (the second tiling is built from it later too)
  ctx->treq = *tl;
  const int tx = ceil_div(ctx->nx, tm), ty = ceil_div(ctx->ny, th);
  ctx->treq_tiles.clear();
  ctx->treq_rows.clear();
  if (tl->sub_rows_by_tile)
    ctx->treq_tiles.assign(tl->sub_rows_by_tile, tl->sub_rows_by_tile + (size_t)tx * ty);
  else if (tl->sub_rows_by_tile_row)
    ctx->treq_rows.assign(tl->sub_rows_by_tile_row, tl->sub_rows_by_tile_row + ty);
  ctx->treq.sub_rows_by_tile = nullptr;
  ctx->treq.sub_rows_by_tile_row = nullptr;
  int s = build_tiling(ctx, ctx->ta, 0);
  if (s) return s;
  s = build_mix(ctx, ctx->ta);
  if (s) return s;
  ctx->have_op = true;
  s = build_schwarz(ctx);
  if (s) ctx->schwarz_req = 0;  // the block-Jacobi operator stays usable
  return s;
}

extern "C" int sevp_set_influence_fp32(sevp_ctx *ctx, double growth_limit) {
  if (!ctx || !(growth_limit == growth_limit)) return SEVP_BAD_ARG;
  drop_inner_graph(ctx);
  ctx->mix_limit = growth_limit > 1.0 ? growth_limit : 0.0;
  return ctx->have_op ? build_mix(ctx, ctx->ta) : SEVP_OK;
}

extern "C" int sevp_influence_fp32_groups(const sevp_ctx *ctx, int *fp32_groups, int *groups,
                                          long long *bytes_per_pass) {
  if (!ctx) return SEVP_BAD_ARG;
  const Tiling &T = ctx->ta;
  if (fp32_groups) *fp32_groups = T.d_matsmix ? T.f32_groups : 0;
  if (groups) *groups = (int)T.grp_nb.size();
  if (bytes_per_pass)
    *bytes_per_pass = T.d_matsmix ? T.mix_bytes_per_pass : T.mats_elems * (long long)sizeof(double);
  return SEVP_OK;
}

extern "C" int sevp_set_schwarz(sevp_ctx *ctx, int shift) {
  if (!ctx || !ctx->have_op) return SEVP_BAD_ARG;
  drop_inner_graph(ctx);
  ctx->schwarz_req = shift;
  int s = build_schwarz(ctx);
  if (s) ctx->schwarz_req = 0;
  return s;
}

extern "C" int sevp_record_coefficients(sevp_ctx *ctx, int cap) {
  if (!ctx || cap < 0) return SEVP_BAD_ARG;
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->hist) cudaFree(ctx->hist), ctx->hist = nullptr;
  ctx->hist_cap = 0;
  if (cap > 0) {
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->hist, sizeof(double) * 2 * (size_t)cap));
    SEVP_CUDA_TRY(cudaMemsetAsync(ctx->hist, 0, sizeof(double) * 2 * (size_t)cap, ctx->stream));
    ctx->hist_cap = cap;
  }
  return SEVP_OK;
}

extern "C" int sevp_read_coefficients(sevp_ctx *ctx, double *alpha, double *beta, int cap,
                                      int *count) {
  if (!ctx || !alpha || !beta || !count || cap < 0) return SEVP_BAD_ARG;
  *count = 0;
  if (!ctx->hist) return SEVP_OK;
  const int n = std::min(cap, ctx->hist_cap);
  std::vector<double> h((size_t)2 * std::max(n, 1));
  SEVP_CUDA_TRY(cudaMemcpyAsync(h.data(), ctx->hist, sizeof(double) * 2 * (size_t)n,
                                cudaMemcpyDeviceToHost, ctx->stream));
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  int last = 0;
  for (int j = 0; j < n; ++j) {
    alpha[j] = h[2 * j];
    beta[j] = h[2 * j + 1];
    if (alpha[j] != 0.0) last = j + 1;
  }
  *count = last;
  return SEVP_OK;
}

extern "C" int sevp_schwarz_shift(const sevp_ctx *ctx) {
  return (ctx && schwarz_on(ctx)) ? ctx->tb.tg.xs : 0;
}

extern "C" long long sevp_schwarz_influence_bytes(const sevp_ctx *ctx) {
  return (ctx && schwarz_on(ctx)) ? ctx->tb.mats_elems * 8 : 0;
}

extern "C" int sevp_apply(sevp_ctx *ctx, const double *x, double *y) {
  if (!ctx || !ctx->have_op || !x || !y) return SEVP_BAD_ARG;
  OpApply<double> op{x, y};
  return launch_stencil(ctx, op, 0);
}

extern "C" int sevp_precondition(sevp_ctx *ctx, const double *r, double *z) {
  if (!ctx || !ctx->have_op || !r || !z) return SEVP_BAD_ARG;
  return precondition_pass<double, false, false>(ctx, nullptr, nullptr, const_cast<double *>(r),
                                                 nullptr, z);
}

extern "C" int sevp_precondition_f32(sevp_ctx *ctx, const float *r, float *z) {
  if (!ctx || !ctx->have_op || !r || !z) return SEVP_BAD_ARG;
  return precondition_pass<float, false, false>(ctx, nullptr, nullptr, const_cast<float *>(r),
                                                nullptr, z);
}

static int read_state(sevp_ctx *ctx) {
  SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(SolveState), cudaMemcpyDeviceToHost,
                                ctx->stream));
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return SEVP_OK;
}

// Residual pass: xout = x + d; r = W (b - A xout) with the residual
// operator and its row weights; the norms into the state (OpResidual).
template <typename R>
static int launch_residual(sevp_ctx *ctx, const double *x, const float *d, double *xout,
                           const double *b, R *r, int set_inner, double tol2,
                           double outer2 = 0.0, int abs_mode = 0) {
  OpResidual<R> op{x, d, xout, b, r, ctx->st, tol2, outer2, set_inner, ctx->resume_dev,
                   ctx->have_res ? ctx->roww : nullptr, abs_mode};
  if (ctx->have_res) return launch_stencil_c(ctx, op, 2, ctx->cres, ctx->res_sym);
  return launch_stencil(ctx, op, 2);
}

__global__ void k_state_init(SolveState *st, double tol2, int max_iter, double *hist = nullptr,
                             int hist_cap = 0) {
  SolveState s{};
  s.tol2 = tol2;
  s.max_iter = max_iter;
  s.hist = hist;
  s.hist_cap = hist_cap;
  s.status = SEVP_OK;
  *st = s;
}

// State for a residual replacement that keeps the search direction: as
// k_state_init, but the last two r.z of the stopped run stay for the next
// beta.
__global__ void k_state_keep(SolveState *st, double tol2, int max_iter) {
  SolveState s{};
  s.tol2 = tol2;
  s.max_iter = max_iter;
  s.status = SEVP_OK;
  s.rz = st->rz;
  s.rz_next = st->rz_next;
  s.keep_dir = 1;
  *st = s;
}

// State for a residual replacement that continues the Chebyshev
// recurrence: as k_state_init, with the Chebyshev scalars kept and the
// launch count at one, so the next launch takes the recurrence's next step
// on the replaced residual instead of starting over.
__global__ void k_state_keep_cheb(SolveState *st, double tol2, int max_iter) {
  SolveState s{};
  s.tol2 = tol2;
  s.max_iter = max_iter;
  s.status = SEVP_OK;
  s.cheb_theta = st->cheb_theta;
  s.cheb_delta = st->cheb_delta;
  s.cheb_sigma = st->cheb_sigma;
  s.cheb_rho = st->cheb_rho;
  s.iter = 1;
  *st = s;
}

// Starts an FP64 PCG run from the residual pass's norms: the recursive
// (row-scaled) residual must fall by the factor the outer test still needs,
// target / ||b - A x||^2 with target = tol^2 ||b||^2 (relative test) or
// tol^2 (absolute test).
__global__ void k_state_from_residual(SolveState *st, double tol2, int abs_mode) {
  const double target = abs_mode ? tol2 : tol2 * st->bb64;
  st->tol2 = st->rr64 > 0.0 ? target / st->rr64 : tol2;
  st->bb = st->rr64w;
  st->rr = st->rr64w;
  st->iter = 0;
  st->done = 0;
  st->beta = 0.0;
}

// The outer stopping test on the FP64 residual pass's norms.
static bool outer_converged(const SolveState *h, const sevp_solve_opts *o) {
  if (o->tol_abs) return sqrt(h->rr64) <= o->tol;
  return h->bb64 == 0.0 || sqrt(h->rr64 / h->bb64) <= o->tol;
}

// Runs check intervals of an inner iteration until the device state says
// done.  interval(cur) issues one interval's launches with the ping-pong
// buffer index cur (and flips it per iteration); with graphs on, one
// interval is captured once per key (buffers, influence precision, method)
// and replayed, which needs an even interval so that the buffers return to
// the same roles.  launches: kernel launches per interval.
template <class Interval>
static int graph_loop(sevp_ctx *ctx, bool graph, const void *const (&key)[5], int check_every,
                      int launches, Interval &&interval, bool pcg_iters = false) {
  int cur = 0;
  graph = graph && ctx->use_graphs && !ctx->prof && check_every % 2 == 0;
  if (graph && !(ctx->inner_graph && ctx->inner_graph_ce == check_every &&
                 std::equal(key, key + 5, ctx->inner_graph_key))) {
    drop_inner_graph(ctx);
    if (!ctx->cap_stream)
      SEVP_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
    cudaStream_t run = ctx->stream;
    const long long l0 = ctx->launches;
    ctx->stream = ctx->cap_stream;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal);
    int s = SEVP_OK;
    if (e == cudaSuccess) {
      int c2 = 0;
      s = interval(c2);
      e = cudaStreamEndCapture(ctx->cap_stream, &g);
    }
    ctx->stream = run;
    ctx->launches = l0;
    if (s) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->inner_graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ctx->inner_graph = nullptr;
      sevp_internal_set_error(e, "capture of the inner iteration loop", __FILE__, __LINE__);
      return SEVP_CUDA_ERROR;
    }
    ctx->inner_graph_ce = check_every;
    std::copy(key, key + 5, ctx->inner_graph_key);
  }
  int it0 = 0;  // the run's iterations before this interval (a run starts at 0)
  for (;;) {
    if (graph) {
      SEVP_CUDA_TRY(cudaGraphLaunch(ctx->inner_graph, ctx->stream));
      ctx->launches += launches;
    } else {
      int s = interval(cur);
      if (s) return s;
    }
    int s = read_state(ctx);
    if (s) return s;
    prof_collect(ctx, pcg_iters ? std::max(ctx->h_st->iter - it0, 0) : -1);
    it0 = ctx->h_st->iter;
    if (ctx->h_st->done) break;
  }
  return SEVP_OK;
}

// PCG pass A: the tile kernel of stencil_tma.cu where the context chose it
// and the grid allows it, else the column-walking k_stencil.
template <typename V>
static int launch_pass_a(sevp_ctx *ctx, const OpPassA<V> &op) {
  if (ctx->pass_a_kernel == SEVP_PASS_A_TILES) {
    PassALaunch<V> L{GridDims{ctx->nx, ctx->ny, ctx->periodic},
                     ctx->c,
                     ctx->sym,
                     op.z,
                     op.pold,
                     op.pnew,
                     op.q,
                     ctx->st,
                     ctx->partials,
                     ctx->partials_n,
                     ctx->tickets + 3,
                     ctx->stream};
    if (pass_a_tma_eligible(L)) {
      ProfScope ps(ctx, 1);
      const int s = pass_a_tma_launch(L);
      ctx->launches++;
      return s;
    }
  }
  return launch_stencil(ctx, op, 3);
}

// Runs PCG iterations on vectors of type V until the device state says done.
// x, r hold the iterate and residual; the first z = M^{-1} r must already be
// in place (with rz, beta = 0 set).  Returns iterations done.
template <typename V>
static int pcg_loop(sevp_ctx *ctx, V *x, V *r, V *z, V *p0, V *p1, V *q, int check_every,
                    int *iters_out) {
  V *pp[2] = {p0, p1};
  auto interval = [&](int &cur) -> int {  // check_every iterations of passes A and B
    for (int k = 0; k < check_every; ++k) {
      OpPassA<V> op{z, pp[cur], pp[cur ^ 1], q, ctx->st};
      int s = launch_pass_a(ctx, op);
      if (s) return s;
      s = precondition_pass<V, true, true>(ctx, x, pp[cur ^ 1], r, q, z);
      if (s) return s;
      cur ^= 1;
    }
    return SEVP_OK;
  };
  // FP32 inner loop: one graph replay per check interval
  const void *const key[5] = {(const void *)x, (const void *)p0,
                              ctx->infl32_active ? (const void *)ctx->ta.d_mats32
                                                 : (const void *)ctx->ta.d_matsmix,
                              (const void *)(schwarz_on(ctx) ? ctx->tb.d_mats : nullptr),
                              (const void *)(uintptr_t)SEVP_METHOD_PCG};
  int s = graph_loop(ctx, sizeof(V) == 4, key, check_every,
                     (schwarz_on(ctx) ? 4 : 2) * check_every, interval, true);
  if (s) return s;
  *iters_out = ctx->h_st->iter;
  return SEVP_OK;
}

// One Chebyshev launch (fused.cu) on the block-Jacobi tiling.
static int launch_cheb_k(sevp_ctx *ctx, const float *din, float *dout, float *x, float *r) {
  const Tiling &T = ctx->ta;
  const bool m32 = ctx->infl32_active && T.d_mats32;
  const bool mix = !m32 && T.d_matsmix;
  ChebLaunch<float> L{ctx->sym, m32 ? 1 : (mix ? 2 : 0), T.tg, T.c, ctx->periodic,
                      m32 ? (const void *)T.d_mats32
                          : (mix ? (const void *)T.d_matsmix : (const void *)T.d_mats),
                      din, dout, x, r,
                      ctx->st, ctx->partials, ctx->tickets + 7, ctx->stream};
  ProfScope ps(ctx, 0);
  int s = cheb_launch<float>(L);
  ctx->launches++;
  return s;
}

__global__ void k_state_cheb(SolveState *st, double theta, double delta) {
  st->cheb_theta = theta;
  st->cheb_delta = delta;
  st->cheb_sigma = theta / delta;
  st->cheb_rho = delta / theta;
}

// Inner FP32 solve A d = r32 from d = 0 (d32 zeroed by the caller) with the
// one-launch Chebyshev iteration: directions in p32[0], p32[1], x = d32, r =
// r32 in place.  cont: continue the recurrence of the previous inner solve
// (its scalars kept by k_state_keep_cheb, its last direction in p32[0])
// instead of starting it.
static int cheb_inner(sevp_ctx *ctx, int check_every, int *iters_out, bool cont) {
  const double lmin = ctx->cheb_lmin, lmax = ctx->cheb_lmax;
  if (!cont) {
    k_state_cheb<<<1, 1, 0, ctx->stream>>>(ctx->st, 0.5 * (lmax + lmin), 0.5 * (lmax - lmin));
    ctx->launches++;
    SEVP_CUDA_TRY(cudaGetLastError());
  }
  float *db[2] = {ctx->p32[0], ctx->p32[1]};
  auto interval = [&](int &cur) -> int {
    for (int k = 0; k < check_every; ++k) {
      int s = launch_cheb_k(ctx, db[cur], db[cur ^ 1], ctx->d32, ctx->r32);
      if (s) return s;
      cur ^= 1;
    }
    return SEVP_OK;
  };
  const void *const key[5] = {(const void *)ctx->d32, (const void *)ctx->p32[0],
                              ctx->infl32_active ? (const void *)ctx->ta.d_mats32
                                                 : (const void *)ctx->ta.d_matsmix,
                              nullptr, (const void *)(uintptr_t)SEVP_METHOD_CHEB};
  int s = graph_loop(ctx, true, key, check_every, check_every, interval);
  if (s) return s;
  *iters_out = ctx->h_st->iter - (cont ? 1 : 0);
  return SEVP_OK;
}

static int solve_fp64(sevp_ctx *ctx, const double *b, double *x, const sevp_solve_opts *o,
                      sevp_report *rep) {
  const double tol2 = o->tol * o->tol;
  int total = 0, status = SEVP_OK;
  for (int restart = 0; restart < 6; ++restart) {
    // the coefficients of the first PCG run are recorded when asked for
    k_state_init<<<1, 1, 0, ctx->stream>>>(ctx->st, tol2, std::max(o->max_iter - total, 0),
                                           restart == 0 ? ctx->hist : nullptr, ctx->hist_cap);
    ctx->launches++;
    // r = b - A x
    int s = launch_residual<double>(ctx, x, nullptr, nullptr, b, ctx->r64, 0, tol2);
    if (s) return s;
    k_state_from_residual<<<1, 1, 0, ctx->stream>>>(ctx->st, tol2, o->tol_abs);
    ctx->launches++;
    s = read_state(ctx);
    if (s) return s;
    if (!std::isfinite(ctx->h_st->rr64) || !std::isfinite(ctx->h_st->bb64)) return SEVP_NONFINITE;
    double rel = ctx->h_st->bb64 > 0 ? sqrt(ctx->h_st->rr64 / ctx->h_st->bb64) : 0.0;
    rep->bnorm = sqrt(ctx->h_st->bb64);
    rep->rel_residual = rel;
    rep->abs_residual = sqrt(ctx->h_st->rr64);
    rep->refinements++;
    if (outer_converged(ctx->h_st, o)) {
      status = SEVP_OK;
      break;
    }
    if (total >= o->max_iter) {
      status = SEVP_MAXITER;
      break;
    }
    // z = M^{-1} r, rz; then iterate
    s = precondition_pass<double, false, true>(ctx, nullptr, nullptr, ctx->r64, nullptr, ctx->z64);
    if (s) return s;
    int it = 0;
    s = pcg_loop<double>(ctx, x, ctx->r64, ctx->z64, ctx->p64[0], ctx->p64[1], ctx->q64,
                         std::max(1, o->check_every), &it);
    if (s) return s;
    total += it;
    status = ctx->h_st->status;
    if (status != SEVP_OK && status != SEVP_MAXITER) break;
  }
  rep->iterations = total;
  return status;
}

// FP32 PCG inside FP64 iterative refinement.
static int ensure_mats32_of(sevp_ctx *ctx, Tiling &T) {
  if (T.d_mats32 || !T.built) return SEVP_OK;
  const size_t n = (size_t)std::max<long long>(T.mats_elems, 1);
  SEVP_CUDA_TRY(cudaMalloc((void **)&T.d_mats32, n * sizeof(float)));
  k_to_float<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 32), 256, 0, ctx->stream>>>(
      T.d_mats, T.d_mats32, n);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}
static int ensure_mats32(sevp_ctx *ctx) {
  int s = ensure_mats32_of(ctx, ctx->ta);
  return s ? s : ensure_mats32_of(ctx, ctx->tb);
}

static int solve_mixed(sevp_ctx *ctx, const double *b, double *x, const sevp_solve_opts *o,
                       sevp_report *rep) {
  if (o->precond_fp32) {
    int s = ensure_mats32(ctx);
    if (s) return s;
  }
  struct Flag {
    sevp_ctx *c;
    ~Flag() { c->infl32_active = false; }
  } flag{ctx};
  ctx->infl32_active = o->precond_fp32 != 0;
  const double inner2 = o->inner_tol * o->inner_tol;
  // the last inner solve stops at half the outer tolerance instead of
  // overshooting it by up to a factor inner_tol
  const double outer2 = 0.25 * o->tol * o->tol;  // relative or absolute (o->tol_abs)
  int total = 0, status = SEVP_MAXITER;
  double *xa = x, *xb = ctx->x64s;  // ping-pong: the residual kernel reads xa, writes xb
  bool have_d = false;
  const int method = o->method;
  // PCG with reliable updates: after the first inner solve, every FP64
  // residual replaces the FP32 recursive residual, the correction is folded
  // into x, and CG goes on along its previous search direction (unless the
  // caller asks for restarts)
  const bool keep = method == SEVP_METHOD_PCG && !o->restart_inner;
  // the Chebyshev counterpart: the recurrence continues on the replaced
  // residual with its last direction
  const bool keep_cheb = method == SEVP_METHOD_CHEB && !o->restart_inner;
  bool have_dir = false;
  for (int refine = 0; refine < 64; ++refine) {
    if (keep && have_dir)
      k_state_keep<<<1, 1, 0, ctx->stream>>>(ctx->st, inner2, std::max(o->max_iter - total, 0));
    else if (keep_cheb && have_dir)
      k_state_keep_cheb<<<1, 1, 0, ctx->stream>>>(ctx->st, inner2,
                                                   std::max(o->max_iter - total, 0) + 1);
    else
      k_state_init<<<1, 1, 0, ctx->stream>>>(ctx->st, inner2, std::max(o->max_iter - total, 0));
    ctx->launches++;
    int s;
    // PCG with reliable updates resumes its run on the FP64 residual: the
    // replaced r enters the next pass B (r - alpha q) and the preconditioned
    // residual of the stopped run's last pass stands in for one step, when
    // the residual pass finds the stopped run's recursive residual close to
    // the replaced one (SolveState::resumed); otherwise the continuation
    // applies the preconditioner to the replaced residual first.  The
    // Schwarz sweep does not resume: on the 64-member ensemble its runs are
    // a few iterations long and resumed solves took 9 iterations against 5
    const bool resume = keep && have_dir && !schwarz_on(ctx) && ctx->resume_dev > 0.0;
    if (have_d)
      s = launch_residual<float>(ctx, xa, ctx->d32, xb, b, ctx->r32, resume ? 2 : 1, inner2, outer2,
                                 o->tol_abs);
    else
      s = launch_residual<float>(ctx, xa, nullptr, nullptr, b, ctx->r32, 1, inner2, outer2,
                                 o->tol_abs);
    if (s) return s;
    if (have_d) std::swap(xa, xb);
    s = read_state(ctx);
    if (s) return s;
    if (!std::isfinite(ctx->h_st->rr64) || !std::isfinite(ctx->h_st->bb64)) {
      status = SEVP_NONFINITE;
      break;
    }
    double rel = ctx->h_st->bb64 > 0 ? sqrt(ctx->h_st->rr64 / ctx->h_st->bb64) : 0.0;
    rep->bnorm = sqrt(ctx->h_st->bb64);
    rep->rel_residual = rel;
    rep->abs_residual = sqrt(ctx->h_st->rr64);
    rep->refinements++;
    if (outer_converged(ctx->h_st, o)) {
      status = SEVP_OK;
      break;
    }
    if (total >= o->max_iter) {
      status = SEVP_MAXITER;
      break;
    }
    // inner solve A d = r32 from d = 0
    SEVP_CUDA_TRY(cudaMemsetAsync(ctx->d32, 0, ctx->n * 4, ctx->stream));
    int it = 0;
    if (method == SEVP_METHOD_PCG) {
      if (!(resume && ctx->h_st->resumed)) {
        s = precondition_pass<float, false, true>(ctx, nullptr, nullptr, ctx->r32, nullptr,
                                                  ctx->z32);
        if (s) return s;
      }
      s = pcg_loop<float>(ctx, ctx->d32, ctx->r32, ctx->z32, ctx->p32[0], ctx->p32[1], ctx->q32,
                          std::max(1, o->check_every), &it);
      // iteration k writes its search direction into p32[(k + 1) & 1]; the
      // next loop starts from p32[0]
      if (!s && keep && (it & 1))
        SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->p32[0], ctx->p32[1], ctx->n * sizeof(float),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
      have_dir = have_dir || it > 0;
    } else {
      s = cheb_inner(ctx, std::max(1, o->check_every), &it, keep_cheb && have_dir);
      // launch j writes its direction into p32[(j + 1) & 1]; the next inner
      // solve continues from p32[0]
      if (!s && keep_cheb && (it & 1))
        SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->p32[0], ctx->p32[1], ctx->n * sizeof(float),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
      have_dir = have_dir || it > 0;
    }
    if (s) return s;
    total += it;
    have_d = true;
    int ist = ctx->h_st->status;
    if (ist != SEVP_OK && ist != SEVP_MAXITER) {
      status = ist;
      break;
    }
  }
  if (xa != x) SEVP_CUDA_TRY(cudaMemcpyAsync(x, xa, ctx->n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  rep->iterations = total;
  return status;
}

extern "C" int sevp_solve(sevp_ctx *ctx, const double *b, double *x, const sevp_solve_opts *o,
                          sevp_report *rep) {
  if (!ctx || !ctx->have_op || !b || !x || !o) return SEVP_BAD_ARG;
  if (ctx->asym) {
    sevp_internal_set_message(
        "sevp_solve: the operator is not symmetric (AR(i,j) != AL(i+1,j) or AT(i,j) != "
        "AB(i,j+1)), so conjugate gradients has no convergence guarantee; scale its rows "
        "(p_sevp_pcg_ does this for PREP's coefficients) or use p_bicgstab_le_");
    if (rep) *rep = sevp_report{}, rep->status = SEVP_NONSYMMETRIC;
    return SEVP_NONSYMMETRIC;
  }
  if (!(o->tol > 0.0) || o->max_iter < 0 || (o->precision != 0 && o->precision != 1))
    return SEVP_BAD_ARG;
  if (o->method != SEVP_METHOD_PCG) {
    const char *why = nullptr;
    if (o->method != SEVP_METHOD_CHEB) why = "unknown method";
    else if (o->precision != 1) why = "the Chebyshev iteration runs in the mixed-precision mode (precision 1)";
    else if (schwarz_on(ctx)) why = "the Chebyshev iteration uses the block-Jacobi tiles (no Schwarz)";
    else if (ctx->ta.tg.hmax > kChebMaxRows) why = "the Chebyshev iteration needs tiles of at most 8 rows";
    else if (!(ctx->cheb_lmax > ctx->cheb_lmin && ctx->cheb_lmin > 0.0))
      why = "Chebyshev needs spectrum bounds (sevp_set_chebyshev_bounds / sevp_estimate_bounds)";
    if (why) {
      std::string m = std::string("sevp_solve: ") + why;
      sevp_internal_set_message(m.c_str());
      return SEVP_BAD_ARG;
    }
  }
  if (o->precision == 1 && !(o->inner_tol > 0.0 && o->inner_tol < 1.0)) return SEVP_BAD_ARG;
  sevp_report local{};
  sevp_report *r = rep ? rep : &local;
  *r = sevp_report{};
  if (!o->use_guess) SEVP_CUDA_TRY(cudaMemsetAsync(x, 0, ctx->n * 8, ctx->stream));
  SEVP_CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  int s = o->precision == 0 ? solve_fp64(ctx, b, x, o, r) : solve_mixed(ctx, b, x, o, r);
  SEVP_CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  SEVP_CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  r->ms = ms;
  r->status = s;
  return s;
}

extern "C" int sevp_solve_host(sevp_ctx *ctx, const double *bh, double *xh,
                               const sevp_solve_opts *o, sevp_report *rep) {
  if (!ctx || !bh || !xh || !o) return SEVP_BAD_ARG;
  if (!ctx->bh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->bh, ctx->n * 8));
  if (!ctx->xh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->xh, ctx->n * 8));
  SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->bh, bh, ctx->n * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (o->use_guess)
    SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->xh, xh, ctx->n * 8, cudaMemcpyHostToDevice, ctx->stream));
  int s = sevp_solve(ctx, ctx->bh, ctx->xh, o, rep);
  cudaError_t e = cudaMemcpyAsync(xh, ctx->xh, ctx->n * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "copy x to host", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  return s;
}

// guess = 2 eta1 - eta2 (mode 2), eta1 (mode 1) or 0 (mode 0)
__global__ void k_guess(const double *eta1, const double *eta2, double *g, size_t n, int mode) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (mode == 1) v = eta1[k];
    if (mode == 2) v = 2.0 * eta1[k] - eta2[k];
    g[k] = v;
  }
}

static int form_guess(sevp_ctx *ctx, const double *eta1, const double *eta2, double *x, int mode) {
  if (mode == SEVP_GUESS_LEARNED) {
    if (!ctx->warm_fn) return SEVP_BAD_ARG;
    int s = ctx->warm_fn(ctx->warm_user, eta1, eta2, ctx->cur_b, x, ctx->nx, ctx->ny,
                         (void *)ctx->stream);
    ctx->launches += ctx->warm_launches_per_call;
    return s;
  }
  if (mode < 0 || mode > 2 || (mode >= 1 && !eta1) || (mode == 2 && !eta2)) return SEVP_BAD_ARG;
  unsigned blocks = (unsigned)std::min<size_t>((ctx->n + 255) / 256, 148 * 16);
  k_guess<<<blocks, 256, 0, ctx->stream>>>(eta1, eta2, x, ctx->n, mode);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

extern "C" int sevp_set_warmstart(sevp_ctx *ctx, sevp_warmstart_fn fn, void *user,
                                  int launches_per_call) {
  if (!ctx) return SEVP_BAD_ARG;
  ctx->warm_fn = fn;
  ctx->warm_user = user;
  ctx->warm_launches_per_call = launches_per_call;
  return SEVP_OK;
}

extern "C" int sevp_solve_step(sevp_ctx *ctx, const double *b, const double *eta1,
                               const double *eta2, double *x, int guess_mode,
                               const sevp_solve_opts *o, sevp_report *rep) {
  if (!ctx || !ctx->have_op || !b || !x || !o) return SEVP_BAD_ARG;
  ctx->cur_b = b;
  int s = form_guess(ctx, eta1, eta2, x, guess_mode);
  if (s) return s;
  sevp_solve_opts oo = *o;
  oo.use_guess = 1;
  return sevp_solve(ctx, b, x, &oo, rep);
}

extern "C" int sevp_solve_step_host(sevp_ctx *ctx, const double *bh, const double *eta1h,
                                    const double *eta2h, double *xh, int guess_mode,
                                    const sevp_solve_opts *o, sevp_report *rep) {
  if (!ctx || !bh || !xh || !o) return SEVP_BAD_ARG;
  if (!ctx->bh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->bh, ctx->n * 8));
  if (!ctx->xh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->xh, ctx->n * 8));
  if (!ctx->e1h) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->e1h, ctx->n * 8));
  if (!ctx->e2h) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->e2h, ctx->n * 8));
  const size_t bytes = ctx->n * 8;
  SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->bh, bh, bytes, cudaMemcpyHostToDevice, ctx->stream));
  if (guess_mode >= 1 && eta1h)
    SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->e1h, eta1h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  if ((guess_mode == 2 || guess_mode == SEVP_GUESS_LEARNED) && eta2h)
    SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->e2h, eta2h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  int s = sevp_solve_step(ctx, ctx->bh, eta1h ? ctx->e1h : nullptr, eta2h ? ctx->e2h : nullptr,
                          ctx->xh, guess_mode, o, rep);
  if (s != SEVP_OK && s != SEVP_MAXITER) return s;
  SEVP_CUDA_TRY(cudaMemcpyAsync(xh, ctx->xh, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return s;
}

// ---------------------------------------------- stepping with device history
static int ensure_step_buffers(sevp_ctx *ctx) {
  for (double *&p : ctx->step_buf)
    if (!p) SEVP_CUDA_TRY(cudaMalloc((void **)&p, ctx->n * 8));
  if (!ctx->bh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->bh, ctx->n * 8));
  return SEVP_OK;
}

extern "C" int sevp_step_history(sevp_ctx *ctx, const double *eta1_host, const double *eta2_host) {
  if (!ctx || (!eta1_host && eta2_host)) return SEVP_BAD_ARG;
  int s = ensure_step_buffers(ctx);
  if (s) return s;
  // x copies of submitted steps may still read the buffers
  if (ctx->cp_out) SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->cp_out));
  const size_t bytes = ctx->n * 8;
  ctx->step_e1 = 0, ctx->step_e2 = 1, ctx->step_hist = 0;
  if (eta1_host) {
    SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->step_buf[0], eta1_host, bytes, cudaMemcpyHostToDevice,
                                  ctx->stream));
    ctx->step_hist = 1;
  }
  if (eta2_host) {
    SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->step_buf[1], eta2_host, bytes, cudaMemcpyHostToDevice,
                                  ctx->stream));
    ctx->step_hist = 2;
  }
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return SEVP_OK;
}

extern "C" int sevp_step_host(sevp_ctx *ctx, const double *bh, double *xh, int guess_mode,
                              const sevp_solve_opts *o, sevp_report *rep) {
  if (!ctx || !ctx->have_op || !bh || !xh || !o || guess_mode < 0 || guess_mode > 3)
    return SEVP_BAD_ARG;
  int s = ensure_step_buffers(ctx);
  if (s) return s;
  const size_t bytes = ctx->n * 8;
  SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->bh, bh, bytes, cudaMemcpyHostToDevice, ctx->stream));
  // the guess needs as much history as there is
  int mode = guess_mode;
  if (ctx->step_hist == 0) mode = SEVP_GUESS_ZERO;
  if (ctx->step_hist == 1 && mode > SEVP_GUESS_PREVIOUS) mode = SEVP_GUESS_PREVIOUS;
  const int out = 3 - ctx->step_e1 - ctx->step_e2;  // the buffer holding neither
  if (ctx->ev_out_set[out]) SEVP_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_out[out], 0));
  s = sevp_solve_step(ctx, ctx->bh, ctx->step_buf[ctx->step_e1], ctx->step_buf[ctx->step_e2],
                      ctx->step_buf[out], mode, o, rep);
  if (s != SEVP_OK && s != SEVP_MAXITER) return s;
  SEVP_CUDA_TRY(cudaMemcpyAsync(xh, ctx->step_buf[out], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->step_e2 = ctx->step_e1;
  ctx->step_e1 = out;
  ctx->step_hist = std::min(ctx->step_hist + 1, 2);
  return s;
}

static int ensure_async_step(sevp_ctx *ctx) {
  int s = ensure_step_buffers(ctx);
  if (s) return s;
  if (ctx->cp_in) return SEVP_OK;
  SEVP_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->cp_in, cudaStreamNonBlocking));
  SEVP_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->cp_out, cudaStreamNonBlocking));
  for (double *&p : ctx->bstage) SEVP_CUDA_TRY(cudaMalloc((void **)&p, ctx->n * 8));
  for (cudaEvent_t &e : ctx->ev_in) SEVP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (cudaEvent_t &e : ctx->ev_out) SEVP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  SEVP_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_solved, cudaEventDisableTiming));
  return SEVP_OK;
}

// Starts the copy of a step's b into the next staging buffer on the copy-in
// stream.  A staging buffer is reused only after the solve that read it has
// returned (the solves are synchronous), so two are enough.
static int stage_b(sevp_ctx *ctx, const double *bh) {
  const int k = ctx->bstage_next;
  ctx->bstage_next ^= 1;
  SEVP_CUDA_TRY(cudaMemcpyAsync(ctx->bstage[k], bh, ctx->n * 8, cudaMemcpyHostToDevice, ctx->cp_in));
  SEVP_CUDA_TRY(cudaEventRecord(ctx->ev_in[k], ctx->cp_in));
  ctx->bstage_src[k] = bh;
  return SEVP_OK;
}

extern "C" int sevp_step_prefetch(sevp_ctx *ctx, const double *bh) {
  if (!ctx || !bh) return SEVP_BAD_ARG;
  int s = ensure_async_step(ctx);
  return s ? s : stage_b(ctx, bh);
}

extern "C" int sevp_step_submit(sevp_ctx *ctx, const double *bh, double *xh, int guess_mode,
                                const sevp_solve_opts *o, sevp_report *rep) {
  if (!ctx || !ctx->have_op || !bh || !xh || !o || guess_mode < 0 || guess_mode > 3)
    return SEVP_BAD_ARG;
  int s = ensure_async_step(ctx);
  if (s) return s;
  // b: the staged copy when it was prefetched, else staged now
  int k = -1;
  for (int q = 0; q < 2; ++q)
    if (ctx->bstage_src[q] == bh) k = q;
  if (k < 0) {
    k = ctx->bstage_next;
    s = stage_b(ctx, bh);
    if (s) return s;
  }
  ctx->bstage_src[k] = nullptr;  // consumed by this step
  SEVP_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[k], 0));
  int mode = guess_mode;
  if (ctx->step_hist == 0) mode = SEVP_GUESS_ZERO;
  if (ctx->step_hist == 1 && mode > SEVP_GUESS_PREVIOUS) mode = SEVP_GUESS_PREVIOUS;
  const int out = 3 - ctx->step_e1 - ctx->step_e2;
  // the output buffer's previous contents must have left for the host
  if (ctx->ev_out_set[out]) SEVP_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_out[out], 0));
  s = sevp_solve_step(ctx, ctx->bstage[k], ctx->step_buf[ctx->step_e1],
                      ctx->step_buf[ctx->step_e2], ctx->step_buf[out], mode, o, rep);
  if (s != SEVP_OK && s != SEVP_MAXITER) return s;
  // x leaves on the copy-out stream while the caller goes on
  SEVP_CUDA_TRY(cudaEventRecord(ctx->ev_solved, ctx->stream));
  SEVP_CUDA_TRY(cudaStreamWaitEvent(ctx->cp_out, ctx->ev_solved, 0));
  SEVP_CUDA_TRY(cudaMemcpyAsync(xh, ctx->step_buf[out], ctx->n * 8, cudaMemcpyDeviceToHost,
                                ctx->cp_out));
  SEVP_CUDA_TRY(cudaEventRecord(ctx->ev_out[out], ctx->cp_out));
  ctx->ev_out_set[out] = true;
  ctx->step_e2 = ctx->step_e1;
  ctx->step_e1 = out;
  ctx->step_hist = std::min(ctx->step_hist + 1, 2);
  return s;
}

extern "C" int sevp_step_wait(sevp_ctx *ctx) {
  if (!ctx) return SEVP_BAD_ARG;
  if (ctx->cp_out) SEVP_CUDA_TRY(cudaStreamSynchronize(ctx->cp_out));
  return SEVP_OK;
}

// ---------------------------------------------------- learned warm start
// Features of the network from (eta1, eta2, b): e = 2 eta1 - eta2 (the
// linear extrapolation), r = b - A e, m = M^{-1} r (one tile-SEVP solve),
// d = eta1 - eta2, averaged over coarse x coarse cells.  scales[0..2] = RMS
// of those averages; the packed input is BF16 NHWC with 16 channels: r/s0,
// m/s1, d/s2, then zeros.

// The network grid is the solver grid averaged over coarse x coarse cells
// (coarse = 1, 2, 4, 8 or 16), padded with zeros to wn x hn (multiples of 8).
// feat holds 16 BF16 channels per network pixel.
__device__ __forceinline__ bool net_cell(size_t k, int wn, int cx, int cy, int coarse, int &i,
                                         int &j) {
  const int ci = (int)(k % wn), cj = (int)(k / wn);
  i = ci * coarse;
  j = cj * coarse;
  return ci < cx && cj < cy;
}

// Coarse-cell averages of r, m and d into avg (3 planes of wn x hn; the
// caller zeroes the padding), and their RMS over the network grid's cells
// as the normalisation scales[0..2] (the last CTA finishes the sums).
// Grid: blockIdx.y is the coarse row, each thread one fine column of it
// (coalesced reads down the coarse rows), and the coarse lanes of a cell
// add their column sums by shuffles (coarse divides 32).
constexpr int kPackThreads = 256;
__global__ void __launch_bounds__(kPackThreads)
    k_pack_avg(const double *r, const double *m, const double *d, float *avg, int nx, int ny,
               int coarse, int wn, int hn, double *partials, unsigned *ticket, float *scales) {
  const int cx = nx / coarse, cy = ny / coarse;
  const size_t n = (size_t)wn * hn;
  const double inv = 1.0 / (coarse * coarse);
  const int cj = blockIdx.y;
  const int i = blockIdx.x * kPackThreads + threadIdx.x;
  double a = 0.0, bm = 0.0, c = 0.0;
  if (i < cx * coarse) {
    for (int dj = 0; dj < coarse; ++dj) {
      const size_t q = (size_t)(cj * coarse + dj) * nx + i;
      a += r[q];
      bm += m[q];
      c += d[q];
    }
  }
  for (int off = coarse >> 1; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    bm += __shfl_down_sync(0xffffffffu, bm, off);
    c += __shfl_down_sync(0xffffffffu, c, off);
  }
  double s[3] = {0.0, 0.0, 0.0};
  if (i % coarse == 0 && i / coarse < cx) {
    const size_t k = (size_t)cj * wn + i / coarse;
    a *= inv, bm *= inv, c *= inv;
    avg[k] = (float)a;
    avg[n + k] = (float)bm;
    avg[2 * n + k] = (float)c;
    s[0] = a * a, s[1] = bm * bm, s[2] = c * c;
  }
  struct Fin {
    float *scales;
    double cells;
    __device__ void operator()(double (&v)[3]) {
      for (int q = 0; q < 3; ++q) {
        const double rms = sqrt(v[q] / cells);
        scales[q] = (float)(rms > 0.0 ? rms : 1.0);
      }
    }
  } fin{scales, (double)cx * cy};
  reduce_and_finish<3>(s, partials, ticket, fin);
}

// The network input: BF16 NHWC with 16 channels, r/s0, m/s1, d/s2, then zeros.
__global__ void k_pack_features(const float *avg, const float *scales, __nv_bfloat16 *feat,
                                size_t n) {
  const float i0 = 1.f / scales[0], i1 = 1.f / scales[1], i2 = 1.f / scales[2];
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    __nv_bfloat16 v[16];
    v[0] = __float2bfloat16(avg[k] * i0);
    v[1] = __float2bfloat16(avg[n + k] * i1);
    v[2] = __float2bfloat16(avg[2 * n + k] * i2);
#pragma unroll
    for (int q = 3; q < 16; ++q) v[q] = __float2bfloat16(0.f);
    uint4 *dst = reinterpret_cast<uint4 *>(feat + k * 16);
    dst[0] = *reinterpret_cast<uint4 *>(&v[0]);
    dst[1] = *reinterpret_cast<uint4 *>(&v[8]);
  }
}

// training target (eta - e - m) / scale_m averaged like the features (0 on
// the padding); combine x = e + m + scale_m * y with y taken from the
// network cell that contains the point
__global__ void k_nn_target(const double *eta, const double *e, const double *m,
                            const float *scales, float *t, int nx, int ny, int coarse, int wn,
                            int hn) {
  const int cx = nx / coarse, cy = ny / coarse;
  const size_t n = (size_t)wn * hn;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    double a = 0.0;
    if (net_cell(k, wn, cx, cy, coarse, i, j)) {
      for (int dj = 0; dj < coarse; ++dj)
        for (int di = 0; di < coarse; ++di) {
          const size_t q = (size_t)(j + dj) * nx + i + di;
          a += eta[q] - e[q] - m[q];
        }
    }
    t[k] = (float)(a / (coarse * coarse) / scales[1]);
  }
}
__global__ void k_nn_combine(const double *e, const double *m, const float *y, const float *scales,
                             double *x, int nx, int ny, int coarse, int wn) {
  const size_t n = (size_t)nx * ny;
  const int cx = nx / coarse, cy = ny / coarse;
  const float inv = 1.f / coarse;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    double c;
    if (coarse == 1) {
      c = y[(size_t)j * wn + i];
    } else {
      // bilinear between network cell centres (clamped at the edges), so
      // the correction adds no steps at cell boundaries
      const float u = (i + 0.5f) * inv - 0.5f, v = (j + 0.5f) * inv - 0.5f;
      const int i0 = max(0, min(cx - 1, (int)floorf(u))), j0 = max(0, min(cy - 1, (int)floorf(v)));
      const int i1 = min(cx - 1, i0 + 1), j1 = min(cy - 1, j0 + 1);
      const float wx = fminf(fmaxf(u - i0, 0.f), 1.f), wy = fminf(fmaxf(v - j0, 0.f), 1.f);
      const float y00 = y[(size_t)j0 * wn + i0], y01 = y[(size_t)j0 * wn + i1];
      const float y10 = y[(size_t)j1 * wn + i0], y11 = y[(size_t)j1 * wn + i1];
      c = (1.f - wy) * ((1.f - wx) * y00 + wx * y01) + wy * ((1.f - wx) * y10 + wx * y11);
    }
    x[k] = e[k] + m[k] + (double)scales[1] * c;
  }
}

static unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

static bool net_grid_ok(const sevp_ctx *ctx, int coarse, int wn, int hn) {
  if (coarse != 1 && coarse != 2 && coarse != 4 && coarse != 8 && coarse != 16) return false;
  if (ctx->nx % coarse || ctx->ny % coarse) return false;
  return wn % 8 == 0 && hn % 8 == 0 && wn >= ctx->nx / coarse && hn >= ctx->ny / coarse;
}

// One stencil pass for the features: e = 2 eta1 - eta2 (the linear
// extrapolation) formed on the fly, d = eta1 - eta2, r = b - A e.
struct OpFeatures {
  using T = double;
  static constexpr int NV = 1;
  static constexpr bool kUsesState = false;
  const double *eta1, *eta2, *b;
  double *e, *d, *r;
  __device__ void prepare(SolveState *) {}
  __device__ double value(size_t idx) const { return 2.0 * eta1[idx] - eta2[idx]; }
  __device__ void emit(size_t idx, int, double vc, double av, double (&)[NV]) const {
    e[idx] = vc;
    d[idx] = eta1[idx] - eta2[idx];
    r[idx] = b[idx] - av;
  }
  __device__ void operator()(double (&)[NV]) {}
};

extern "C" int sevp_nn_features(sevp_ctx *ctx, const double *eta1, const double *eta2,
                                const double *b, double *e, double *m, double *d, void *feat,
                                float *scales, int coarse, int wn, int hn) {
  if (!ctx || !ctx->have_op || !eta1 || !eta2 || !b || !e || !m || !d || !feat || !scales ||
      !net_grid_ok(ctx, coarse, wn, hn))
    return SEVP_BAD_ARG;
  const size_t nn = (size_t)wn * hn;
  if (ctx->nn_avg_n < nn) {
    if (ctx->nn_avg) {
      SEVP_CUDA_TRY(cudaFree(ctx->nn_avg));
      ctx->nn_avg = nullptr;
    }
    SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->nn_avg, 3 * nn * sizeof(float)));
    ctx->nn_avg_n = nn;
  }
  OpFeatures op{eta1, eta2, b, e, d, ctx->r64};
  int s = launch_stencil(ctx, op, 6);
  if (s) return s;
  // the feature is the block-Jacobi preconditioner's response (what the
  // network was trained on), whichever preconditioner the solves use
  s = launch_tile<double, false, false>(ctx, ctx->ta, nullptr, nullptr, ctx->r64, nullptr, m, 1);
  if (s) return s;
  SEVP_CUDA_TRY(cudaMemsetAsync(ctx->nn_avg, 0, 3 * nn * sizeof(float), ctx->stream));
  const dim3 pgrid((unsigned)ceil_div(ctx->nx / coarse * coarse, kPackThreads),
                   (unsigned)(ctx->ny / coarse));
  k_pack_avg<<<pgrid, kPackThreads, 0, ctx->stream>>>(ctx->r64, m, d, ctx->nn_avg, ctx->nx,
                                                      ctx->ny, coarse, wn, hn, ctx->partials,
                                                      ctx->tickets + 5, scales);
  k_pack_features<<<grid_for(nn), 256, 0, ctx->stream>>>(ctx->nn_avg, scales,
                                                         (__nv_bfloat16 *)feat, nn);
  ctx->launches += 2;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

extern "C" int sevp_nn_target(sevp_ctx *ctx, const double *eta, const double *e, const double *m,
                              const float *scales, float *t, int coarse, int wn, int hn) {
  if (!ctx || !eta || !e || !m || !scales || !t || !net_grid_ok(ctx, coarse, wn, hn))
    return SEVP_BAD_ARG;
  k_nn_target<<<grid_for((size_t)wn * hn), 256, 0, ctx->stream>>>(eta, e, m, scales, t, ctx->nx,
                                                                 ctx->ny, coarse, wn, hn);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

extern "C" int sevp_nn_combine(sevp_ctx *ctx, const double *e, const double *m, const float *y,
                               const float *scales, double *x, int coarse, int wn, int hn) {
  if (!ctx || !e || !m || !y || !scales || !x || !net_grid_ok(ctx, coarse, wn, hn))
    return SEVP_BAD_ARG;
  k_nn_combine<<<grid_for(ctx->n), 256, 0, ctx->stream>>>(e, m, y, scales, x, ctx->nx, ctx->ny,
                                                         coarse, wn);
  ctx->launches++;
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

extern "C" void *sevp_stream(const sevp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
extern "C" int sevp_add_launches(sevp_ctx *ctx, int n) {
  if (!ctx) return SEVP_BAD_ARG;
  ctx->launches += n;
  return SEVP_OK;
}

extern "C" int sevp_relative_residual(sevp_ctx *ctx, const double *b, const double *x,
                                      double *relres) {
  if (!ctx || !ctx->have_op || !b || !x || !relres) return SEVP_BAD_ARG;
  int s = launch_residual<double>(ctx, x, nullptr, nullptr, b, (double *)nullptr, 0, 0.0);
  if (s) return s;
  s = read_state(ctx);
  if (s) return s;
  *relres = ctx->h_st->bb64 > 0 ? sqrt(ctx->h_st->rr64 / ctx->h_st->bb64) : 0.0;
  return SEVP_OK;
}

// Extreme eigenvalues of the symmetric tridiagonal matrix (diagonal d,
// off-diagonal e) by bisection on Sturm sequence counts.
static void tridiag_extremes(const std::vector<double> &d, const std::vector<double> &e,
                             double *lo, double *hi) {
  const int n = (int)d.size();
  double gl = d[0], gu = d[0];
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(e[i]) : 0.0);
    gl = std::min(gl, d[i] - r);
    gu = std::max(gu, d[i] + r);
  }
  // eigenvalues below x
  auto count = [&](double x) {
    int c = 0;
    double q = d[0] - x;
    if (q < 0) ++c;
    for (int i = 1; i < n; ++i) {
      const double qq = q != 0.0 ? q : 1e-300;
      q = d[i] - x - e[i - 1] * e[i - 1] / qq;
      if (q < 0) ++c;
    }
    return c;
  };
  auto kth = [&](int k) {  // k-th smallest (0-based)
    double a = gl, b = gu;
    for (int it = 0; it < 200 && b - a > 1e-15 * std::max(std::fabs(a), std::fabs(b)); ++it) {
      const double m = 0.5 * (a + b);
      if (count(m) > k) b = m;
      else a = m;
    }
    return 0.5 * (a + b);
  };
  *lo = kth(0);
  *hi = kth(n - 1);
}

extern "C" int sevp_set_chebyshev_bounds(sevp_ctx *ctx, double lmin, double lmax) {
  if (!ctx || !(lmin > 0.0) || !(lmax > lmin) || !std::isfinite(lmax)) return SEVP_BAD_ARG;
  ctx->cheb_lmin = lmin;
  ctx->cheb_lmax = lmax;
  drop_inner_graph(ctx);
  return SEVP_OK;
}

extern "C" int sevp_estimate_bounds(sevp_ctx *ctx, const double *b, double *lmin, double *lmax,
                                    int *iterations) {
  if (!ctx || !ctx->have_op || !b || !lmin || !lmax) return SEVP_BAD_ARG;
  const int cap = 2000;
  double *keep_hist = ctx->hist;
  const int keep_cap = ctx->hist_cap;
  double *hist = nullptr;
  SEVP_CUDA_TRY(cudaMalloc((void **)&hist, sizeof(double) * 2 * cap));
  SEVP_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(double) * 2 * cap, ctx->stream));
  if (!ctx->xh) SEVP_CUDA_TRY(cudaMalloc((void **)&ctx->xh, ctx->n * 8));
  ctx->hist = hist;
  ctx->hist_cap = cap;
  sevp_solve_opts o{};
  o.precision = 0;
  o.tol = 1e-13;
  o.max_iter = cap;
  o.check_every = 4;
  o.method = SEVP_METHOD_PCG;
  sevp_report rep{};
  int s = sevp_solve(ctx, b, ctx->xh, &o, &rep);
  ctx->hist = keep_hist;
  ctx->hist_cap = keep_cap;
  std::vector<double> h((size_t)2 * cap);
  cudaError_t e = cudaMemcpy(h.data(), hist, sizeof(double) * 2 * cap, cudaMemcpyDeviceToHost);
  cudaFree(hist);
  if (s != SEVP_OK && s != SEVP_MAXITER) return s;
  if (e != cudaSuccess) {
    sevp_internal_set_error(e, "copy of the PCG coefficients", __FILE__, __LINE__);
    return SEVP_CUDA_ERROR;
  }
  int k = 0;
  while (k < cap && h[2 * k] != 0.0) ++k;
  if (k == 0) return SEVP_BREAKDOWN;
  // CG-Lanczos tridiagonal: diagonal 1/alpha_j + beta_{j-1}/alpha_{j-1},
  // off-diagonal sqrt(beta_j)/alpha_j
  std::vector<double> d((size_t)k), off((size_t)std::max(k - 1, 1));
  for (int j = 0; j < k; ++j) {
    d[j] = 1.0 / h[2 * j];
    if (j > 0) d[j] += h[2 * (j - 1) + 1] / h[2 * (j - 1)];
    if (j + 1 < k) off[j] = std::sqrt(std::fabs(h[2 * j + 1])) / h[2 * j];
  }
  tridiag_extremes(d, off, lmin, lmax);
  if (iterations) *iterations = k;
  return SEVP_OK;
}

// One Chebyshev launch on caller buffers with the given scalars (a test
// hook for the kernel itself; see the header).
__global__ void k_state_step(SolveState *st, int iter, double theta, double delta, double rho) {
  SolveState s{};
  s.iter = iter;
  s.max_iter = 1 << 30;
  s.tol2 = 0.0;
  s.bb = 1.0;
  s.cheb_theta = theta;
  s.cheb_delta = delta;
  s.cheb_sigma = theta / delta;
  s.cheb_rho = rho;
  s.status = SEVP_OK;
  *st = s;
}

extern "C" int sevp_cheb_step(sevp_ctx *ctx, int iter, double theta, double delta, double rho,
                              const float *din, float *dout, float *x, float *r,
                              double *rr_out) {
  if (!ctx || !ctx->have_op || !din || !dout || !x || !r || iter < 0 || !(delta > 0.0))
    return SEVP_BAD_ARG;
  if (ctx->ta.tg.hmax > kChebMaxRows) return SEVP_BAD_ARG;
  k_state_step<<<1, 1, 0, ctx->stream>>>(ctx->st, iter, theta, delta, rho);
  int s = launch_cheb_k(ctx, din, dout, x, r);
  if (!s) s = read_state(ctx);
  if (s) return s;
  if (rr_out) *rr_out = ctx->h_st->rr;
  return ctx->h_st->status;
}

// One pass A on caller buffers (test hook): p = z + beta p_old (z alone for
// beta = 0), q = A p; returns p.q through pq_out.
__global__ void k_state_pass_a(SolveState *st, double beta) {
  SolveState s{};
  s.beta = beta;
  s.rz = 1.0;
  s.bb = 1.0;
  s.max_iter = 1 << 30;
  s.status = SEVP_OK;
  *st = s;
}

template <typename V>
static int pass_a_step(sevp_ctx *ctx, const V *z, const V *pold, double beta, V *pnew, V *q,
                       double *pq_out) {
  if (!ctx || !ctx->have_op || !z || !pold || !pnew || !q) return SEVP_BAD_ARG;
  k_state_pass_a<<<1, 1, 0, ctx->stream>>>(ctx->st, beta);
  OpPassA<V> op{z, pold, pnew, q, ctx->st};
  int s = launch_pass_a(ctx, op);
  if (!s) s = read_state(ctx);
  if (s) return s;
  if (pq_out) *pq_out = ctx->h_st->pq;
  return ctx->h_st->status;
}

extern "C" int sevp_pass_a_f32(sevp_ctx *ctx, const float *z, const float *pold, double beta,
                               float *pnew, float *q, double *pq_out) {
  return pass_a_step(ctx, z, pold, beta, pnew, q, pq_out);
}
extern "C" int sevp_pass_a_f64(sevp_ctx *ctx, const double *z, const double *pold, double beta,
                               double *pnew, double *q, double *pq_out) {
  return pass_a_step(ctx, z, pold, beta, pnew, q, pq_out);
}
