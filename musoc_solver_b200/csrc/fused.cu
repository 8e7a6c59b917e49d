// Fused one-launch iterations of the tile-SEVP preconditioned solvers.
//
// The two-pass PCG of solver.cu makes two grid passes per iteration (the
// stencil pass A and the tile pass B) because each of its two global dot
// products must be complete before the next vector update.  The kernels
// here make ONE grid pass per iteration: the operator apply is done inside
// the tile kernel, on the direction vector of the previous launch, whose
// values at the tile's halo (the rows above and below the tile, the columns
// beside it) are read from global memory as the previous launch left them.
// Each launch reads every vector once and writes every vector once, and the
// coefficient planes are read once per iteration instead of twice.
//
// kCG: conjugate gradients with the preconditioned operator recursion.  With
// q = A p and t = M^-1 q, z_{k+1} = M^-1 r_{k+1} = z_k - alpha_k t_k, and
// (r_{k+1}, z_{k+1}) = (r,z)_k - 2 alpha_k (z_k, q_k) + alpha_k^2 (q_k, t_k)
// (M symmetric), so all three dot products of an iteration come from one
// pass and the residual r itself is never formed:
//   launch k: z_k = z_{k-1} - alpha_{k-1} t_{k-1}; p_k = z_k + beta_{k-1} p_{k-1}
//             (own points and halo); x_k = x_{k-1} + alpha_{k-1} p_{k-1};
//             q_k = A p_k; t_k = M^-1 q_k (tile SEVP march);
//             partial (p_k, q_k), (z_k, q_k), (q_k, t_k)
//   finisher: alpha_k = rz_k / (p,q); rz_{k+1} from the expansion;
//             beta_k = rz_{k+1} / rz_k.
// The last update x += alpha_k p_k is folded into the FP64 residual pass
// that follows the inner solve.
//
// kCheb: preconditioned Chebyshev iteration (the reference's P-CSI without
// preconditioner is M/sevp.f90:553-616; bounds here come from CG-Lanczos):
//   theta = (lmax + lmin) / 2, delta = (lmax - lmin) / 2, sigma = theta/delta,
//   rho_0 = 1/sigma, d_0 = M^-1 r_0 / theta;
//   launch k+1: x += d_k; r -= A d_k; z = M^-1 r;
//               rho_{k+1} = 1 / (2 sigma - rho_k);
//               d_{k+1} = rho_{k+1} rho_k d_k + (2 rho_{k+1} / delta) z;
//               partial (r, r).
// No dot product feeds the next launch, so the iteration has no global
// dependency besides the halo.
#include <algorithm>

#include "solver_core.cuh"

namespace sevp {

namespace {

// Finishes a kCG launch: alpha_k, the next (r, z) and beta_k.
struct FinCG {
  SolveState *st;
  __device__ void operator()(double (&s)[3]) {
    const double pq = s[0], zq = s[1], qt = s[2];
    st->iter += 1;
    if (!isfinite(pq) || !isfinite(zq) || !isfinite(qt)) {
      st->status = SEVP_NONFINITE;
      st->done = 1;
      return;
    }
    if (pq == 0.0) {
      st->status = SEVP_BREAKDOWN;
      st->done = 1;
      return;
    }
    const double rz = st->rz, alpha = rz / pq;
    const double rzn = (rz - 2.0 * alpha * zq) + alpha * alpha * qt;
    st->alpha = alpha;
    st->pq = pq;
    st->rr = rzn;
    // converged, or (r, z) changed sign: the recursion is at its rounding
    // floor and the FP64 residual pass takes over
    if (fabs(rzn) <= st->tol2 * fabs(st->bb) || rzn / rz <= 0.0) {
      st->status = SEVP_OK;
      st->done = 1;
      return;
    }
    if (st->iter >= st->max_iter) {
      st->status = SEVP_MAXITER;
      st->done = 1;
      return;
    }
    st->beta = rzn / rz;
    st->rz = rzn;
  }
};

// Finishes a kCheb launch: the Chebyshev scalar of this launch and the
// stopping test on (r, r).
struct FinCheb {
  SolveState *st;
  __device__ void operator()(double (&s)[1]) {
    const bool first = st->iter == 0;
    st->cheb_rho = first ? 1.0 / st->cheb_sigma : 1.0 / (2.0 * st->cheb_sigma - st->cheb_rho);
    st->iter += 1;
    st->rr = s[0];
    if (!isfinite(s[0])) {
      st->status = SEVP_NONFINITE;
      st->done = 1;
      return;
    }
    if (s[0] <= st->tol2 * st->bb) {
      st->status = SEVP_OK;
      st->done = 1;
      return;
    }
    if (st->iter > st->max_iter) {
      st->status = SEVP_MAXITER;
      st->done = 1;
    }
  }
};

// One fused iteration (see the file comment).  Vector arguments:
//   kCG:   zi, ti, pi: z_{k-1}, t_{k-1}, p_{k-1}; zo, to, po: z_k, t_k, p_k;
//          x: x_{k-1} in, x_k out; r unused
//   kCheb: zi: d_k; zo: d_{k+1}; x, r: in place; ti, pi, to, po unused
template <typename V, typename MT, bool SYM, int HM, int MODE>
__global__ void __launch_bounds__(kTileWarps * 32, 2)
    k_fused(TileGeom tg, Coeffs c, int periodic, const MT *__restrict__ mats, const V *zi,
            const V *ti, const V *pi, V *zo, V *to, V *po, V *x, V *r, SolveState *st,
            double *partials, unsigned *ticket) {
  if (st->done) return;
  constexpr bool kChain = sizeof(V) == 4;
  constexpr int NV = MODE == kFusedCG ? 3 : 1;
  __shared__ double dv_all[kTileWarps * 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *dv = dv_all + wib * 32;
  const bool first = st->iter == 0;
  V a_prev = V(0), b_prev = V(0), c1 = V(0), c2 = V(0);
  if constexpr (MODE == kFusedCG) {
    if (!first) a_prev = (V)st->alpha, b_prev = (V)st->beta;
  } else {
    if (first) {
      c2 = (V)(1.0 / st->cheb_theta);
    } else {
      const double rho1 = 1.0 / (2.0 * st->cheb_sigma - st->cheb_rho);
      c1 = (V)(rho1 * st->cheb_rho);
      c2 = (V)(2.0 * rho1 / st->cheb_delta);
    }
  }
  // the direction at grid index g: p_k (kCG) or d_k (kCheb)
  auto dir = [&](size_t g) -> V {
    if constexpr (MODE == kFusedCG) {
      if (first) return zi[g];
      return (zi[g] - a_prev * ti[g]) + b_prev * pi[g];
    } else {
      return first ? V(0) : zi[g];
    }
  };
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  const int nx = tg.nx, ny = tg.ny;
  const int ntasks = tg.ty * tg.txg;
  for (int gw = blockIdx.x * kTileWarps + wib; gw < ntasks; gw += gridDim.x * kTileWarps) {
    const int b = gw / tg.txg;
    const int grp = gw - b * tg.txg;
    const int seg = lane / tg.wseg, n = lane - seg * tg.wseg, segbase = seg * tg.wseg;
    const int a = grp * tg.tpw + seg;
    const int mw = (a < tg.tx) ? tile_width(tg, a) : 0;
    const bool active = n < mw;
    const int j0 = b * tg.th, hh = tile_height(tg, b), nb = tg.grp_nb[(size_t)b * tg.txg + grp];
    const int i = tile_col(tg, a, n);
    const MT *mt = mats + (mw > 0 ? tg.moff[(size_t)b * tg.tx + a] : 0);
    const size_t idx0 = (size_t)j0 * nx + i;

    // west / east neighbours: a shuffle from the lane holding that column,
    // or (at the warp's edge and across the periodic seam) a load
    int src_w = lane, src_e = lane, iw = -1, ie = -1;
    bool ld_w = false, ld_e = false;
    if (active) {
      if (n > 0) src_w = lane - 1;
      else if (seg > 0) src_w = lane - tg.wseg + tg.tm - 1;
      else ld_w = true, iw = i > 0 ? i - 1 : (periodic ? nx - 1 : -1);
      if (n < mw - 1) src_e = lane + 1;
      else if (seg + 1 < tg.tpw && a + 1 < tg.tx) src_e = lane - n + tg.wseg;
      else ld_e = true, ie = i + 1 < nx ? i + 1 : (periodic ? 0 : -1);
    }

    // ---- loads of the task's rows
    V pv[HM], zc[MODE == kFusedCG ? HM : 1], xr[HM], rv[MODE == kFusedCheb ? HM : 1];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      const size_t g = ok ? idx0 + (size_t)k * nx : 0;
      if constexpr (MODE == kFusedCG) {
        V zz = ok ? zi[g] : V(0), xx = ok ? x[g] : V(0);
        V pp = zz;
        if (!first && ok) {
          const V tv = ti[g], po_ = pi[g];
          zz = zz - a_prev * tv;
          pp = zz + b_prev * po_;
          xx = xx + a_prev * po_;
        }
        zc[k] = zz;
        pv[k] = pp;
        xr[k] = xx;
      } else {
        pv[k] = (ok && !first) ? zi[g] : V(0);
        xr[k] = ok ? x[g] : V(0);
        rv[k] = ok ? r[g] : V(0);
      }
    }
    float cc_[HM], ce_[HM], cn_[HM], cw_[SYM ? 1 : HM], cs_[SYM ? 1 : HM];
    load_task_coeffs<SYM, HM>(c, idx0, nx, hh, active, cc_, ce_, cn_, cw_, cs_);
    const bool has_s = active && j0 > 0, has_n = active && j0 + hh < ny;
    const V ps = has_s ? dir(idx0 - nx) : V(0);
    const V pn = has_n ? dir(idx0 + (size_t)hh * nx) : V(0);
    float ab0 = 0.f;
    if constexpr (SYM) ab0 = has_s ? __ldg(c.at + idx0 - nx) : 0.f;

    // ---- q = A p on the task's rows (the full operator, across tile edges)
    V q[HM];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      V pw = __shfl_sync(0xffffffffu, pv[k], src_w);
      V pe = __shfl_sync(0xffffffffu, pv[k], src_e);
      float cw = SYM ? __shfl_sync(0xffffffffu, ce_[k], src_w) : cw_[SYM ? 0 : k];
      const bool ok = active && k < hh;
      if (ld_w) {
        const bool okw = ok && iw >= 0;
        const size_t gwi = okw ? (size_t)(j0 + k) * nx + iw : 0;
        pw = okw ? dir(gwi) : V(0);
        if constexpr (SYM) cw = okw ? __ldg(c.ar + gwi) : 0.f;
      }
      if (ld_e) {
        const bool oke = ok && ie >= 0;
        pe = oke ? dir((size_t)(j0 + k) * nx + ie) : V(0);
      }
      const float cb = SYM ? (k == 0 ? ab0 : cn_[k > 0 ? k - 1 : 0]) : cs_[SYM ? 0 : k];
      const V vb = k == 0 ? ps : pv[k > 0 ? k - 1 : 0];
      const V va = (k + 1 < hh) ? pv[k + 1 < HM ? k + 1 : k] : pn;
      V av = V(cb) * vb;
      av += V(cw) * pw;
      av += V(cc_[k]) * pv[k];
      av += V(ce_[k]) * pe;
      av += V(cn_[k]) * va;
      q[k] = ok ? av : V(0);
    }

    // ---- elementwise updates and stores of the own rows
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      if (!ok) continue;
      const size_t g = idx0 + (size_t)k * nx;
      if constexpr (MODE == kFusedCG) {
        zo[g] = zc[k];
        po[g] = pv[k];
        x[g] = xr[k];
        acc[0] += (double)pv[k] * (double)q[k];
        acc[1] += (double)zc[k] * (double)q[k];
      } else {
        const V rn = rv[k] - q[k];
        rv[k] = rn;
        r[g] = rn;
        x[g] = xr[k] + pv[k];
        acc[0] += (double)rn * (double)rn;
      }
    }

    // ---- tile SEVP solve: t = M^-1 q (kCG) or z = M^-1 r (kCheb)
    auto rhs = [&](int k) -> double {
      if constexpr (MODE == kFusedCG)
        return (double)q[k];
      else
        return (double)rv[k];
    };
    auto emit = [&](int k, double zk) {
      const size_t g = idx0 + (size_t)k * nx;
      if constexpr (MODE == kFusedCG) {
        const V tv = (V)zk;
        to[g] = tv;
        acc[2] += (double)q[k] * (double)tv;
      } else {
        zo[g] = c1 * pv[k] + c2 * (V)zk;
      }
    };
    march_task_regs<MT, SYM, kChain, HM, false>(cc_, ce_, cn_, cw_, cs_, hh, nb, n, mw, active,
                                                lane, segbase, dv, mt, rhs, emit);
  }
  if constexpr (MODE == kFusedCG) {
    FinCG fin{st};
    reduce_and_finish<NV>(acc, partials, ticket, fin);
  } else {
    FinCheb fin{st};
    reduce_and_finish<NV>(acc, partials, ticket, fin);
  }
}

template <typename V, typename MT, bool SYM, int HM, int MODE>
int launch_k(const FusedLaunch<V> &L) {
  auto kern = k_fused<V, MT, SYM, HM, MODE>;
  static int slots = 0;
  if (!slots) {
    int per_sm = 0, dev = 0, sms = 0;
    SEVP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileWarps * 32, 0));
    SEVP_CUDA_TRY(cudaGetDevice(&dev));
    SEVP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    slots = (per_sm > 0 ? per_sm : 1) * sms;
  }
  const size_t warps = (size_t)L.tg.ty * L.tg.txg;
  const unsigned blocks =
      (unsigned)std::min<size_t>((warps + kTileWarps - 1) / kTileWarps, (size_t)slots);
  kern<<<blocks, kTileWarps * 32, 0, L.stream>>>(L.tg, L.c, L.periodic, (const MT *)L.mats, L.zi,
                                                L.ti, L.pi, L.zo, L.to, L.po, L.x, L.r, L.st,
                                                L.partials, L.ticket);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

template <typename V, typename MT, bool SYM, int MODE>
int launch_h(const FusedLaunch<V> &L) {
  if (L.tg.hmax <= 6) return launch_k<V, MT, SYM, 6, MODE>(L);
  return launch_k<V, MT, SYM, kFusedMaxRows, MODE>(L);
}

template <typename V, int MODE>
int launch_m(const FusedLaunch<V> &L) {
  if (L.mats_fp32)
    return L.sym ? launch_h<V, float, true, MODE>(L) : launch_h<V, float, false, MODE>(L);
  return L.sym ? launch_h<V, double, true, MODE>(L) : launch_h<V, double, false, MODE>(L);
}

}  // namespace

template <typename V>
int fused_launch(const FusedLaunch<V> &L) {
  if (L.tg.hmax > kFusedMaxRows) return SEVP_BAD_ARG;
  return L.mode == kFusedCG ? launch_m<V, kFusedCG>(L) : launch_m<V, kFusedCheb>(L);
}
template int fused_launch<float>(const FusedLaunch<float> &);

}  // namespace sevp
