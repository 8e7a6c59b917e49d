// The one-launch Chebyshev iteration with the tile-SEVP preconditioner.
//
// The PCG of solver.cu makes two grid passes per iteration (the stencil
// pass A and the tile pass B) because each of its two global dot products
// must be complete before the next vector update.  A Chebyshev iteration
// has no dot product that feeds the next update, so one launch does a whole
// iteration: the operator is applied inside the tile kernel to the previous
// launch's direction, whose values at the tile's halo (the rows above and
// below the tile, the columns beside it) are read from global memory as the
// previous launch left them.
//
// Preconditioned Chebyshev on the spectrum bounds [lmin, lmax] of M^-1 A
// (the reference's P-CSI, M/sevp.f90:553-616, is the unpreconditioned form
// with bounds from lanczos/ratqr; here the bounds come from CG-Lanczos):
//   theta = (lmax + lmin) / 2, delta = (lmax - lmin) / 2, sigma = theta/delta,
//   rho_0 = 1/sigma, d_0 = M^-1 r_0 / theta;
//   launch k+1: x += d_k; r -= A d_k; z = M^-1 r;
//               rho_{k+1} = 1 / (2 sigma - rho_k);
//               d_{k+1} = rho_{k+1} rho_k d_k + (2 rho_{k+1} / delta) z;
//               partial (r, r) for the stopping test.
// The first launch (state iter 0) only forms d_0.
//
// A one-launch CG is possible too (with t = M^-1 A p, z_{k+1} = z_k -
// alpha t_k and the three dot products of an iteration from one pass), but
// its residual is only implied through z, so the FP32 rounding of the
// stored z and t enters the residual multiplied by the tile operator's
// norm: measured on the bench grid, the recursion lost its accuracy after
// a residual reduction of about 1e-4, short of what an inner solve needs.
#include <algorithm>

#include "solver_core.cuh"

namespace sevp {

namespace {

// Finishes a launch: the Chebyshev scalar of this launch and the stopping
// test on (r, r).
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

// One Chebyshev iteration (see the file comment): din = d_k (read on the
// task's rows and its halo), dout = d_{k+1}; x and r updated in place.
template <typename V, typename MT, bool SYM, int HM>
__global__ void __launch_bounds__(kTileWarps * 32, 2)
    k_cheb(TileGeom tg, Coeffs c, int periodic, const MT *__restrict__ mats,
           const V *__restrict__ din, V *__restrict__ dout, V *__restrict__ x,
           V *__restrict__ r, SolveState *st, double *partials, unsigned *ticket) {
  if (st->done) return;
  constexpr bool kChain = sizeof(V) == 4;
  __shared__ double dv_all[kTileWarps * 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *dv = dv_all + wib * 32;
  const bool first = st->iter == 0;
  V c1 = V(0), c2;
  if (first) {
    c2 = (V)(1.0 / st->cheb_theta);
  } else {
    const double rho1 = 1.0 / (2.0 * st->cheb_sigma - st->cheb_rho);
    c1 = (V)(rho1 * st->cheb_rho);
    c2 = (V)(2.0 * rho1 / st->cheb_delta);
  }
  // d_k at grid index g (zero before the first launch)
  auto dir = [&](size_t g) -> V { return first ? V(0) : din[g]; };
  double acc[1] = {0.0};
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
    const MT *mt = tile_mats(mats, tg, b, grp, a, mw);
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
    V dk[HM], xr[HM], rv[HM];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      const size_t g = ok ? idx0 + (size_t)k * nx : 0;
      dk[k] = ok ? dir(g) : V(0);
      xr[k] = ok ? x[g] : V(0);
      rv[k] = ok ? r[g] : V(0);
    }
    float cc_[HM], ce_[HM], cn_[HM], cw_[SYM ? 1 : HM], cs_[SYM ? 1 : HM];
    load_task_coeffs<SYM, HM>(c, idx0, nx, hh, active, cc_, ce_, cn_, cw_, cs_);
    const bool has_s = active && j0 > 0, has_n = active && j0 + hh < ny;
    const V ds = has_s ? dir(idx0 - nx) : V(0);
    const V dn = has_n ? dir(idx0 + (size_t)hh * nx) : V(0);
    float ab0 = 0.f;
    if constexpr (SYM) ab0 = has_s ? __ldg(c.at + idx0 - nx) : 0.f;

    // ---- r -= A d on the task's rows (the full operator, across tile
    //      edges; in the vector type, the same explicitly rounded
    //      multiply-adds as the PCG's stencil pass) and x += d
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      V dw = __shfl_sync(0xffffffffu, dk[k], src_w);
      V de = __shfl_sync(0xffffffffu, dk[k], src_e);
      float cw = SYM ? __shfl_sync(0xffffffffu, ce_[k], src_w) : cw_[SYM ? 0 : k];
      const bool ok = active && k < hh;
      if (ld_w) {
        const bool okw = ok && iw >= 0;
        const size_t gwi = okw ? (size_t)(j0 + k) * nx + iw : 0;
        dw = okw ? dir(gwi) : V(0);
        if constexpr (SYM) cw = okw ? __ldg(c.ar + gwi) : 0.f;
      }
      if (ld_e) {
        const bool oke = ok && ie >= 0;
        de = oke ? dir((size_t)(j0 + k) * nx + ie) : V(0);
      }
      const float cb = SYM ? (k == 0 ? ab0 : cn_[k > 0 ? k - 1 : 0]) : cs_[SYM ? 0 : k];
      const V vb = k == 0 ? ds : dk[k > 0 ? k - 1 : 0];
      const V va = (k + 1 < hh) ? dk[k + 1 < HM ? k + 1 : k] : dn;
      const V av = stencil5<V>(cb, vb, cw, dw, cc_[k], dk[k], ce_[k], de, cn_[k], va);
      if (ok) {
        const size_t g = idx0 + (size_t)k * nx;
        const V rn = rv[k] - av;
        rv[k] = rn;
        r[g] = rn;
        x[g] = xr[k] + dk[k];
        acc[0] += (double)rn * (double)rn;
      } else {
        rv[k] = V(0);
      }
    }

    // ---- z = M^-1 r (tile SEVP march) and d_{k+1} = c1 d_k + c2 z
    auto rhs = [&](int k) -> double { return (double)rv[k]; };
    auto emit = [&](int k, double zk) {
      dout[idx0 + (size_t)k * nx] = c1 * dk[k] + c2 * (V)zk;
    };
    march_task_regs<MT, SYM, kChain, HM, false>(cc_, ce_, cn_, cw_, cs_, hh, nb, n, mw, active,
                                                lane, segbase, dv, mt, rhs, emit);
  }
  FinCheb fin{st};
  reduce_and_finish<1>(acc, partials, ticket, fin);
}

template <typename V, typename MT, bool SYM, int HM>
int launch_k(const ChebLaunch<V> &L) {
  auto kern = k_cheb<V, MT, SYM, HM>;
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
  kern<<<blocks, kTileWarps * 32, 0, L.stream>>>(L.tg, L.c, L.periodic, (const MT *)L.mats, L.din,
                                                L.dout, L.x, L.r, L.st, L.partials, L.ticket);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

template <typename V, typename MT, bool SYM>
int launch_h(const ChebLaunch<V> &L) {
  if (L.tg.hmax <= 6) return launch_k<V, MT, SYM, 6>(L);
  return launch_k<V, MT, SYM, kChebMaxRows>(L);
}

}  // namespace

template <typename V>
int cheb_launch(const ChebLaunch<V> &L) {
  if (L.tg.hmax > kChebMaxRows) return SEVP_BAD_ARG;
  if (L.mats_fp32 == 2)  // precision per warp group (MixMat)
    return L.sym ? launch_h<V, MixMat, true>(L) : launch_h<V, MixMat, false>(L);
  if (L.mats_fp32)
    return L.sym ? launch_h<V, float, true>(L) : launch_h<V, float, false>(L);
  return L.sym ? launch_h<V, double, true>(L) : launch_h<V, double, false>(L);
}
template int cheb_launch<float>(const ChebLaunch<float> &);

}  // namespace sevp
