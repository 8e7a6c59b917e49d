// PCG pass B with the task data brought in by the tensor memory accelerator:
// x += alpha p, r -= alpha q, z = M^-1 r on the block-Jacobi tiles, r.z and
// r.r, and the finish of the iteration (the pass of k_tile_short in
// solver.cu, operation for operation: x, r and z come out bit-identical).
//
// The register kernel loads a task's rows (r, x, p, q and the planes AC, AR,
// AT) and, after the forward march, its influence matrices from global
// memory, so every task waits out two memory round trips with only 16 warps
// per SM to cover them.  Here each warp keeps a shared-memory stage of one
// task: while it marches task t, the copies of task t + stride are in
// flight.  Lane 0 issues them:
//   - the rows, as seven 2-D tensor copies of a 32 x th box (columns
//     32 g .. 32 g + 31 of tile group g, so every box starts 16-byte
//     aligned; points past the grid arrive as zeros), right after the warp
//     has moved task t's rows from the stage into registers;
//   - the influence matrices of a full task (th rows, one sub-block), one
//     bulk copy per tile, right after task t's mat-vec has read the stage's
//     matrices (other tasks read theirs from global memory).
// Each kind of copy completes on its own mbarrier of the warp.  Waits are
// bounded: a wait that gives up marks the pass failed (the finisher reports
// SEVP_TIMEOUT), the warp stops, and lane 0 waits, with the same bound, for
// the copies it issued before the warp exits.  Only this GPU's memory is
// read, and no copy uses cluster multicast.
#include <algorithm>

#include "solver_core.cuh"
#include "tma_util.cuh"

namespace sevp {

namespace {

constexpr int kHM = kShortTileRows;
constexpr int kArrays = 7;                          // r, x, p, q, AC, AR, AT
constexpr uint32_t kArrBytes = kHM * 32 * 4;        // one array's rows of a task
constexpr uint32_t kRowBytes = kArrays * kArrBytes;  // 128-byte multiple

__host__ __device__ inline uint32_t mat_bytes(int tm) { return 32u * (uint32_t)tm * 8u; }
__host__ __device__ inline uint32_t stage_bytes(int tm) {
  return (kRowBytes + mat_bytes(tm) + 16u + 127u) & ~127u;
}
__host__ __device__ inline uint32_t copy_bytes(int mw) {
  return ((uint32_t)mw * (uint32_t)mw * 8u + 15u) & ~15u;
}

struct RowMaps {
  CUtensorMap r, x, p, q, ac, ar, at;
};

// r.z and r.r as TileFin; a failed wait anywhere reports SEVP_TIMEOUT.
struct PassBFin {
  SolveState *st;
  __device__ void operator()(double (&s)[3]) {
    if (s[2] != 0.0) {
      st->status = SEVP_TIMEOUT;
      st->done = 1;
      return;
    }
    double v[2] = {s[0], s[1]};
    TileFin{st}(v);
  }
};

// out(n) = sum_k dv[seg + k] M[k mw + n] for k < mw, in the order of
// seg_matvec_w, from the matrix staged in shared memory.
template <int WMAX>
__device__ __forceinline__ double stage_matvec(const double *dv, int segbase, const double *M,
                                               int mw, int n) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < WMAX; ++k)
    if (k < mw) s += dv[segbase + k] * M[k * mw + n];
  return s;
}

template <int HM>
__global__ void __launch_bounds__(kTileWarps * 32, 2)
    k_pass_b_tma(const __grid_constant__ RowMaps maps, TileGeom tg,
                 const double *__restrict__ mats, float *x, float *r, float *z, SolveState *st,
                 double *partials, unsigned *ticket) {
  if (st->done) return;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  __shared__ double dv_all[kTileWarps * 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *dv = dv_all + wib * 32;
  const uint32_t sb = stage_bytes(tg.tm);
  const uint32_t raw_u = tma::smem_u32(sm_raw);
  const uint32_t base_u = (raw_u + 127u) & ~127u;
  const uint32_t wu = base_u + (uint32_t)wib * sb;  // this warp's stage
  const unsigned char *wg = sm_raw + (wu - raw_u);
  const float *srow = reinterpret_cast<const float *>(wg);
  const double *smat = reinterpret_cast<const double *>(wg + kRowBytes);
  const uint32_t bar_rows = wu + kRowBytes + mat_bytes(tg.tm), bar_mats = bar_rows + 8;
  if (lane == 0) {
    tma::mbar_init(bar_rows, 1);
    tma::mbar_init(bar_mats, 1);
    tma::fence_mbar_init();
  }
  __syncwarp();

  const double alpha = st->alpha;
  const int ntasks = tg.ty * tg.txg;
  const int stride = gridDim.x * kTileWarps;
  const int nx = tg.nx;
  // a task (b, grp) is full when its tiles have HM rows and one sub-block
  auto full = [&](int b, int grp) {
    return tile_height(tg, b) == HM && tg.grp_nb[(size_t)b * tg.txg + grp] == 1;
  };
  // lane 0: the copies of task (b, grp)'s rows / matrices
  auto issue_rows = [&](int b, int grp) {
    const int i0 = grp * 32, j0 = b * tg.th;
    tma::fence_proxy_async();
    tma::mbar_expect_tx(bar_rows, (uint32_t)(kArrays * 32 * tg.th * 4));
    tma::load_2d(wu + 0 * kArrBytes, &maps.r, i0, j0, bar_rows);
    tma::load_2d(wu + 1 * kArrBytes, &maps.x, i0, j0, bar_rows);
    tma::load_2d(wu + 2 * kArrBytes, &maps.p, i0, j0, bar_rows);
    tma::load_2d(wu + 3 * kArrBytes, &maps.q, i0, j0, bar_rows);
    tma::load_2d(wu + 4 * kArrBytes, &maps.ac, i0, j0, bar_rows);
    tma::load_2d(wu + 5 * kArrBytes, &maps.ar, i0, j0, bar_rows);
    tma::load_2d(wu + 6 * kArrBytes, &maps.at, i0, j0, bar_rows);
  };
  auto issue_mats = [&](int b, int grp) {
    uint32_t bytes = 0;
    for (int s = 0; s < tg.tpw && grp * tg.tpw + s < tg.tx; ++s)
      bytes += copy_bytes(tile_width(tg, grp * tg.tpw + s));
    tma::fence_proxy_async();
    tma::mbar_expect_tx(bar_mats, bytes);
    for (int s = 0; s < tg.tpw && grp * tg.tpw + s < tg.tx; ++s) {
      const int a = grp * tg.tpw + s;
      tma::load_bulk(wu + kRowBytes + (uint32_t)(s * tg.tm * tg.tm * 8),
                     mats + tg.moff[(size_t)b * tg.tx + a], copy_bytes(tile_width(tg, a)),
                     bar_mats);
    }
  };

  double acc_rz = 0.0, acc_rr = 0.0;
  unsigned ph_rows = 0, ph_mats = 0;
  bool failed = false;
  // lane constants, and the warp's task stepping without divisions: the
  // task index t = b * txg + grp advances by stride = db * txg + dg
  const int seg = lane / tg.wseg, n = lane - seg * tg.wseg, segbase = seg * tg.wseg;
  const int db = stride / tg.txg, dg = stride - db * tg.txg;
  int t = blockIdx.x * kTileWarps + wib;
  int b = t / tg.txg, grp = t - b * tg.txg;
  bool is_full = t < ntasks && full(b, grp);
  bool rows_pending = t < ntasks, mats_pending = is_full;
  if (lane == 0 && rows_pending) {
    issue_rows(b, grp);
    if (mats_pending) issue_mats(b, grp);
  }
  for (; t < ntasks;) {
    const int tn = t + stride;
    const bool has_next = tn < ntasks;
    int bn = b + db, gn = grp + dg;
    if (gn >= tg.txg) gn -= tg.txg, ++bn;
    const bool full_next = has_next && full(bn, gn);
    const int a = grp * tg.tpw + seg;
    const int mw = (a < tg.tx) ? tile_width(tg, a) : 0;
    const bool active = n < mw;
    const int j0 = b * tg.th, hh = tile_height(tg, b);
    const int i = tile_col(tg, a, n);
    const size_t idx0 = (size_t)j0 * nx + i;

    // ---- this task's rows: stage -> registers, then the next task's copies
    const bool ok_rows = tma::mbar_wait(bar_rows, ph_rows);
    if (__any_sync(0xffffffffu, !ok_rows)) {
      failed = true;
      break;
    }
    ph_rows ^= 1u;
    rows_pending = false;
    float rr[HM], xx[HM], pp[HM], qq[HM];
    float cc_[HM], ce_[HM], cn_[HM], cw_[1], cs_[1];
#pragma unroll
    for (int k = 0; k < HM; ++k) {
      const bool ok = active && k < hh;
      const int e = k * 32 + lane;
      rr[k] = ok ? srow[0 * HM * 32 + e] : 0.f;
      xx[k] = ok ? srow[1 * HM * 32 + e] : 0.f;
      pp[k] = ok ? srow[2 * HM * 32 + e] : 0.f;
      qq[k] = ok ? srow[3 * HM * 32 + e] : 0.f;
      cc_[k] = ok ? srow[4 * HM * 32 + e] : 0.f;
      ce_[k] = ok ? srow[5 * HM * 32 + e] : 0.f;
      cn_[k] = ok ? srow[6 * HM * 32 + e] : 0.f;
    }
    __syncwarp();
    if (has_next) {
      if (lane == 0) issue_rows(bn, gn);
      rows_pending = true;
      // the matrix stage is free while a task without staged matrices runs
      if (!is_full && full_next) {
        if (lane == 0) issue_mats(bn, gn);
        mats_pending = true;
      }
    }

    auto rhs = [&](int k) -> double {
      if (!active) return 0.0;
      const size_t idx = idx0 + (size_t)k * nx;
      const float xn = xx[k] + (float)alpha * pp[k];
      const float rn = rr[k] - (float)alpha * qq[k];
      x[idx] = xn;
      r[idx] = rn;
      rr[k] = rn;
      const double rv = (double)rn;
      acc_rr += rv * rv;
      return rv;
    };
    auto emit = [&](int k, double zk) {
      const float zv = (float)zk;
      z[idx0 + (size_t)k * nx] = zv;
      acc_rz += (double)rr[k] * (double)zv;
    };
    if (is_full) {
      const double *sm = smat + seg * tg.tm * tg.tm;
      auto mv = [&]() -> double {
        if (!tma::mbar_wait(bar_mats, ph_mats)) failed = true;
        if (tg.tm <= 8) return stage_matvec<8>(dv, segbase, sm, mw, n);
        if (tg.tm <= 16) return stage_matvec<16>(dv, segbase, sm, mw, n);
        return stage_matvec<32>(dv, segbase, sm, mw, n);
      };
      // every lane has read the matrices: the stage takes the next task's
      auto post = [&]() {
        if (__any_sync(0xffffffffu, failed)) {
          failed = true;
          return;
        }
        ph_mats ^= 1u;
        mats_pending = false;
        if (full_next) {
          if (lane == 0) issue_mats(bn, gn);
          mats_pending = true;
        }
      };
      march_task_full_mv<true, true, HM, false>(cc_, ce_, cn_, cw_, cs_, n, mw, active, lane, dv,
                                                rhs, emit, mv, post);
      if (failed) break;
    } else {
      const double *mt = tile_mats(mats, tg, b, grp, a, mw);
      const int nb = tg.grp_nb[(size_t)b * tg.txg + grp];
      march_task_regs<double, true, true, HM, false>(cc_, ce_, cn_, cw_, cs_, hh, nb, n, mw,
                                                     active, lane, segbase, dv, mt, rhs, emit);
    }
    t = tn, b = bn, grp = gn, is_full = full_next;
  }
  if (lane == 0) {
    // copies issued and not consumed (only after a failed wait)
    if (rows_pending) tma::mbar_wait(bar_rows, ph_rows);
    if (mats_pending) tma::mbar_wait(bar_mats, ph_mats);
  }
  double v3[3] = {acc_rz, acc_rr, failed ? 1.0 : 0.0};
  PassBFin fin{st};
  reduce_and_finish<3>(v3, partials, ticket, fin);
}

// Tensor maps of recent launches (a solve alternates between two p buffers).
struct MapKey {
  const void *p[7];
  int nx, ny, th;
  bool operator==(const MapKey &o) const {
    for (int k = 0; k < 7; ++k)
      if (p[k] != o.p[k]) return false;
    return nx == o.nx && ny == o.ny && th == o.th;
  }
};
struct MapEntry {
  MapKey key;
  RowMaps maps;
  bool used;
};
constexpr int kMapCache = 16;
thread_local MapEntry g_maps[kMapCache];
thread_local int g_maps_next = 0;

const RowMaps *row_maps(const PassBLaunch &L) {
  const int nx = L.tg.nx, ny = L.tg.ny, th = L.tg.th;
  const MapKey key{{L.r, L.x, L.p, L.q, L.c.ac, L.c.ar, L.c.at}, nx, ny, th};
  for (auto &e : g_maps)
    if (e.used && e.key == key) return &e.maps;
  auto enc = tma::encoder();
  if (!enc) return nullptr;
  RowMaps m{};
  const void *src[kArrays] = {L.r, L.x, L.p, L.q, L.c.ac, L.c.ar, L.c.at};
  CUtensorMap *dst[kArrays] = {&m.r, &m.x, &m.p, &m.q, &m.ac, &m.ar, &m.at};
  for (int k = 0; k < kArrays; ++k)
    if (!tma::encode(enc, dst[k], src[k], false, nx, ny, 32, th)) return nullptr;
  MapEntry &e = g_maps[g_maps_next];
  g_maps_next = (g_maps_next + 1) % kMapCache;
  e.key = key;
  e.maps = m;
  e.used = true;
  return &e.maps;
}

}  // namespace

bool pass_b_tma_eligible(const PassBLaunch &L) {
  const TileGeom &tg = L.tg;
  if (tg.xs != 0 || tg.tm != tg.wseg || (tg.tm != 8 && tg.tm != 16 && tg.tm != 32)) return false;
  if (tg.th < 1 || tg.th > kHM || tg.hmax != tg.th) return false;
  if (tg.nx % 4 != 0 || tg.nx < 32 || tg.ny < tg.th) return false;
  if (tg.grp_f32 || L.blocks < 1 || (size_t)L.blocks * 3 > L.partials_n) return false;
  for (const void *p : {(const void *)L.x, (const void *)L.p, (const void *)L.r,
                        (const void *)L.q, (const void *)L.c.ac, (const void *)L.c.ar,
                        (const void *)L.c.at, (const void *)L.mats})
    if (!p || !tma::aligned16(p)) return false;
  // the maps are cached: the launch that follows finds them
  return row_maps(L) != nullptr;
}

int pass_b_tma_launch(const PassBLaunch &L) {
  if (!pass_b_tma_eligible(L)) return SEVP_BAD_ARG;
  const RowMaps *mp = row_maps(L);
  if (!mp) return SEVP_BAD_ARG;
  auto kern = k_pass_b_tma<kHM>;
  const size_t smem = (size_t)kTileWarps * stage_bytes(L.tg.tm) + 128;
  static size_t set_smem = 0;
  if (set_smem != smem) {
    SEVP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set_smem = smem;
  }
  kern<<<L.blocks, kTileWarps * 32, smem, L.stream>>>(*mp, L.tg, L.mats, L.x, L.r, L.z, L.st,
                                                      L.partials, L.ticket);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

}  // namespace sevp
