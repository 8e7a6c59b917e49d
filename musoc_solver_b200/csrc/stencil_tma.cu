// PCG pass A with TMA-staged tiles: p = z + beta p_old, q = A p and the
// partial sums of p.q (the pass of k_stencil<OpPassA>, see solver.cu).
//
// The column-walking k_stencil spends most of its issue slots on address
// arithmetic, predicated loads and shuffles (about 90 instructions per grid
// point for 28 bytes moved).  Here the tensor memory accelerator moves every
// array of a 64 x 32 tile, with its halo, into shared memory: one thread
// issues a handful of 2-D bulk copies per tile, two or three tiles are in
// flight per CTA (an mbarrier per stage counts their bytes), and the 256
// threads then read the five-point neighbourhoods from shared memory.
//
// Boxes of a tile with origin (x0, j0) (x0 a multiple of 64, so every box's
// first column is 16-byte aligned, as a tensor copy requires):
//   z, p_old  (64 + 2h) x 34 at (x0 - h, j0 - 1), h = 16 bytes / sizeof(V)
//   AC        64 x 32 at (x0, j0)
//   AR        68 x 32 at (x0 - 4, j0)       (its column x0 - 1 is AL of x0)
//   AT        64 x 33 at (x0, j0 - 1)       (its row j0 - 1 is AB of row j0)
//   AL, AB    64 x 32 at (x0, j0)           (only for a nonsymmetric operator)
// Points outside the grid arrive as zeros (the copy's fill), which is the
// operator's zero data outside the domain; on a grid periodic in x the two
// tiles at the seam patch the wrapped halo column with plain loads.
//
// Waits on the stage barriers are bounded: a wait that gives up marks the
// pass failed (the finisher then reports SEVP_TIMEOUT) and the CTA still
// waits, with the same bound, for the copies it issued before it exits.
#include <algorithm>

#include "solver_core.cuh"
#include "tma_util.cuh"

namespace sevp {

namespace {

constexpr int kTW = 64, kTH = 32;   // output tile
constexpr int kThreads = 256;       // 4 row groups of 8 rows x 64 columns
constexpr int kRowsPerThread = kTH / (kThreads / kTW);
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::smem_u32;

__host__ __device__ constexpr uint32_t round128(uint32_t b) { return (b + 127u) & ~127u; }

// Shared-memory layout of one stage.
template <typename V, bool SYM>
struct Stage {
  static constexpr int kH = 16 / (int)sizeof(V);  // vector halo columns on each side
  static constexpr int kBW = kTW + 2 * kH;        // vector box width
  static constexpr uint32_t kVec = round128(kBW * (kTH + 2) * sizeof(V));
  static constexpr uint32_t kAC = round128(kTW * kTH * 4);
  static constexpr uint32_t kAR = round128((kTW + 4) * kTH * 4);
  static constexpr uint32_t kAT = round128(kTW * (kTH + 1) * 4);
  static constexpr uint32_t kOff_z = 0, kOff_p = kVec, kOff_ac = 2 * kVec,
                            kOff_ar = kOff_ac + kAC, kOff_at = kOff_ar + kAR,
                            kOff_al = kOff_at + kAT, kOff_ab = kOff_al + kAC;
  static constexpr uint32_t kBytes = kOff_al + (SYM ? 0 : 2 * kAC);
  // bytes the copies of one stage deliver (the full boxes, fill included)
  static constexpr uint32_t kTx = 2 * kBW * (kTH + 2) * sizeof(V) + kTW * kTH * 4 +
                                  (kTW + 4) * kTH * 4 + kTW * (kTH + 1) * 4 +
                                  (SYM ? 0 : 2 * kTW * kTH * 4);
};

struct Maps {
  CUtensorMap z, p, ac, ar, at, al, ab;
};

// Finisher of pass A: alpha = r.z / p.q (see PassAFin); a failed wait
// anywhere reports SEVP_TIMEOUT.
struct TmaFin {
  SolveState *st;
  __device__ void operator()(double (&s)[2]) {
    if (s[1] != 0.0) {
      st->status = SEVP_TIMEOUT;
      st->done = 1;
      return;
    }
    double v[1] = {s[0]};
    PassAFin{st}(v);
  }
};

template <typename V, bool SYM, int STAGES>
__global__ void __launch_bounds__(kThreads, 2)
    k_pass_a_tma(const __grid_constant__ Maps maps, GridDims g, const V *__restrict__ z,
                 const V *__restrict__ pold, const float *__restrict__ ar_g, V *pnew, V *q,
                 SolveState *st, double *partials, unsigned *ticket) {
  using S = Stage<V, SYM>;
  if (st->done) return;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  __shared__ __align__(8) uint64_t full[STAGES];
  const uint32_t sbase = (smem_u32(sm_raw) + 127u) & ~127u;
  unsigned char *sgen = sm_raw + (sbase - smem_u32(sm_raw));
  const int tid = threadIdx.x;
  const V beta = (V)st->beta;
  const bool first = st->beta == 0.0;
  const int nx = g.nx, ny = g.ny;
  const int TX = (nx + kTW - 1) / kTW, TY = (ny + kTH - 1) / kTH, ntile = TX * TY;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(smem_u32(&full[s]), 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int k) {  // the copies of this CTA's k-th tile
    const int t = blockIdx.x + k * gridDim.x;
    if (t >= ntile) return;
    const int x0 = (t % TX) * kTW, j0 = (t / TX) * kTH;
    const uint32_t st0 = sbase + (uint32_t)(k % STAGES) * S::kBytes;
    const uint32_t bar = smem_u32(&full[k % STAGES]);
    // the stage's previous tile was read and written through the generic
    // proxy (ordered before this thread by the CTA barrier)
    tma::fence_proxy_async();
    mbar_expect_tx(bar, S::kTx);
    tma::load_2d(st0 + S::kOff_z, &maps.z, x0 - S::kH, j0 - 1, bar);
    tma::load_2d(st0 + S::kOff_p, &maps.p, x0 - S::kH, j0 - 1, bar);
    tma::load_2d(st0 + S::kOff_ac, &maps.ac, x0, j0, bar);
    tma::load_2d(st0 + S::kOff_ar, &maps.ar, x0 - 4, j0, bar);
    tma::load_2d(st0 + S::kOff_at, &maps.at, x0, j0 - 1, bar);
    if (!SYM) {
      tma::load_2d(st0 + S::kOff_al, &maps.al, x0, j0, bar);
      tma::load_2d(st0 + S::kOff_ab, &maps.ab, x0, j0, bar);
    }
  };
  const int nmine = blockIdx.x < ntile ? (ntile - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0)
    for (int k = 0; k < STAGES - 1 && k < nmine; ++k) issue(k);
  double acc[2] = {0.0, 0.0};
  bool failed = false;
  int kfail = nmine;  // first tile whose wait gave up
  const int tx = tid % kTW, ty = tid / kTW;
  for (int k = 0; k < nmine; ++k) {
    if (tid == 0 && k + STAGES - 1 < nmine) issue(k + STAGES - 1);
    const int t = blockIdx.x + k * gridDim.x;
    const int x0 = (t % TX) * kTW, j0 = (t / TX) * kTH;
    unsigned char *sp = sgen + (size_t)(k % STAGES) * S::kBytes;
    V *zb = reinterpret_cast<V *>(sp + S::kOff_z);
    V *pb = reinterpret_cast<V *>(sp + S::kOff_p);
    float *sac = reinterpret_cast<float *>(sp + S::kOff_ac);
    float *sar = reinterpret_cast<float *>(sp + S::kOff_ar);
    float *sat = reinterpret_cast<float *>(sp + S::kOff_at);
    float *sal = reinterpret_cast<float *>(sp + S::kOff_al);
    float *sab = reinterpret_cast<float *>(sp + S::kOff_ab);
    if (!mbar_wait(smem_u32(&full[k % STAGES]), (unsigned)(k / STAGES) & 1u)) failed = true;
    if (__syncthreads_or(failed)) {
      failed = true;
      kfail = k;
      break;
    }
    {
      // periodic seam: the halo column across it wraps around the grid
      if (g.periodic && (x0 == 0 || x0 + kTW >= nx)) {
        for (int e = tid; e < 2 * (kTH + 2); e += kThreads) {
          const int row = e % (kTH + 2), side = e / (kTH + 2);
          const int j = j0 - 1 + row;
          if (j < 0 || j >= ny) continue;
          if (side == 0 && x0 == 0) {
            const size_t gi = (size_t)j * nx + (nx - 1);
            zb[row * S::kBW + S::kH - 1] = z[gi];
            pb[row * S::kBW + S::kH - 1] = pold[gi];
            if (SYM && row >= 1 && row <= kTH) sar[(row - 1) * (kTW + 4) + 3] = ar_g[gi];
          }
          if (side == 1 && x0 + kTW >= nx) {
            const size_t gi = (size_t)j * nx;
            zb[row * S::kBW + (nx - x0) + S::kH] = z[gi];
            pb[row * S::kBW + (nx - x0) + S::kH] = pold[gi];
          }
        }
        __syncthreads();
      }
      // p = z + beta p_old on the tile and its halo, in place of z
      if (!first)
        for (int e = tid; e < S::kBW * (kTH + 2); e += kThreads) zb[e] = fma_rn(beta, pb[e], zb[e]);
      __syncthreads();
      // q = A p on the own points; p and q out
      const int col = x0 + tx;
      const int r0 = ty * kRowsPerThread;
      V vb = zb[r0 * S::kBW + tx + S::kH];
      V vc = zb[(r0 + 1) * S::kBW + tx + S::kH];
#pragma unroll
      for (int u = 0; u < kRowsPerThread; ++u) {
        const int r = r0 + u;
        const V va = zb[(r + 2) * S::kBW + tx + S::kH];
        const V vw = zb[(r + 1) * S::kBW + tx + S::kH - 1];
        const V ve = zb[(r + 1) * S::kBW + tx + S::kH + 1];
        const float cc = sac[r * kTW + tx];
        const float ce = sar[r * (kTW + 4) + tx + 4];
        const float cn = sat[(r + 1) * kTW + tx];
        float cw, cb;
        if (SYM) {
          cw = sar[r * (kTW + 4) + tx + 3];
          cb = sat[r * kTW + tx];
        } else {
          cw = sal[r * kTW + tx];
          cb = sab[r * kTW + tx];
        }
        const V av = stencil5(cb, vb, cw, vw, cc, vc, ce, ve, cn, va);
        const int j = j0 + r;
        if (col < nx && j < ny) {
          const size_t gi = (size_t)j * nx + col;
          pnew[gi] = vc;
          q[gi] = av;
          acc[0] += (double)vc * (double)av;
        }
        vb = vc;
        vc = va;
      }
    }
    __syncthreads();  // the stage is free for the copies of tile k + STAGES
  }
  if (failed && tid == 0) {
    // wait (bounded) for the copies still in flight before the CTA exits:
    // tiles kfail .. kfail + STAGES - 1 were issued and not consumed
    for (int k = kfail; k < nmine && k < kfail + STAGES; ++k)
      mbar_wait(smem_u32(&full[k % STAGES]), (unsigned)(k / STAGES) & 1u);
  }
  acc[1] = failed ? 1.0 : 0.0;
  TmaFin fin{st};
  reduce_and_finish<2>(acc, partials, ticket, fin);
}

using tma::aligned16;
using tma::encode;
using tma::encoder;

// Tensor maps of recent launches (a solve alternates between two p buffers;
// a few contexts may share the thread).
struct MapKey {
  const void *p[7];
  int nx, ny, fp64;
  bool operator==(const MapKey &o) const {
    for (int k = 0; k < 7; ++k)
      if (p[k] != o.p[k]) return false;
    return nx == o.nx && ny == o.ny && fp64 == o.fp64;
  }
};
struct MapEntry {
  MapKey key;
  Maps maps;
  bool used;
};
constexpr int kMapCache = 16;
thread_local MapEntry g_maps[kMapCache];
thread_local int g_maps_next = 0;

template <typename V, bool SYM>
const Maps *tensor_maps(const PassALaunch<V> &L) {
  using S = Stage<V, SYM>;
  const bool f64 = sizeof(V) == 8;
  const int nx = L.g.nx, ny = L.g.ny;
  const MapKey key{{L.z, L.pold, L.c.ac, L.c.ar, L.c.at, SYM ? nullptr : L.c.al,
                    SYM ? nullptr : L.c.ab},
                   nx, ny, f64 ? 1 : 0};
  for (auto &e : g_maps)
    if (e.used && e.key == key) return &e.maps;
  auto enc = encoder();
  if (!enc) return nullptr;
  Maps m{};
  if (!encode(enc, &m.z, L.z, f64, nx, ny, S::kBW, kTH + 2) ||
      !encode(enc, &m.p, L.pold, f64, nx, ny, S::kBW, kTH + 2) ||
      !encode(enc, &m.ac, L.c.ac, false, nx, ny, kTW, kTH) ||
      !encode(enc, &m.ar, L.c.ar, false, nx, ny, kTW + 4, kTH) ||
      !encode(enc, &m.at, L.c.at, false, nx, ny, kTW, kTH + 1))
    return nullptr;
  if (!SYM && (!encode(enc, &m.al, L.c.al, false, nx, ny, kTW, kTH) ||
               !encode(enc, &m.ab, L.c.ab, false, nx, ny, kTW, kTH)))
    return nullptr;
  MapEntry &e = g_maps[g_maps_next];
  g_maps_next = (g_maps_next + 1) % kMapCache;
  e.key = key;
  e.maps = m;
  e.used = true;
  return &e.maps;
}

template <typename V, bool SYM>
int launch(const PassALaunch<V> &L) {
  using S = Stage<V, SYM>;
  // FP32 vectors: two CTAs per SM with two stages each (one CTA computes
  // while the other waits at a barrier); FP64: one CTA with three stages
  constexpr int kStages = 2 * (2 * S::kBytes + 128) <= 220 * 1024
                              ? 2
                              : (3 * S::kBytes + 128 <= 220 * 1024 ? 3 : 2);
  const Maps *mp = tensor_maps<V, SYM>(L);
  if (!mp) {
    sevp_internal_set_message("pass A: tensor map encoding failed");
    return SEVP_CUDA_ERROR;
  }
  const int nx = L.g.nx, ny = L.g.ny;
  auto kern = k_pass_a_tma<V, SYM, kStages>;
  const size_t smem = (size_t)kStages * S::kBytes + 128;
  static int slots = 0;
  if (!slots) {
    SEVP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, dev = 0, sms = 0;
    SEVP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    SEVP_CUDA_TRY(cudaGetDevice(&dev));
    SEVP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    slots = std::max(1, per_sm) * sms;
  }
  const int ntile = ((nx + kTW - 1) / kTW) * ((ny + kTH - 1) / kTH);
  const unsigned blocks =
      (unsigned)std::min<size_t>(std::min(ntile, slots), std::max<size_t>(1, L.partials_n / 2));
  kern<<<blocks, kThreads, smem, L.stream>>>(*mp, L.g, L.z, L.pold, L.c.ar, L.pnew, L.q, L.st,
                                             L.partials, L.ticket);
  SEVP_CUDA_TRY(cudaGetLastError());
  return SEVP_OK;
}

}  // namespace

// The tensor copies need rows of a multiple of 16 bytes and 16-byte
// aligned bases, and the driver must accept the maps; other grids use
// k_stencil.
template <typename V>
bool pass_a_tma_eligible(const PassALaunch<V> &L) {
  if (L.g.nx % 4 != 0 || L.g.nx < kTW / 2 || L.g.ny < 2) return false;
  for (const void *p : {(const void *)L.z, (const void *)L.pold, (const void *)L.c.ac,
                        (const void *)L.c.ar, (const void *)L.c.at, (const void *)L.pnew,
                        (const void *)L.q})
    if (!aligned16(p)) return false;
  if (!L.sym && (!aligned16(L.c.al) || !aligned16(L.c.ab))) return false;
  // the maps are cached: the launch that follows finds them
  return (L.sym ? tensor_maps<V, true>(L) : tensor_maps<V, false>(L)) != nullptr;
}

template <typename V>
int pass_a_tma_launch(const PassALaunch<V> &L) {
  if (!pass_a_tma_eligible(L)) return SEVP_BAD_ARG;
  return L.sym ? launch<V, true>(L) : launch<V, false>(L);
}
template bool pass_a_tma_eligible<float>(const PassALaunch<float> &);
template bool pass_a_tma_eligible<double>(const PassALaunch<double> &);
template int pass_a_tma_launch<float>(const PassALaunch<float> &);
template int pass_a_tma_launch<double>(const PassALaunch<double> &);

}  // namespace sevp
