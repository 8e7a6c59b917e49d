// Block-Jacobi tile SEVP: device structures shared by the precompute and the
// apply kernels.
//
// The grid (nx columns, ny rows; element (i, j) at j * nx + i, the memory
// order of the reference's column-major (I2, J2) arrays) is cut into tiles of
// at most tm x th points.  Tile (a, b) covers columns [a*tm, a*tm + mw) and
// rows [b*th, b*th + hh), clipped at the domain edge.  Inside a tile the
// equations are solved exactly with zero Dirichlet data outside the tile by
// SEVP marching in the north direction.  A tile of hh rows is split into nb
// sub-blocks whose boundaries are k_t = (t * hh) / nb, t = 0..nb; nb is set
// per tile so that the marching error growth, which depends on the local
// coefficient anisotropy (and is largest over land, where the free-surface
// term dominates the floored depths), stays bounded.  The tiles that share a
// warp (a group of tpw neighbours in a tile row) share nb.
//
// Influence data per tile, all FP64, mw x mw, element [k][n] at k * mw + n
// (k = input column, n = output column):
//   Sinv_t  t = 0..nb-1  inverse of the guess-row -> last-equation map of
//                        sub-block t (the reference's RINV after MATINV)
//   R1_t    t = 0..nb-2  minus Sinv_t times the guess-row -> top-row map
//                        (the reference's RINV1)
// stored consecutively: Sinv_0..Sinv_{nb-1}, R1_0..R1_{nb-2}.
//
// Shifted tilings (the second tiling of the overlapping Schwarz
// preconditioner): with a column shift xs, tile column a covers the grid
// columns (a*tm + n + xs) mod nx, n = 0..mw-1, i.e. the standard tiling of
// the grid rolled west by xs; the tile that reaches the last column wraps
// to column 0.  On a periodic grid that tile couples across the seam like
// any other column pair.  On a closed grid the tiling reads AL and AR planes
// whose couplings across the seam are zero, so that tile holds two
// independent pieces.
#pragma once
#include "common.cuh"

namespace sevp {

struct TileGeom {
  int nx, ny, tm, th, tx, ty;
  int wseg;   // lanes per tile segment: 8, 16 or 32 (>= tm)
  int tpw;    // tiles per warp = 32 / wseg
  int txg;    // tile groups per tile row = ceil(tx / tpw)
  int hmax;   // max tile height (= th)
  int nbmax;  // max sub-blocks per tile
  int xs;     // column shift of the tiling (0 <= xs < nx)
  const int *grp_nb;         // [ty * txg] sub-blocks of the tiles of one warp group
  const long long *moff;     // [ty * tx] offset of each tile's influence data
  // [ty * txg] 1 where the group's matrices are stored as FP32 in a
  // per-group-precision copy of the influence data (MixMat); may be null
  const unsigned char *grp_f32;
};

__host__ __device__ inline int tile_width(const TileGeom &g, int a) {
  int w = g.nx - a * g.tm;
  return w < g.tm ? (w > 0 ? w : 0) : g.tm;
}
__host__ __device__ inline int tile_height(const TileGeom &g, int b) {
  int h = g.ny - b * g.th;
  return h < g.th ? h : g.th;
}
__host__ __device__ inline int sub_start(int t, int hh, int nb) { return (t * hh) / nb; }
// Grid column of lane n of tile column a (n < tile_width; 0 otherwise).
__host__ __device__ inline int tile_col(const TileGeom &g, int a, int n) {
  int c = a * g.tm + n;
  if (c >= g.nx) return 0;
  c += g.xs;
  return c >= g.nx ? c - g.nx : c;
}

}  // namespace sevp
