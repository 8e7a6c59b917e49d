/*
 * sevp_b200.h -- C ABI of the B200 (sm_100a) SEVP barotropic elliptic solver.
 *
 * Two layers:
 *
 *  1. Fortran-compatible entry points.  Same names (gfortran mangling: lower
 *     case plus a trailing underscore), same argument lists and same array
 *     layouts as the reference routines; every argument is passed by
 *     reference and every array is a column-major HOST array.  A gfortran
 *     caller links them in place of the reference objects.  They copy their
 *     inputs to the GPU, run the computation there and copy the outputs
 *     back.  The reference stops the program on failure; these return
 *     normally and record a status that sevp_last_status() reports.
 *
 *  2. A native API on DEVICE pointers: an operator context holding the
 *     coefficients and the tile influence data, and status-returning solves
 *     (FP64 PCG, or FP32 PCG inside FP64 iterative refinement).
 *
 * Reference paths are relative to the reference project; M/ is
 * MAIN/template/GLOBAL/src/ and P/ is PREP/template/GLOBAL/src/.
 *
 * Array conventions (as in the reference):
 *   coefficients AX,AY,BB,CX,CY = west, south, centre, east, north
 *   (called as AL,AB,AC,AR,AT), REAL*4 (I2, J2);
 *   X, H REAL*8 (I0, J0) with one ghost cell on each side (I0 = I2 + 2);
 *   F, S REAL*4 (I2, J2); RINV REAL*8 (I2, I2, NB0); RINV1 (I2, I2, NB0-1);
 *   IE INTEGER (NB0) block boundaries.
 */
#ifndef SEVP_B200_H
#define SEVP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SEVP_OK 0
#define SEVP_MAXITER 1     /* iteration cap reached before the tolerance */
#define SEVP_BREAKDOWN 2   /* a Krylov scalar became zero */
#define SEVP_NONFINITE 3   /* NaN or Inf in a residual or an input */
#define SEVP_TIMEOUT 4     /* a bounded device wait gave up */
#define SEVP_BAD_ARG 5     /* invalid size, pointer or option */
#define SEVP_CUDA_ERROR 6  /* a CUDA runtime call failed (see sevp_last_error) */
#define SEVP_SINGULAR 7    /* an influence matrix had a zero pivot */
#define SEVP_NONSYMMETRIC 8 /* conjugate gradients asked of a nonsymmetric operator */

const char *sevp_status_string(int status);
/* Text of the last CUDA error seen by the library (empty if none). */
const char *sevp_last_error(void);
/* Status of the most recent Fortran-compatible call in this thread. */
int sevp_last_status(void);
/* Periodic east-west ghost refresh used by the Krylov drop-ins; the reference
 * compiles it in with FLAG_PERIODIC_WE (M/sevp.f90:780-786).  Default 1. */
void sevp_set_periodic_we(int periodic);
int sevp_get_periodic_we(void);
/* Device copies of the read-only inputs of rep1_, rep_, repbir_ and
 * repbir_period_ (coefficients, RINV, RINV1, IE) kept between calls
 * (enable != 0), keyed by host address and size: a model that reads the EVP
 * file once and calls REP1 every step (M/fs_GLOBAL.f90:1852) then copies
 * only F, X, H and the DUM workspaces per call.  The caller promises that
 * those arrays keep their values while caching is on.  While it is on, the
 * device blocks of every drop-in's per-call copies (workspaces, X, F, the
 * Krylov drop-ins' vectors) are also kept and reused, so repeated calls make
 * no cudaMalloc / cudaFree.  sevp_dropin_cache(0) frees the copies and the
 * blocks and turns caching off (the default).  Not part of the reference
 * interface. */
int sevp_dropin_cache(int enable);

/* ------------------------------------------- Fortran-compatible drop-ins */

/* Replaces SUBROUTINE REP1, M/sevp.f90:11-107 (periodic, full width). */
void rep1_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
           const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
           const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
           const int *nblk);

/* Replaces SUBROUTINE REP, M/sevp.f90:335-438 (non-periodic, full width). */
void rep_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
          const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
          const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
          const int *nblk);

/* Replaces SUBROUTINE REPBIR, M/sevp.f90:218-328 (one strip of M2 columns;
 * coefficients with leading dimension I2, X with I0, F and RINV with M2). */
void repbir_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
             const double *rinv, const double *rinv1, double *dum0, double *dum1, double *dum2,
             const float *f, double *h, double *x, const int *ie, const int *i0, const int *i2,
             const int *m0, const int *m2, const int *nblk);

/* Replaces SUBROUTINE REPBIR_PERIOD, M/sevp.f90:109-217 (defined for M0 == I0). */
void repbir_period_(const float *ax, const float *ay, const float *bb, const float *cx,
                    const float *cy, const double *rinv, const double *rinv1, double *dum0,
                    double *dum1, double *dum2, const float *f, double *h, double *x,
                    const int *ie, const int *i0, const int *i2, const int *m0, const int *m2,
                    const int *nblk);

/* Replaces the internal PRE1 of P/prep_GLOBAL.f90:327-386 (called at :271). */
void pre1_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
           double *rinv, double *rinv1, double *h, const int *ie, const int *i0, const int *i2,
           const int *nblk);

/* Replaces the internal PRE of P/prep_GLOBAL.f90:457-513 (called at :292, :315). */
void pre_(const float *ax, const float *ay, const float *bb, const float *cx, const float *cy,
          double *rinv, double *rinv1, double *h, const int *ie, const int *i2, const int *m0,
          const int *m2, const int *nblk);

/* Replaces the internal MATINV of P/prep_GLOBAL.f90:516-568 (no pivoting). */
void matinv_(double *b, const int *n);

/* Replaces subroutine p_sqprod, M/sevp.f90:696-713: r(interior) = A x. */
void p_sqprod_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
               const double *x, double *r, const int *i2, const int *j2);

/* Replaces subroutine p_sqprod_T, M/sevp.f90:714-742. */
void p_sqprod_t_(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const double *x, double *r, const int *i2, const int *j2);

/* Replaces subroutine p_inprod, M/sevp.f90:743-757. */
void p_inprod_(const double *r, const double *p, double *tp, const int *i2, const int *j2);

/* Replaces subroutine solver_boundary_update, M/sevp.f90:773-787. */
void solver_boundary_update_(double *x, const int *i2, const int *j2);

/* Replaces subroutine p_bicgstab_le, M/sevp.f90:443-552. */
void p_bicgstab_le_(const float *al, const float *ab, const float *ac, const float *ar,
                    const float *at, const float *b, double *x, const float *cl, const float *cb,
                    const float *cc, const float *cr, const float *ct, const int *i2,
                    const int *j2);

/* Replaces subroutine p_csi, M/sevp.f90:553-616. */
void p_csi_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
            const double *mineig, const double *maxeig, const float *b, double *x,
            const float *cl, const float *cb, const float *cc, const float *cr, const float *ct,
            const int *i2, const int *j2);

/* Replaces subroutine lanczos, M/sevp.f90:618-694 (figi :838-904 and ratqr
 * :906-1006 run on the host: they act on a 10x10 tridiagonal matrix). */
void lanczos_(const float *al, const float *ab, const float *ac, const float *ar, const float *at,
              double *mineig, double *maxeig, const int *i2, const int *j2);

/* Overlapping-strip Schwarz sweeps of FS_SOLVER, M/fs_GLOBAL.f90:1904-1966
 * (FL_EVP_STP == 1): niter sweeps over nbir strips of REPBIR.  RINV is
 * (IBIR*IBIR, NB0, NBIR) and RINV1 (IBIR*IBIR, NB0-1, NBIR) as written by
 * PREP; xx ((IBIR+2), J0) is the caller's persistent wrap-strip scratch.
 * fix_wrap = 0 reproduces the reference, which copies the wrapped strip's
 * side boundaries for rows 1..J2 only (:1925-1926); fix_wrap = 1 also copies
 * rows J2+1 and J2+2. */
void sevp_bir_sweeps_(const float *al, const float *ab, const float *ac, const float *ar,
                      const float *at, const float *s, const double *rinv, const double *rinv1,
                      double *x, double *xx, const int *ie, const int *i2, const int *j2,
                      const int *nb0, const int *nbir, const int *niter, const int *fix_wrap);

/* Influence precompute for all BIR strips, P/prep_GLOBAL.f90:272-318. */
void sevp_pre_strips_(const float *al, const float *ab, const float *ac, const float *ar,
                      const float *at, double *rinv, double *rinv1, const int *ie, const int *i2,
                      const int *j2, const int *nb0, const int *nbir);

/* ------------------------------------------------ PREP's preprocessing */

/* Row-block boundaries IE(NB0) of the reference's SEVP blocks,
 * P/prep_GLOBAL.f90:148-168: NN = ANINT(REAL(J2) / REAL(NB0)),
 * IE(N) = MIN(1 + NN N, J1), then the validity test of :156-165 and
 * IE(NB0) = J1.  Host code, no GPU.  Where the reference prints "IE(NB1),J1
 * not properly defined" and stops, this returns SEVP_BAD_ARG with that text
 * in sevp_last_error (ie is still filled).  nb0 >= 2; dimen 2 or 3. */
int sevp_block_partition(int j2, int nb0, int dimen, int *ie);

/* Five-point coefficients of the barotropic operator, PREP's assembly
 * (P/prep_GLOBAL.f90:170-261) on the GPU, equal to the reference's REAL*4
 * results bit for bit.  DEVICE arrays with the reference's shapes
 * (column-major): ODX, ODY, OCS (J0), CSV, ODYV (J1), ODZ (K1) REAL*4;
 * IU (I0, J0, K1) and IV (I0, J1, K1) INTEGER*2 layer masks (read for
 * K = 2..K1; unused when dimen == 2 or k1 == 1, may then be NULL).
 * dimen 2: the constant couplings of :170-181 (ODX(1), ODY(1), ODZ(1) only);
 * dimen 3: the top layer all water plus the masked lower layers (:183-212).
 * nbir == 1: closed side walls and the pressure pin AB(I2/2,1) = AB(I2/2,2)
 * (:214-230).  gamma is the free-surface term (1/(0.5 DT^2 G) under FLAG_FS,
 * :232-236, else 0).  idealised != 0 applies the reference's constant test
 * stencil with Neumann north and south rows (:244-258), which the reference
 * as shipped always applies.  Outputs AL, AR, AB, AT, AC (I2, J2). */
int sevp_prep_assemble(int i2, int j2, int k1, int dimen, const float *odx, const float *ody,
                       const float *csv, const float *ocs, const float *odyv, const float *odz,
                       const int16_t *iu, const int16_t *iv, int nbir, float gamma, int idealised,
                       float *al, float *ar, float *ab, float *at, float *ac, void *stream);
/* The same on HOST arrays (copied to the GPU and back inside the call). */
int sevp_prep_assemble_host(int i2, int j2, int k1, int dimen, const float *odx,
                            const float *ody, const float *csv, const float *ocs,
                            const float *odyv, const float *odz, const int16_t *iu,
                            const int16_t *iv, int nbir, float gamma, int idealised, float *al,
                            float *ar, float *ab, float *at, float *ac);

/* ---------------------------------------------------- native device API */

typedef struct sevp_ctx sevp_ctx;

/* Tile decomposition of the block-Jacobi SEVP preconditioner. */
typedef struct {
  int tile_m;   /* tile width in columns: 1..32 */
  int tile_h;   /* tile height in rows: 1..32 */
  int sub_rows; /* marching sub-block height in rows (>= 1) when no rule below applies */
  /* optional host array of ceil(ny / tile_h) heights, one per tile row */
  const int *sub_rows_by_tile_row;
  /* optional host array of ceil(ny/tile_h) * ceil(nx/tile_m) heights, one per
   * tile, tile rows first; takes precedence over the per-row array */
  const int *sub_rows_by_tile;
  /* > 1 and no array given: each tile's height is the largest s with z^s <=
   * growth_limit, where z + 1/z is the tile's largest (|AC|+|AL|+|AR|)/|AT|
   * (the worst-case amplification of one marched row) */
  double growth_limit;
} sevp_tiling;
/* Tile counts and the sub-blocks used by each tile (tiles sharing a warp use
 * their largest count); nb_per_tile may be NULL. */
int sevp_tile_layout(const sevp_ctx *ctx, int *tiles_x, int *tiles_y, int *nb_per_tile);

typedef struct {
  int precision;     /* 0: FP64 PCG; 1: FP32 PCG inside FP64 iterative refinement */
  double tol;        /* target ||b - A x||_2 / ||b||_2 evaluated in FP64 */
  int max_iter;      /* cap on the total number of PCG iterations */
  double inner_tol;  /* precision 1: relative reduction asked of each FP32 solve */
  int use_guess;     /* 1: x holds the initial guess on entry; 0: start from zero */
  int check_every;   /* PCG iterations between convergence reads by the host */
  int precond_fp32;  /* precision 1: FP32 copy of the influence matrices in the inner solve */
  int tol_abs;       /* 1: stop on ||b - A x||_2 <= tol (absolute, the reference's rule,
                        M/sevp.f90:482); 0: the relative test above */
  int method;        /* SEVP_METHOD_*: the outer iteration */
  int restart_inner; /* precision 1: 1 restarts the inner iteration at every FP64
                        residual; 0 (default) replaces the FP32 residual by the FP64 one
                        and continues: CG keeps its search direction (reliable
                        updates), Chebyshev its recurrence and last direction */
} sevp_solve_opts;
/* Outer iterations of sevp_solve. */
#define SEVP_METHOD_PCG 0     /* preconditioned CG, two grid passes per iteration */
/* Chebyshev iteration on the spectrum bounds [lmin, lmax] of M^-1 A
 * (precision 1, block-Jacobi tiles of at most 8 rows; needs
 * sevp_set_chebyshev_bounds).  No dot product feeds its next update, so
 * each iteration is ONE kernel launch that applies the operator to the
 * previous launch's direction inside the tile kernel (halo values read from
 * global memory) and then runs the tile SEVP solve.  The reference's P-CSI
 * (M/sevp.f90:553-616) is the unpreconditioned form. */
#define SEVP_METHOD_CHEB 1

typedef struct {
  int status;          /* SEVP_* */
  int iterations;      /* total PCG iterations */
  int refinements;     /* FP64 residual evaluations (precision 1) */
  double rel_residual; /* final ||b - A x|| / ||b||, FP64 */
  double abs_residual; /* final ||b - A x||, FP64 */
  double bnorm;        /* ||b||_2 */
  double ms;           /* device time of the solve */
} sevp_report;

/* Creates a context for an nx x ny interior grid (periodic in x if
 * periodic != 0) bound to a CUDA stream (NULL = default stream).  The
 * context is tied to the current device. */
int sevp_create(sevp_ctx **ctx, int nx, int ny, int periodic, void *stream);
int sevp_destroy(sevp_ctx *ctx);
/* Binds the five FP32 coefficient planes (device pointers, (nx, ny)
 * column-major, not copied: they must outlive the context's use) and
 * computes the tile influence data on the GPU. */
int sevp_set_operator(sevp_ctx *ctx, const float *al, const float *ab, const float *ac,
                      const float *ar, const float *at, const sevp_tiling *tiling);
/* 1 when the bound operator is exactly symmetric (AR(i,j) = AL(i+1,j),
 * AT(i,j) = AB(i,j+1)); the kernels then read only AC, AR and AT.  A
 * nonsymmetric operator can be applied and preconditioned, but sevp_solve
 * refuses it with SEVP_NONSYMMETRIC (CG needs a symmetric operator). */
int sevp_operator_symmetric(const sevp_ctx *ctx);
/* Operator of the FP64 residual passes, when it is not the operator bound
 * by sevp_set_operator (not part of the reference interface).  PREP's
 * coefficients (P/prep_GLOBAL.f90:170-244) are symmetric only after each row
 * J is scaled by 1 / (OCS(J+1) ODY(J+1)); p_sevp_pcg_ binds the scaled,
 * symmetrised planes with sevp_set_operator and the caller's own planes
 * here, with the row weights w (ny doubles, device; NULL: all 1).  Every
 * residual pass then forms ru = b - A x with these planes, scales it by w_j
 * for the PCG recursion, and tests ||ru|| (unscaled) against the tolerance,
 * so the solve converges to the caller's operator.  al == NULL unbinds. */
int sevp_set_residual_operator(sevp_ctx *ctx, const float *al, const float *ab, const float *ac,
                               const float *ar, const float *at, const double *row_weight);
/* force != 0: always read all five planes (call before sevp_set_operator). */
/* CUDA graphs for the FP32 inner PCG iterations of mixed solves (default on):
 * one check interval (check_every iterations of the two passes) is captured
 * once per context on a private stream and replayed on the context stream.
 * Not part of the reference interface. */
int sevp_set_graphs(sevp_ctx *ctx, int enable);
/* Kernel of the PCG's stencil pass (p = z + beta p_old, q = A p, p.q):
 * SEVP_PASS_A_TILES (default) stages 64 x 32 tiles and their halos in shared
 * memory with tensor copies where the grid allows it (nx a multiple of 4,
 * 16-byte aligned buffers; other grids fall back);
 * SEVP_PASS_A_COLUMNS walks columns with warp shuffles.  Both give the same
 * p and q bit for bit.  Not part of the reference interface. */
#define SEVP_PASS_A_TILES 0
#define SEVP_PASS_A_COLUMNS 1
int sevp_set_pass_a_kernel(sevp_ctx *ctx, int kind);
/* Kernel of the FP32 PCG's tile pass (x += alpha p, r -= alpha q, z = M^-1 r,
 * r.z, r.r) on block-Jacobi tiles of at most 6 rows:
 * SEVP_PASS_B_REGISTERS (default) loads each task's rows and influence
 * matrices into registers when it starts; SEVP_PASS_B_STAGED has every warp keep
 * a shared-memory stage that tensor copies fill with the next task's rows
 * and matrices while it marches the current one, where the tiling and the
 * buffers allow it (tiles 8, 16 or 32 columns wide, nx a multiple of 4,
 * symmetric operator, FP64 influence data; otherwise the register kernel
 * runs).  Both give the same x, r and z bit for bit.  Not part of the
 * reference interface. */
#define SEVP_PASS_B_REGISTERS 0
#define SEVP_PASS_B_STAGED 1
int sevp_set_pass_b_kernel(sevp_ctx *ctx, int kind);
/* Mixed-precision PCG with block-Jacobi tiles (restart_inner 0): after each
 * FP64 residual the stopped run resumes with the preconditioned residual of
 * its last pass, one step behind, when the distance between its recursive
 * FP32 residual and the replaced one is at most max_rel_dev times the
 * replaced residual's norm (default 0.3); otherwise, and always with the
 * Schwarz preconditioner, the replaced residual is preconditioned afresh
 * before CG goes on along its last direction.  max_rel_dev <= 0 never
 * resumes.  Not part of the reference interface. */
int sevp_set_resume_check(sevp_ctx *ctx, double max_rel_dev);
/* The kernel the context's last FP32 PCG tile pass ran: SEVP_PASS_B_REGISTERS
 * or SEVP_PASS_B_STAGED, -1 before the first.  Test hook; not part of the
 * reference interface. */
int sevp_pass_b_kernel_used(const sevp_ctx *ctx);
/* One stencil pass on caller device buffers with the context's operator and
 * pass A kernel: p = z + beta p_old (z alone when beta == 0), q = A p, and
 * p.q through pq_out.  Test hook; not part of the reference interface. */
int sevp_pass_a_f32(sevp_ctx *ctx, const float *z, const float *pold, double beta, float *pnew,
                    float *q, double *pq_out);
int sevp_pass_a_f64(sevp_ctx *ctx, const double *z, const double *pold, double beta,
                    double *pnew, double *q, double *pq_out);

int sevp_set_full_coefficients(sevp_ctx *ctx, int force);
/* Device bytes held by the tile influence data (block-Jacobi tiling). */
long long sevp_influence_bytes(const sevp_ctx *ctx);
/* Influence-data precision chosen per warp group of tiles for the FP32
 * inner iterations of mixed solves and sevp_precondition_f32 (not part of
 * the reference interface).  growth_limit > 1: the groups whose every tile
 * has a marching growth bound z^s <= growth_limit over its sub-blocks of s
 * rows (z as in sevp_tiling.growth_limit) read their matrices as FP32, the
 * others keep FP64; their mat-vecs then read half the bytes.  The inverse
 * influence matrices are about as ill-conditioned as that growth, so the
 * limit bounds the relative error FP32 storage brings into a tile's
 * correction (about 6e-8 times the limit).  growth_limit <= 1 turns it off
 * (the default).  A solve that sets sevp_solve_opts.precond_fp32 still
 * reads every tile as FP32.  Kept across sevp_set_operator (the choice is
 * rebuilt for the new operator). */
int sevp_set_influence_fp32(sevp_ctx *ctx, double growth_limit);
/* Warp groups of the block-Jacobi tiling reading FP32 influence data, all
 * groups, and the influence bytes one preconditioner pass reads with that
 * choice (sevp_influence_bytes when it is off).  Pointers may be NULL. */
int sevp_influence_fp32_groups(const sevp_ctx *ctx, int *fp32_groups, int *groups,
                               long long *bytes_per_pass);
/* Overlapping Schwarz preconditioner (not part of the reference interface;
 * the reference's BIR method, M/fs_GLOBAL.f90:1902-1966, sweeps overlapping
 * strips with 50 % overlap as a stand-alone solver).  shift != 0 adds a
 * second tiling, the first one rolled west by `shift` columns (shift < 0:
 * the shift nearest tile_m / 2 whose tile edges all fall inside tiles of
 * the first tiling), and makes every preconditioner application the
 * symmetric multiplicative Schwarz sweep over the two tilings:
 *   z1 = M_a r,  z2 = M_b (r - A z1),  z = z1 + z2 + M_a (r - A (z1 + z2)).
 * The residuals are formed from the couplings across the previous tiling's
 * boundaries.  Tiles must be at most 8 rows high.  shift = 0 returns to the
 * block-Jacobi preconditioner.  Kept across sevp_set_operator.  Returns
 * SEVP_BAD_ARG when no valid shift exists or the tiles are too high. */
int sevp_set_schwarz(sevp_ctx *ctx, int shift);
/* PCG coefficient record (not part of the reference interface; the
 * reference estimates extreme eigenvalues with a 10-step Lanczos run,
 * M/sevp.f90:618-694).  cap > 0: every later FP64 solve (precision 0)
 * writes alpha_j and beta_j of its first PCG run, j = 1..cap, into a device
 * buffer; cap = 0 stops recording and frees the buffer.  The CG-Lanczos
 * tridiagonal built from them has the extreme Ritz values of the
 * preconditioned operator M^-1 A. */
int sevp_record_coefficients(sevp_ctx *ctx, int cap);
/* Copies the last recorded coefficients to host arrays of cap entries;
 * *count = iterations recorded (0 when nothing was recorded). */
int sevp_read_coefficients(sevp_ctx *ctx, double *alpha, double *beta, int cap, int *count);
/* Column shift of the second tiling, 0 when the preconditioner is block-Jacobi. */
int sevp_schwarz_shift(const sevp_ctx *ctx);
/* Device bytes held by the second tiling's influence data. */
long long sevp_schwarz_influence_bytes(const sevp_ctx *ctx);
/* Spectrum bounds of the preconditioned operator M^-1 A used by
 * SEVP_METHOD_CHEB (0 < lmin < lmax).  sevp_estimate_bounds runs one FP64
 * PCG solve of b (to 1e-13, not changing any caller buffer) and returns the
 * extreme Ritz values of its CG-Lanczos tridiagonal (the reference gets its
 * bounds from a 10-step Lanczos run and RATQR, M/sevp.f90:618-694); they
 * lie inside the spectrum, so widen them a little before setting them. */
int sevp_set_chebyshev_bounds(sevp_ctx *ctx, double lmin, double lmax);
int sevp_estimate_bounds(sevp_ctx *ctx, const double *b, double *lmin, double *lmax,
                         int *iterations);
/* One launch of the Chebyshev iteration on caller buffers (FP32 device
 * vectors of the grid), for testing the kernel against a host restatement;
 * not part of the reference interface.  iter = k (0: the first launch, which
 * ignores din and forms d_0 = M^-1 r / theta); theta = (lmax + lmin) / 2,
 * delta = (lmax - lmin) / 2, rho = rho_k.  din is d_k, dout receives d_{k+1};
 * x += d_k and r -= A d_k in place.  *rr_out = ||r||^2 after the update. */
int sevp_cheb_step(sevp_ctx *ctx, int iter, double theta, double delta, double rho,
                   const float *din, float *dout, float *x, float *r, double *rr_out);
/* Solves A x = b (device pointers, (nx, ny) column-major FP64). */
int sevp_solve(sevp_ctx *ctx, const double *b, double *x, const sevp_solve_opts *opts,
               sevp_report *report);
/* Same with host buffers: copies b (and the guess) in and x out. */
int sevp_solve_host(sevp_ctx *ctx, const double *b_host, double *x_host,
                    const sevp_solve_opts *opts, sevp_report *report);
/* Warm starts for a time sequence of solves. */
#define SEVP_GUESS_ZERO 0     /* x = 0 */
#define SEVP_GUESS_PREVIOUS 1 /* x = eta_{n-1} */
#define SEVP_GUESS_LINEAR 2   /* x = 2 eta_{n-1} - eta_{n-2} */
#define SEVP_GUESS_LEARNED 3  /* x = network(eta_{n-1}, eta_{n-2}, b_n), see sevp_set_warmstart */
/* A learned warm start: writes the guess x (device) from the two previous
 * solutions and the right-hand side on the given CUDA stream; returns SEVP_*. */
typedef int (*sevp_warmstart_fn)(void *user, const double *eta1, const double *eta2,
                                 const double *b, double *x, int nx, int ny, void *stream);
int sevp_set_warmstart(sevp_ctx *ctx, sevp_warmstart_fn fn, void *user, int launches_per_call);
/* One step of a sequence: x = guess(eta1, eta2, b), then the solve of A x = b
 * from that guess (device pointers; eta1/eta2 may be NULL when unused). */
int sevp_solve_step(sevp_ctx *ctx, const double *b, const double *eta1, const double *eta2,
                    double *x, int guess_mode, const sevp_solve_opts *opts, sevp_report *report);
/* Time stepping with the history held on the device (not part of the
 * reference interface; the reference's FS_SOLVER passes the previous
 * solution in X, M/fs_GLOBAL.f90:1852).  The context keeps the last two
 * solutions in device memory, so a step copies only b in and x out:
 * sevp_step_host solves A x = b from the guess of guess_mode built from
 * that history (zero while it is empty, the previous solution while it holds
 * one) and then makes x the newest solution.  sevp_step_history loads a
 * history from host arrays (eta2 may be NULL; both NULL empties it). */
int sevp_step_history(sevp_ctx *ctx, const double *eta1_host, const double *eta2_host);
int sevp_step_host(sevp_ctx *ctx, const double *b_host, double *x_host, int guess_mode,
                   const sevp_solve_opts *opts, sevp_report *report);
/* Asynchronous stepping with the same device history.  sevp_step_submit
 * stages b (or takes the copy that sevp_step_prefetch started), solves, and
 * starts copying x out on a copy stream; it returns when the solve is done,
 * before x has arrived.  sevp_step_wait waits for the submitted x copies.
 * Prefetching step n+1's b before submitting step n overlaps that copy with
 * the solve.  b_host and x_host must be pinned and left untouched until
 * sevp_step_wait returns. */
int sevp_step_prefetch(sevp_ctx *ctx, const double *b_host);
int sevp_step_submit(sevp_ctx *ctx, const double *b_host, double *x_host, int guess_mode,
                     const sevp_solve_opts *opts, sevp_report *report);
int sevp_step_wait(sevp_ctx *ctx);
/* Same with host buffers: copies b, eta1, eta2 in and x out inside the call. */
int sevp_solve_step_host(sevp_ctx *ctx, const double *b_host, const double *eta1_host,
                         const double *eta2_host, double *x_host, int guess_mode,
                         const sevp_solve_opts *opts, sevp_report *report);
/* y = A x on the unpadded grid (device pointers). */
int sevp_apply(sevp_ctx *ctx, const double *x, double *y);
/* z = M^{-1} r: tiles solved by SEVP marching (device); block-Jacobi, or the
 * Schwarz sweep after sevp_set_schwarz. */
int sevp_precondition(sevp_ctx *ctx, const double *r, double *z);
/* Same in the FP32 vector format of the mixed-precision inner solve. */
int sevp_precondition_f32(sevp_ctx *ctx, const float *r, float *z);
/* Writes ||b - A x||_2 / ||b||_2 (FP64). */
int sevp_relative_residual(sevp_ctx *ctx, const double *b, const double *x, double *relres);
/* Number of kernel launches issued by this context since creation. */
long long sevp_kernel_launches(const sevp_ctx *ctx);
/* Per-kernel-class device timing with CUDA events on the context stream:
 * enable != 0 starts (and zeroes) it.  sevp_profile_read fills ms[4] and
 * count[4] for class 0 = tile pass B (the x, r update and the first tile
 * solve; with dot products unless the Schwarz sweep follows),
 * 1 = stencil passes (apply, pass A, residuals), 2 = tile precondition
 * without update, 3 = Schwarz stages on boundary couplings. */
int sevp_profile(sevp_ctx *ctx, int enable);
int sevp_profile_read(sevp_ctx *ctx, double *ms, long long *count);

/* ------------------------- fast solver behind the reference's solver call */

/* Options of p_sevp_pcg_ (process-wide; sevp_fs_default_options fills the
 * defaults, which apply until sevp_fs_set_options is called). */
typedef struct {
  int precision;       /* 0: FP64 PCG; 1 (default): FP32 PCG inside FP64 refinement */
  int tol_abs;         /* 0 (default): ||S - A X|| / ||S|| <= tol;
                          1: ||S - A X|| <= tol, the reference's rule (M/sevp.f90:482) */
  double tol;          /* default 1e-12 (the reference's absolute rule uses 1e-8) */
  int max_iter;        /* default 5000 */
  double inner_tol;    /* precision 1: reduction asked of each FP32 solve, default 1e-5 */
  int tile_m, tile_h;  /* tile shape of the SEVP preconditioner, default 16 x 6 */
  double growth_limit; /* marching growth bound per sub-block, default 1e10 */
  int schwarz;         /* 1: overlapping Schwarz preconditioner (tiles <= 8 rows) */
  int verify;          /* 1 (default): hash the coefficient planes on every call and
                          rebuild the cached operator when they changed; 0: trust that
                          the arrays at the same addresses still hold the same values */
  int method;          /* SEVP_METHOD_* */
} sevp_fs_options;
void sevp_fs_default_options(sevp_fs_options *o);
int sevp_fs_set_options(const sevp_fs_options *o);

/* Same argument list as subroutine p_bicgstab_le, M/sevp.f90:443-552
 * (called at M/fs_GLOBAL.f90:1853, 1968, 2024), so a Fortran caller swaps
 * the call's name: al..at and cl..ct REAL*4 (i2, j2) PREP planes (not
 * symmetric: row J carries OCS(J+1) ODY(J+1), P/prep_GLOBAL.f90:186-189),
 * b REAL*4 (i2, j2), x REAL*8 (i2+2, j2+2) in/out with its ghost ring as
 * boundary data.  Solves A x = b with the tile-SEVP preconditioned CG on
 * the GPU: row weights that make the operator symmetric are found from the
 * planes, the preconditioner and inner iterations use the symmetrised cl..ct,
 * and the FP64 residual uses al..at unchanged.  Periodic in x per
 * sevp_set_periodic_we (as the reference's FLAG_PERIODIC_WE).  The device
 * operator is cached between calls (see sevp_fs_options.verify).  Status in
 * sevp_last_status(): SEVP_NONSYMMETRIC when no row scaling symmetrises the
 * operator (x untouched), SEVP_MAXITER with the last iterate in x. */
void p_sevp_pcg_(const float *al, const float *ab, const float *ac, const float *ar,
                 const float *at, const float *b, double *x, const float *cl, const float *cb,
                 const float *cc, const float *cr, const float *ct, const int *i2, const int *j2);
/* The row scaling p_sevp_pcg_ applies, on host arrays (no GPU needed): the
 * weights w[j2] with w_{J+1} / w_J = AT(I,J) / AB(I,J+1) (the same for every
 * I up to 1e-5), normalised so that max |w_J AC(I,J)| = 1, and the five
 * planes of W A made exactly symmetric (each coupling the mean of its two
 * scaled copies) into sym[5 i2 j2] (AL, AB, AC, AR, AT).  Couplings to points
 * outside the grid are zero in sym.  SEVP_NONSYMMETRIC when no row scaling
 * symmetrises the planes (message in sevp_last_error). */
int sevp_row_symmetrize(const float *al, const float *ab, const float *ac, const float *ar,
                        const float *at, int i2, int j2, int periodic, double *w, float *sym);
/* Report of the last p_sevp_pcg_ call (iterations, residuals, device ms). */
int sevp_fs_last_report(sevp_report *r);
/* Frees the cached device operator of p_sevp_pcg_. */
int sevp_fs_release(void);

/* ------------------------------------------------- allocation-free entry */

/* Interior dot product of two padded (i2+2, j2+2) FP64 fields, the sum that
 * p_inprod computes, written to *result.  r, p and result are DEVICE
 * pointers; stream may be NULL.  This entry point has no counterpart in the
 * reference.  It is for callers that cannot let a library allocate GPU
 * memory: a model whose memory pool owns the device, or one that overlaps
 * this call with work on other streams (cudaFree would synchronise the
 * device).  It calls no cudaMalloc or cudaFree; its scratch is a static
 * device array of 16384 + 32 doubles (128 KB) that every GPU loading the
 * library holds until exit.  Limit: j2 <= 16384 (larger grids get
 * SEVP_BAD_ARG and a message in sevp_last_error).  The first call on a
 * device looks up the array's device address; make that first call before
 * any stream capture (a first call on a capturing stream returns
 * SEVP_BAD_ARG with a message saying so).  Calls share the array, so calls
 * that overlap on the GPU race; calls ordered in one stream do not. */
int sevp_inprod_noalloc(const double *r, const double *p, int i2, int j2, double *result,
                        void *stream);

/* ---------------------------------------------------------------------
 * Barotropic pressure correction of FS (M/fs_GLOBAL.f90:1154-1283), the
 * ITMASK loop around the solve.  Device arrays, column-major with the
 * reference's shapes: U (I0,J0,K1), V (I0,J1,K1), IU0 / IV0 (I0,J0) and
 * IU (I0,J0,K1) / IV (I0,J1,K1) INTEGER*2, ODX / ODY / OCS (J0), CSV / ODYV
 * (J1), ODZ (K1) REAL*4, S (I2,J2), P0 (I0,J0), SCR (I0,J0,4) REAL*4; X is
 * the solver's unpadded (I2,J2) FP64 field (the interior of the reference's
 * padded X).  The REAL*4 / REAL*8 steps follow the Fortran order, so the
 * results equal the CPU oracle's bit for bit.  The reference's local
 * override U = 1, V = 0 (:1173-1175) is not reproduced. */
/* U(:,:,1) *= IU0 on interior (and, if periodic, the two wrap) U faces and
 * V(:,:,1) *= IV0 on interior V faces (:1158-1171). */
int sevp_fs_mask(int i0, int j0, float *u, float *v, const int16_t *iu0, const int16_t *iv0,
                 int periodic, void *stream);
/* S from continuity (FLAG_FS branch, :1177-1192): W integrated upwards from
 * W(:,:,K0) = 0; S(I-1,J-1) = W(I,J,1).  s (REAL*4) and/or b (FP64 copy for
 * the solver, multiplied by rscale(J-1) when rscale (J2 values) is given, to
 * match a row-scaled symmetric operator) may be NULL. */
int sevp_fs_rhs(int i0, int j0, int k0, const float *u, const float *v, const float *odx,
                const float *ody, const float *ocs, const float *csv, const float *odz,
                const float *rscale, float *s, double *b, void *stream);
/* After the solve (:1216-1276): P0 += ODT X; SCR(:,:,1) / (:,:,2) = the U /
 * V corrections -dX * ODX / ODYV (U periodic when periodic != 0), added to
 * every layer (masked by IU / IV below the top) and accumulated in
 * SCR(:,:,3) / (:,:,4); *vmax (device) = the largest top-layer velocity on
 * land faces. */
int sevp_fs_correct(int i0, int j0, int k0, const double *x, float odt, const float *odx,
                    const float *odyv, const int16_t *iu, const int16_t *iv, const int16_t *iu0,
                    const int16_t *iv0, float *p0, float *u, float *v, float *scr, int periodic,
                    float *vmax, void *stream);
/* The whole loop on the context's stream: mask, S, solve A X = S (the
 * context's operator, I2 x J2, from zero; opts as for sevp_solve), correct,
 * until the land velocity <= tolerance or mxmask passes.  b, x (I2*J2 FP64)
 * and vmax_dev (one float) are device scratch supplied by the caller.
 * Reports the passes, the final land velocity and the total PCG iterations. */
int sevp_fs_barotropic(sevp_ctx *ctx, int i0, int j0, int k0, float *u, float *v, float *p0,
                       float *scr, const int16_t *iu0, const int16_t *iv0, const int16_t *iu,
                       const int16_t *iv, const float *odx, const float *ody, const float *ocs,
                       const float *csv, const float *odyv, const float *odz,
                       const float *rscale, float odt, int periodic, float tolerance, int mxmask,
                       const sevp_solve_opts *opts, double *b, double *x, float *vmax_dev,
                       int *itmask_out, float *vmax_out, int *iterations_out);

/* ---------------------------------------------------------------------
 * EVP influence file, the record that PREP's INITFS writes
 * (P/prep_GLOBAL.f90:320: WRITE(FNO_EVP) AL,AR,AB,AT,AC,RINV,RINV1,IE) and
 * MAIN reads (M/input_GLOBAL.f90:440-443: READ(FN_EVP) AL,AR,AB,AT,AC,OAC,
 * RINV,RINV1,IE): one big-endian Fortran unformatted sequential record in
 * gfortran's framing (4-byte markers; records over 2147483639 bytes split
 * into subrecords).  Host arrays, column-major as in the reference: the
 * planes are (I2, J2) REAL*4, RINV / RINV1 hold n_rinv / n_rinv1 REAL*8
 * ((I2, I2, NB0) and (I2, I2, NB1) for REP1, or the BIR strip shapes), IE
 * NB0 INTEGER*4.  Influence data computed on the GPU by pre1_ / pre_ /
 * sevp_pre_strips_ written here is read by MAIN unchanged.
 * oac: NULL writes PREP's layout (no OAC plane); non-NULL writes MAIN's.
 * The reader decides from the record length whether OAC is present, reports
 * it in *has_oac (optional) and fills oac only if given; sizes that match
 * neither layout return SEVP_BAD_ARG. */
int sevp_evp_write(const char *path, int i2, int j2, const float *al, const float *ar,
                   const float *ab, const float *at, const float *ac, const float *oac,
                   const double *rinv, long long n_rinv, const double *rinv1, long long n_rinv1,
                   const int *ie, int nb0);
/* The same with a smaller subrecord limit (1 .. 2147483639 bytes). */
int sevp_evp_write_sub(const char *path, int i2, int j2, const float *al, const float *ar,
                       const float *ab, const float *at, const float *ac, const float *oac,
                       const double *rinv, long long n_rinv, const double *rinv1, long long n_rinv1,
                       const int *ie, int nb0, long long max_subrecord);
int sevp_evp_read(const char *path, int i2, int j2, float *al, float *ar, float *ab, float *at,
                  float *ac, float *oac, double *rinv, long long n_rinv, double *rinv1,
                  long long n_rinv1, int *ie, int nb0, int *has_oac);

#ifdef __cplusplus
}
#endif
#endif /* SEVP_B200_H */
