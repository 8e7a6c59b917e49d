"""Host-side interface of the native SEVP-PCG solver.

``SevpSolver`` owns a device operator (five FP32 coefficient planes and the
tile influence data) and solves ``A x = b`` on the GPU with the block-Jacobi
tile SEVP preconditioned conjugate gradient, either all in FP64 or as FP32
inner solves inside FP64 iterative refinement.

Device memory, streams and the upload of inputs use PyTorch (plumbing); every
arithmetic step runs in ``libsevp_b200.so``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native as N


def default_sub_rows(problem_or_ratio, tile_h: int, growth_limit: float = 1e6) -> list[int]:
    """Sub-block heights per tile row from the marching amplification bound.

    Marching north multiplies the worst Fourier mode by z per row, where
    z + 1/z = (2|AL+AR| + |AB+AT| + |gamma|)/|AT| (largest over the band).
    The height is the largest s with z**s <= growth_limit (at least 1).
    """
    p = problem_or_ratio
    al, ab, ac, ar, at = (np.abs(a.astype(np.float64)) for a in p.coeffs())
    ny = p.ny
    ty = -(-ny // tile_h)
    out = []
    for b in range(ty):
        sl = slice(b * tile_h, min(ny, (b + 1) * tile_h))
        atn = np.maximum(at[sl], 1e-300)
        # use the interior rows (the last domain row has AT = 0 and is not marched)
        ratio = (np.abs(ac[sl]) + al[sl] + ar[sl]) / atn
        valid = at[sl] > 0
        c = float(ratio[valid].max()) if valid.any() else 2.0
        c = max(c, 2.0 + 1e-12)
        z = 0.5 * (c + np.sqrt(c * c - 4.0))
        s = int(np.floor(np.log(growth_limit) / np.log(z))) if z > 1.0 else tile_h
        out.append(max(1, min(tile_h, s)))
    return out


def tile_sub_blocks(problem, tile_m: int, tile_h: int, growth_limit: float = 1e10) -> np.ndarray:
    """Sub-blocks per tile, shape (tiles_y, tiles_x): the host statement of
    the library's per-tile rule (k_tile_growth + the warp-group maximum).

    Each tile's height is the largest s with z**s <= growth_limit, where
    z + 1/z is the largest (|AC|+|AL|+|AR|)/|AT| over the tile's marched
    rows; tiles that share a warp (groups of 32/W neighbours, W the lane
    segment width 8/16/32) use the largest sub-block count of the group.
    """
    p = problem
    al, ab, ac, ar, at = (np.abs(a.astype(np.float64)) for a in p.coeffs())
    nx, ny = p.nx, p.ny
    tx, ty = -(-nx // tile_m), -(-ny // tile_h)
    wseg = 8 if tile_m <= 8 else (16 if tile_m <= 16 else 32)
    tpw = 32 // wseg
    out = np.ones((ty, tx), np.int64)
    for b in range(ty):
        j0 = b * tile_h
        hh = min(tile_h, ny - j0)
        rows = slice(j0, j0 + hh - 1)  # marched rows: all but the tile's last
        for a in range(tx):
            cols = slice(a * tile_m, min(nx, (a + 1) * tile_m))
            s = tile_h
            if hh > 1:
                atv = at[rows, cols]
                if (atv == 0).any():
                    s = 1
                else:
                    c = max(2.0, float(((ac[rows, cols] + al[rows, cols] + ar[rows, cols]) / atv).max()))
                    z = 0.5 * (c + np.sqrt(max(c * c - 4.0, 0.0)))
                    if z > 1.0:
                        s = int(np.floor(np.log(growth_limit) / np.log(z)))
            s = max(1, min(tile_h, s))
            out[b, a] = -(-hh // min(s, hh))
    for b in range(ty):
        for g in range(0, tx, tpw):
            out[b, g:g + tpw] = out[b, g:g + tpw].max()
    return out.astype(np.int32)


@dataclass
class SolveResult:
    status: int
    iterations: int
    refinements: int
    rel_residual: float
    bnorm: float
    ms: float
    abs_residual: float = 0.0

    @classmethod
    def of(cls, rep) -> "SolveResult":
        return cls(rep.status, rep.iterations, rep.refinements, rep.rel_residual, rep.bnorm,
                   rep.ms, rep.abs_residual)


class SevpSolver:
    """Device operator + solver context (one GPU, one CUDA stream)."""

    def __init__(self, problem, tile_m: int = 16, tile_h: int = 16, sub_rows=None,
                 growth_limit: float = 1e10, device: str = "cuda", stream=None,
                 full_coefficients: bool = False, precond_fp32: bool = False,
                 schwarz=False):
        import torch

        self.precond_fp32 = bool(precond_fp32)
        self.method = N.METHOD_PCG
        # mixed precision: True restarts CG at every FP64 residual
        self.restart_inner = False

        self.torch = torch
        self.p = problem
        self.nx, self.ny = problem.nx, problem.ny
        self.device = torch.device(device)
        self.stream = stream or torch.cuda.current_stream(self.device)
        dev = self.device
        self.coef = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
                     for a in problem.coeffs()]
        torch.cuda.synchronize(dev)
        h = C.c_void_p()
        N.check(N.lib().sevp_create(C.byref(h), self.nx, self.ny, int(problem.periodic),
                                    C.c_void_p(self.stream.cuda_stream)), "sevp_create")
        self.h = h
        if full_coefficients:
            N.check(N.lib().sevp_set_full_coefficients(self.h, 1), "sevp_set_full_coefficients")
        self.tile_m, self.tile_h = tile_m, tile_h
        if sub_rows is not None:
            # explicit heights per tile row
            rows = list(np.broadcast_to(np.asarray(sub_rows, np.int32), (-(-self.ny // tile_h),)))
            self._srow = (C.c_int * len(rows))(*rows)
            self.tiling = N.Tiling(tile_m, tile_h, int(max(rows)), self._srow, None, 0.0)
        else:
            # heights per tile from the marching growth bound (computed on the GPU)
            self.tiling = N.Tiling(tile_m, tile_h, tile_h, None, None, float(growth_limit))
        N.check(N.lib().sevp_set_operator(self.h, *[N.ptr(t) for t in self.coef],
                                          C.byref(self.tiling)), "sevp_set_operator")
        self.tile_nb = self.layout()
        if schwarz:
            self.set_schwarz(-1 if schwarz is True else int(schwarz))

    def layout(self) -> np.ndarray:
        """Sub-blocks used by each tile, shape (tiles_y, tiles_x)."""
        tx, ty = C.c_int(), C.c_int()
        N.check(N.lib().sevp_tile_layout(self.h, C.byref(tx), C.byref(ty), None), "sevp_tile_layout")
        out = np.zeros(tx.value * ty.value, np.int32)
        N.check(N.lib().sevp_tile_layout(self.h, C.byref(tx), C.byref(ty),
                                         out.ctypes.data_as(C.POINTER(C.c_int))), "sevp_tile_layout")
        return out.reshape(ty.value, tx.value)

    def close(self):
        if getattr(self, "h", None):
            N.lib().sevp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------
    def influence_bytes(self) -> int:
        return int(N.lib().sevp_influence_bytes(self.h))

    def set_influence_fp32(self, growth_limit: float):
        """Per-group influence precision of the FP32 inner iterations: the
        warp groups whose tiles' marching growth bound is <= growth_limit
        read FP32 matrices, the rest FP64 (growth_limit <= 1: all FP64)."""
        N.check(N.lib().sevp_set_influence_fp32(self.h, float(growth_limit)),
                "sevp_set_influence_fp32")

    def influence_fp32_groups(self):
        """(FP32 groups, all groups, influence bytes read per tile pass)."""
        f, g, b = C.c_int(), C.c_int(), C.c_longlong()
        N.check(N.lib().sevp_influence_fp32_groups(self.h, C.byref(f), C.byref(g), C.byref(b)),
                "sevp_influence_fp32_groups")
        return f.value, g.value, b.value

    def launches(self) -> int:
        return int(N.lib().sevp_kernel_launches(self.h))

    def profile(self, enable: bool = True):
        """Starts (zeroes) or stops per-kernel-class CUDA-event timing."""
        N.check(N.lib().sevp_profile(self.h, int(enable)), "sevp_profile")

    def profile_read(self):
        """{class: (total_ms, launches)} for 'tile', 'stencil', 'precond', 'couple'."""
        ms = (C.c_double * 4)()
        n = (C.c_longlong * 4)()
        N.check(N.lib().sevp_profile_read(self.h, ms, n), "sevp_profile_read")
        return {"tile": (ms[0], n[0]), "stencil": (ms[1], n[1]), "precond": (ms[2], n[2]),
                "couple": (ms[3], n[3])}

    def opts(self, precision=0, tol=1e-12, max_iter=5000, inner_tol=1e-5, use_guess=False,
             check_every=4, precond_fp32=None, tol_abs=False, method=None, restart_inner=None):
        if precond_fp32 is None:
            precond_fp32 = self.precond_fp32
        if method is None:
            # the Chebyshev iteration is a mixed-precision method
            method = self.method if int(precision) == 1 else N.METHOD_PCG
        if restart_inner is None:
            restart_inner = self.restart_inner
        return N.SolveOpts(int(precision), float(tol), int(max_iter), float(inner_tol),
                           int(use_guess), int(check_every), int(precond_fp32), int(bool(tol_abs)),
                           int(method), int(bool(restart_inner)))

    def set_schwarz(self, shift: int = -1):
        """Overlapping Schwarz preconditioner: a second tiling rolled west by
        ``shift`` columns (-1: about half a tile), applied as the symmetric
        multiplicative sweep first tiling -> second -> first.  0 returns to
        block-Jacobi.  Tiles must be at most 8 rows high."""
        N.check(N.lib().sevp_set_schwarz(self.h, int(shift)), "sevp_set_schwarz")

    @property
    def schwarz_shift(self) -> int:
        """Column shift of the second tiling (0: block-Jacobi)."""
        return int(N.lib().sevp_schwarz_shift(self.h))

    def condition_estimate(self, b, cap: int = 4000, tol: float = 1e-12):
        """Extreme eigenvalues of the preconditioned operator M^-1 A (the
        context's preconditioner): one FP64 PCG solve of ``b`` from zero
        records its coefficients alpha_j, beta_j on the device; the Ritz
        values of the CG-Lanczos tridiagonal (diagonal 1/alpha_j +
        beta_{j-1}/alpha_{j-1}, off-diagonal sqrt(beta_j)/alpha_j) estimate
        them from inside.  Returns dict(lambda_min, lambda_max, kappa,
        iterations)."""
        lib = N.lib()
        N.check(lib.sevp_record_coefficients(self.h, int(cap)), "sevp_record_coefficients")
        try:
            x = self.torch.zeros_like(b)
            self.solve(b, x=x, precision=0, tol=tol, max_iter=cap)
            a = np.zeros(cap)
            bt = np.zeros(cap)
            cnt = C.c_int()
            N.check(lib.sevp_read_coefficients(self.h, a.ctypes.data_as(N.DP),
                                               bt.ctypes.data_as(N.DP), int(cap), C.byref(cnt)),
                    "sevp_read_coefficients")
        finally:
            lib.sevp_record_coefficients(self.h, 0)
        k = cnt.value
        if k == 0:
            raise RuntimeError("no PCG iterations were recorded")
        a, bt = a[:k], bt[:k]
        d = 1.0 / a
        d[1:] += bt[:-1] / a[:-1]
        e = np.sqrt(bt[:-1]) / a[:-1]
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        ev = np.linalg.eigvalsh(T)
        return dict(lambda_min=float(ev[0]), lambda_max=float(ev[-1]),
                    kappa=float(ev[-1] / ev[0]), iterations=k)

    def set_method(self, method: int):
        """Outer iteration of the mixed-precision solves: N.METHOD_PCG (two
        passes per iteration) or N.METHOD_CHEB (one launch per iteration;
        needs bounds, see chebyshev_setup)."""
        self.method = int(method)

    def estimate_bounds(self, b):
        """(lambda_min, lambda_max, iterations) of M^-1 A from the CG-Lanczos
        tridiagonal of one FP64 PCG solve of b (computed in the library)."""
        lo, hi, it = C.c_double(), C.c_double(), C.c_int()
        N.check(N.lib().sevp_estimate_bounds(self.h, N.ptr(b), C.byref(lo), C.byref(hi),
                                             C.byref(it)), "sevp_estimate_bounds")
        return lo.value, hi.value, it.value

    def set_chebyshev_bounds(self, lmin: float, lmax: float):
        N.check(N.lib().sevp_set_chebyshev_bounds(self.h, float(lmin), float(lmax)),
                "sevp_set_chebyshev_bounds")

    def chebyshev_setup(self, b, widen: float = 0.02):
        """Estimates the bounds from a solve of b, widens them by the factor
        (1 -/+ widen) (Ritz values lie inside the spectrum) and sets them."""
        lo, hi, _ = self.estimate_bounds(b)
        self.set_chebyshev_bounds(lo * (1.0 - widen), hi * (1.0 + widen))
        return lo, hi

    def schwarz_influence_bytes(self) -> int:
        return int(N.lib().sevp_schwarz_influence_bytes(self.h))

    def graphs(self, enable: bool = True):
        """CUDA-graph replay of the FP32 inner iterations (default on)."""
        N.check(N.lib().sevp_set_graphs(self.h, int(bool(enable))), "sevp_set_graphs")

    @property
    def symmetric(self) -> bool:
        return bool(N.lib().sevp_operator_symmetric(self.h))

    def solve(self, b, x=None, precision=0, tol=1e-12, max_iter=5000, inner_tol=1e-5,
              check_every=4, x_is_guess=True):
        """Solves on device tensors (float64, shape (ny, nx)).  ``x`` holds the
        initial guess when given and receives the solution; with
        ``x_is_guess=False`` it only receives the solution of a solve from
        zero (the library zeroes it)."""
        torch = self.torch
        use_guess = x is not None and x_is_guess
        if x is None:
            x = torch.zeros((self.ny, self.nx), dtype=torch.float64, device=self.device)
        o = self.opts(precision, tol, max_iter, inner_tol, use_guess, check_every)
        rep = N.Report()
        s = N.lib().sevp_solve(self.h, N.ptr(b), N.ptr(x), C.byref(o), C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_solve")
        return x, SolveResult.of(rep)

    def solve_host(self, b: np.ndarray, x: np.ndarray | None = None, precision=0, tol=1e-12,
                   max_iter=5000, inner_tol=1e-5, check_every=4):
        """Solves with host arrays (copies in and out inside the call)."""
        b = np.ascontiguousarray(b, np.float64)
        use_guess = x is not None
        out = np.ascontiguousarray(x, np.float64).copy() if use_guess else np.zeros_like(b)
        o = self.opts(precision, tol, max_iter, inner_tol, use_guess, check_every)
        rep = N.Report()
        s = N.lib().sevp_solve_host(self.h, N.ptr(b), N.ptr(out), C.byref(o), C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_solve_host")
        return out, SolveResult.of(rep)

    def solve_step(self, b, eta1, eta2, x, guess=N.GUESS_LINEAR, precision=1, tol=1e-12,
                   max_iter=5000, inner_tol=1e-5, check_every=4):
        """One sequence step on device tensors: x <- guess(eta1, eta2, b), then
        solve from it."""
        o = self.opts(precision, tol, max_iter, inner_tol, True, check_every)
        rep = N.Report()
        s = N.lib().sevp_solve_step(self.h, N.ptr(b), N.ptr(eta1) if eta1 is not None else None,
                                    N.ptr(eta2) if eta2 is not None else None, N.ptr(x), int(guess),
                                    C.byref(o), C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_solve_step")
        return x, SolveResult.of(rep)

    def solve_step_host(self, b, eta1, eta2, x, guess=N.GUESS_LINEAR, precision=1, tol=1e-12,
                        max_iter=5000, inner_tol=1e-5, check_every=4):
        """One sequence step with host (numpy, ideally pinned) buffers."""
        o = self.opts(precision, tol, max_iter, inner_tol, True, check_every)
        rep = N.Report()
        s = N.lib().sevp_solve_step_host(self.h, N.ptr(b), N.ptr(eta1) if eta1 is not None else None,
                                         N.ptr(eta2) if eta2 is not None else None, N.ptr(x),
                                         int(guess), C.byref(o), C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_solve_step_host")
        return x, SolveResult.of(rep)

    def step_history(self, eta1=None, eta2=None):
        """Loads the device-held history of step_host from host arrays (eta1
        the newest; both None empties it)."""
        keep = [np.ascontiguousarray(a, np.float64) for a in (eta1, eta2) if a is not None]
        N.check(N.lib().sevp_step_history(self.h, *(N.ptr(a) for a in keep),
                                          *([None] * (2 - len(keep)))), "sevp_step_history")

    def step_host(self, b, x, guess=N.GUESS_LINEAR, precision=1, tol=1e-12, max_iter=5000,
                  inner_tol=1e-5, check_every=4):
        """One time step with the history held on the device: copies b (host)
        in and the solution into x (host) out; x becomes the newest solution
        of the history."""
        o = self.opts(precision, tol, max_iter, inner_tol, True, check_every)
        rep = N.Report()
        s = N.lib().sevp_step_host(self.h, N.ptr(b), N.ptr(x), int(guess), C.byref(o),
                                   C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_step_host")
        return x, SolveResult.of(rep)

    def step_prefetch(self, b):
        """Starts copying a later step's b (pinned host array) to the device."""
        N.check(N.lib().sevp_step_prefetch(self.h, N.ptr(b)), "sevp_step_prefetch")

    def step_submit(self, b, x, guess=N.GUESS_LINEAR, precision=1, tol=1e-12, max_iter=5000,
                    inner_tol=1e-5, check_every=4):
        """step_host without waiting for x: the copy of x (pinned host array)
        completes by the next step_wait."""
        o = self.opts(precision, tol, max_iter, inner_tol, True, check_every)
        rep = N.Report()
        s = N.lib().sevp_step_submit(self.h, N.ptr(b), N.ptr(x), int(guess), C.byref(o),
                                     C.byref(rep))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_step_submit")
        return SolveResult.of(rep)

    def step_wait(self):
        N.check(N.lib().sevp_step_wait(self.h), "sevp_step_wait")

    def apply(self, x):
        y = self.torch.empty_like(x)
        N.check(N.lib().sevp_apply(self.h, N.ptr(x), N.ptr(y)), "sevp_apply")
        return y

    def set_pass_a_kernel(self, kind: int):
        """Kernel of the PCG's stencil pass: N.PASS_A_TILES (tensor-copied
        tiles, the default where the grid allows) or N.PASS_A_COLUMNS."""
        N.check(N.lib().sevp_set_pass_a_kernel(self.h, int(kind)), "sevp_set_pass_a_kernel")

    def set_pass_b_kernel(self, kind: int):
        """Kernel of the FP32 PCG's tile pass: N.PASS_B_REGISTERS (the
        default) or N.PASS_B_STAGED (tensor-copied task stages, where the
        tiling allows)."""
        N.check(N.lib().sevp_set_pass_b_kernel(self.h, int(kind)), "sevp_set_pass_b_kernel")

    def set_resume_check(self, max_rel_dev: float):
        """Largest ||r_true - r_recursive|| / ||r_true|| at which a mixed PCG
        run resumes on a replaced residual (default 0.3; <= 0: never)."""
        N.check(N.lib().sevp_set_resume_check(self.h, float(max_rel_dev)),
                "sevp_set_resume_check")

    def pass_b_kernel_used(self) -> int:
        """The kernel the last FP32 tile pass ran (N.PASS_B_*), -1 before
        the first."""
        return int(N.lib().sevp_pass_b_kernel_used(self.h))

    def pass_a(self, z, pold, beta: float):
        """One stencil pass: (p, q, p.q) with p = z + beta p_old, q = A p."""
        pnew = self.torch.empty_like(z)
        q = self.torch.empty_like(z)
        pq = C.c_double()
        fn = N.lib().sevp_pass_a_f64 if z.dtype == self.torch.float64 else N.lib().sevp_pass_a_f32
        N.check(fn(self.h, N.ptr(z), N.ptr(pold), float(beta), N.ptr(pnew), N.ptr(q),
                   C.byref(pq)), "sevp_pass_a")
        return pnew, q, pq.value

    def precondition(self, r):
        z = self.torch.empty_like(r)
        fn = N.lib().sevp_precondition if r.dtype == self.torch.float64 else N.lib().sevp_precondition_f32
        N.check(fn(self.h, N.ptr(r), N.ptr(z)), "sevp_precondition")
        return z

    def relative_residual(self, b, x) -> float:
        v = C.c_double()
        N.check(N.lib().sevp_relative_residual(self.h, N.ptr(b), N.ptr(x), C.byref(v)),
                "sevp_relative_residual")
        return v.value
