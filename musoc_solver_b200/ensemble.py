"""Batched ensemble solves: all members in every kernel launch.

The members (one grid size, each with its own coefficients and right-hand
side) are stacked along y into one block-diagonal system
(``problems.stack``); the tile height is chosen to divide a member's row
count, so no tile crosses two members, and every pass of the PCG (stencil,
tile SEVP) is one launch over all members.  The FP32 inner iterations of
the mixed solve replay one CUDA graph per check interval.

Stopping: the solver's test is on the stacked residual, so the tolerance
handed to it is tightened by the smallest member's share of ||b||,
  tol_stack = tol * min_k ||b_k|| / ||b||,
which guarantees ||b_k - A_k x_k|| <= tol ||b_k|| for every member k; the
per-member residuals are measured after the solve and reported.
"""
from __future__ import annotations

import numpy as np

from . import native as N
from . import problems as P
from .solver import SevpSolver


def member_tile_height(ny: int, prefer=(6, 8, 12, 10, 16, 18, 20, 15, 24)) -> int:
    """A tile height that divides the member row count (tiles never straddle
    two members).  Short tiles come first: on a B200 the 64 x 720x360
    ensemble's mixed solve takes 11.8 ms with 16x6 tiles, 13.0 ms with 16x8
    and 16.4 ms with 16x18 (6-row tiles run the short-tile kernel)."""
    for h in prefer:
        if ny % h == 0:
            return h
    raise ValueError(f"no tile height in {prefer} divides {ny}")


class EnsembleSolver:
    def __init__(self, members, tile_m: int = 16, tile_h: int | None = None, growth_limit=1e10,
                 device="cuda", stream=None, schwarz=False):
        import torch

        self.torch = torch
        self.members = list(members)
        self.m = len(self.members)
        self.ny, self.nx = self.members[0].ny, self.members[0].nx
        self.problem = P.stack(self.members)
        th = tile_h or member_tile_height(self.ny)
        if self.ny % th:
            raise ValueError("tile height must divide the member row count")
        self.solver = SevpSolver(self.problem, tile_m=tile_m, tile_h=th, growth_limit=growth_limit,
                                 device=device, stream=stream, schwarz=schwarz)
        self.device = self.solver.device

    def rhs(self):
        """Stacked right-hand sides of the members, on the device."""
        return self.torch.from_numpy(self.problem.b).to(self.device)

    def member_norms(self, v):
        return v.reshape(self.m, -1).norm(dim=1)

    def stacked_tol(self, b, tol=1e-12):
        """The stacked system's tolerance that guarantees ``tol`` for every
        member (see the module note)."""
        bn = self.member_norms(b)
        return tol * float(bn.min() / b.norm()) if float(b.norm()) > 0 else tol

    def solve(self, b, x=None, precision=1, tol=1e-12, max_iter=5000, inner_tol=1e-5,
              residuals=True, tol_stack=None, x_is_guess=True):
        """Solves all members; returns (x, result, per-member relative
        residuals as a host array, or None with ``residuals=False``).
        ``tol_stack`` (from ``stacked_tol``) skips recomputing the stacked
        tolerance; ``x_is_guess=False`` solves from zero into ``x``."""
        if tol_stack is None:
            tol_stack = self.stacked_tol(b, tol)
        x, res = self.solver.solve(b, x=x, precision=precision, tol=tol_stack, max_iter=max_iter,
                                   inner_tol=inner_tol, x_is_guess=x_is_guess)
        return x, res, (self.member_residuals(b, x) if residuals else None)

    def member_residuals(self, b, x):
        r = b - self.solver.apply(x)
        bn = self.member_norms(b)
        return (self.member_norms(r) / self.torch.where(bn > 0, bn, self.torch.ones_like(bn))).cpu().numpy()

    def close(self):
        self.solver.close()
