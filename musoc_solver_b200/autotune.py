"""Tile-shape autotuning of the tile-SEVP PCG.

The tile shape trades preconditioner strength against work per iteration:
wider and taller tiles solve more of the coupling exactly (fewer PCG
iterations) but carry larger influence matrices (more bytes per iteration)
and, on anisotropic high-latitude rows, more marching sub-blocks.  The best
shape depends on the grid, so it is measured: every candidate from 16x4 to
32x32 gets a solver (its influence data precomputed on the GPU), one
untimed solve and `repeats` timed solves of the same right-hand side from a
zero guess; the fastest wins.
"""
from __future__ import annotations

import time

from .solver import SevpSolver

CANDIDATES = ((8, 8), (8, 16), (16, 4), (16, 6), (16, 8), (16, 12), (16, 16), (16, 24),
              (32, 8), (32, 16), (32, 32))


def autotune(problem, b, candidates=CANDIDATES, precision=1, tol=1e-12, repeats=2,
             growth_limit=1e10, device="cuda"):
    """Returns (best, table): best = dict(tile_m, tile_h, ms, ...) of the
    fastest candidate, table = one such dict per candidate measured.  b is
    the right-hand side on the device (float64, shape (ny, nx))."""
    import torch

    table = []
    for tm, th in candidates:
        if tm > problem.nx or th > problem.ny:
            continue
        t0 = time.perf_counter()
        s = SevpSolver(problem, tile_m=tm, tile_h=th, growth_limit=growth_limit, device=device)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        x = torch.zeros_like(b)
        s.solve(b, x=x, precision=precision, tol=tol)
        best_ms, res = None, None
        for _ in range(repeats):
            x.zero_()
            _, res = s.solve(b, x=x, precision=precision, tol=tol)
            best_ms = res.ms if best_ms is None else min(best_ms, res.ms)
        table.append(dict(tile_m=tm, tile_h=th, ms=best_ms, iterations=res.iterations,
                          status=res.status, rel_residual=res.rel_residual,
                          influence_mb=s.influence_bytes() / 1e6, setup_s=setup_s))
        s.close()
        del s
    ok = [r for r in table if r["status"] == 0]
    if not ok:
        raise RuntimeError("no tile shape reached the tolerance")
    return min(ok, key=lambda r: r["ms"]), table
