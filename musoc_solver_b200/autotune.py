"""Autotuning of the tile-SEVP PCG: tile shape, preconditioner, inner tolerance.

The tile shape trades preconditioner strength against work per iteration:
wider and taller tiles solve more of the coupling exactly (fewer PCG
iterations) but carry larger influence matrices (more bytes per iteration)
and, on anisotropic high-latitude rows, more marching sub-blocks.  The
overlapping Schwarz preconditioner (a second tiling shifted by half a tile,
tiles of at most 8 rows) costs about three tile passes per iteration and
cuts the iterations by about three.  The mixed solve's inner tolerance sets
how many FP64 refinements (each a PCG restart) the solve needs.  The best
choice depends on the grid, so it is measured: every candidate shape gets a
solver (its influence data precomputed on the GPU) for each preconditioner,
one untimed solve and `repeats` timed solves of the same right-hand side,
from a zero guess or from the linear extrapolation of a given history, per
inner tolerance; the fastest wins.  The outer iteration is a candidate too:
PCG (two grid passes per iteration) or, for block-Jacobi tiles of at most 8
rows, the one-launch Chebyshev iteration on the CG-Lanczos spectrum bounds
(estimated once per candidate, untimed: they belong to the operator's set-up
like the influence data).
"""
from __future__ import annotations

import time

from .solver import SevpSolver

CANDIDATES = ((8, 8), (8, 16), (16, 4), (16, 6), (16, 8), (16, 12), (16, 16), (16, 24),
              (32, 8), (32, 16), (32, 32))
# the Schwarz stage kernel and the Chebyshev kernel hold at most this many
# tile rows
SCHWARZ_MAX_ROWS = 8
CHEB_MAX_ROWS = 8


def autotune(problem, b, candidates=CANDIDATES, precision=1, tol=1e-12, repeats=2,
             growth_limit=1e10, device="cuda", schwarz=(False, True), inner_tols=(1e-5,),
             history=None, methods=(0,)):
    """Returns (best, table): best = dict(tile_m, tile_h, schwarz, inner_tol,
    ms, ...) of the fastest candidate, table = one such dict per candidate
    measured.  b is the right-hand side on the device (float64, shape
    (ny, nx)).  inner_tols only matter for precision 1.  history = (eta1,
    eta2), the two previous solutions: each solve then starts from their
    linear extrapolation (the warm start of a time sequence) instead of
    zero."""
    import torch

    from . import native as N

    def run(s, x, itol):
        if history is None:
            x.zero_()
            return s.solve(b, x=x, precision=precision, tol=tol, inner_tol=itol)[1]
        return s.solve_step(b, history[0], history[1], x, guess=N.GUESS_LINEAR,
                            precision=precision, tol=tol, inner_tol=itol)[1]

    table = []
    for tm, th in candidates:
        if tm > problem.nx or th > problem.ny:
            continue
        for sw in schwarz:
            if sw and th > SCHWARZ_MAX_ROWS:
                continue
            t0 = time.perf_counter()
            s = SevpSolver(problem, tile_m=tm, tile_h=th, growth_limit=growth_limit, device=device,
                           schwarz=sw)
            torch.cuda.synchronize()
            setup_s = time.perf_counter() - t0
            x = torch.zeros_like(b)
            for method in methods:
                if method == N.METHOD_CHEB and (precision != 1 or sw or th > CHEB_MAX_ROWS):
                    continue
                if method == N.METHOD_CHEB:
                    s.chebyshev_setup(b)
                s.set_method(method)
                for itol in (inner_tols if precision == 1 else inner_tols[:1]):
                    run(s, x, itol)
                    best_ms, res = None, None
                    for _ in range(repeats):
                        res = run(s, x, itol)
                        best_ms = res.ms if best_ms is None else min(best_ms, res.ms)
                    table.append(dict(tile_m=tm, tile_h=th, schwarz=bool(sw), inner_tol=itol,
                                      method=int(method), ms=best_ms, iterations=res.iterations,
                                      refinements=res.refinements, status=res.status,
                                      rel_residual=res.rel_residual,
                                      influence_mb=(s.influence_bytes()
                                                    + s.schwarz_influence_bytes()) / 1e6,
                                      setup_s=setup_s))
            s.close()
            del s
    ok = [r for r in table if r["status"] == 0]
    if not ok:
        raise RuntimeError("no tile shape reached the tolerance")
    return min(ok, key=lambda r: r["ms"]), table
