"""One solve on a synthetic global grid, as a target for ncu captures.

    python -m musoc_solver_b200.profile_case --nx 3600 --ny 2400 --tiles 16x6 --precision 1 --max-iter 3

Builds ``problems.global_grid(nx, ny, seed=11)`` and a solver with the given
tiles (growth bound 1e10; ``--schwarz``: the overlapping Schwarz
preconditioner), then runs one solve with the given precision and
iteration cap.  The first launch of each kernel belongs to the set-up, so
skip one launch (``-s 1``) to capture a PCG iteration.
"""
from __future__ import annotations

import argparse


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=3600)
    ap.add_argument("--ny", type=int, default=2400)
    ap.add_argument("--tiles", default="16x16")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--max-iter", type=int, default=3)
    ap.add_argument("--schwarz", action="store_true")
    args = ap.parse_args(argv)
    import torch

    from . import build, problems as P
    from .solver import SevpSolver

    build.build()
    p = P.global_grid(args.nx, args.ny, seed=11)
    tm, th = (int(v) for v in args.tiles.lower().split("x"))
    s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=1e10, schwarz=args.schwarz)
    b = torch.from_numpy(p.b).cuda()
    _, rep = s.solve(b, precision=args.precision, max_iter=args.max_iter)
    torch.cuda.synchronize()
    print("ok", rep)
    s.close()


if __name__ == "__main__":
    main()
