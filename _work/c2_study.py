"""Preconditioner comparison on a global grid at two time steps.

    python -m musoc_solver_b200.c2_study --nx 1440 --ny 720

For dt = 60 s and dt = 900 s (the longer step weakens the free-surface
term, so the operator is worse conditioned) and for the block-Jacobi and
Schwarz preconditioners: FP64 and mixed solve times (median of repeats, to
1e-12 from zero), iterations, and the extreme eigenvalues of M^-1 A from
the CG-Lanczos tridiagonal of an FP64 solve.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1440)
    ap.add_argument("--ny", type=int, default=720)
    ap.add_argument("--dts", default="60,900")
    ap.add_argument("--tiles", default="16x6,16x8")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--inner-tol", type=float, default=1e-6)
    args = ap.parse_args(argv)
    import numpy as np
    import torch

    from . import build, problems as P
    from .solver import SevpSolver

    build.build()
    out = {"grid": [args.nx, args.ny], "inner_tol": args.inner_tol, "runs": []}
    for dt in (float(v) for v in args.dts.split(",")):
        p = P.global_grid(args.nx, args.ny, seed=1, dt=dt)
        b = torch.from_numpy(p.b).cuda()
        for tiles in args.tiles.split(","):
            tm, th = (int(v) for v in tiles.split("x"))
            for sw in (False, True):
                s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=1e10, schwarz=sw)
                row = {"dt": dt, "tiles": tiles, "preconditioner": "schwarz" if sw else "block-Jacobi"}
                row.update(s.condition_estimate(b))
                for name, prec in (("fp64", 0), ("mixed", 1)):
                    x = torch.zeros_like(b)
                    s.solve(b, x=x, precision=prec, inner_tol=args.inner_tol)
                    ms = []
                    for _ in range(args.repeats):
                        x.zero_()
                        _, rep = s.solve(b, x=x, precision=prec, inner_tol=args.inner_tol)
                        ms.append(rep.ms)
                    row[name] = {"ms": float(np.median(ms)), "iterations": rep.iterations,
                                 "refinements": rep.refinements, "rel_residual": rep.rel_residual,
                                 "status": rep.status}
                out["runs"].append(row)
                s.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
