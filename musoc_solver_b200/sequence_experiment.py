"""Learned warm start on a time sequence of solves (the c4 configuration).

    python -m musoc_solver_b200.sequence_experiment --nx 1440 --ny 720 --steps 400 --train 300

A 400-step sequence of right-hand sides (300 seeded Gaussian eddies, radius
50-150 km, advected at 0.2 m/s with slow amplitude drift) on the periodic
global grid is solved in FP64 to 1e-12 from the linear extrapolation of the
two previous solutions; those solutions are the training data.  The U-Net
is trained on steps 2..train-1 and tested on the remaining steps.  It
reports, for each guess (zero, previous step, linear extrapolation,
learned), the mean iterations and the mean device time (guess + solve) to
1e-12 in mixed precision, the error against the FP64 solutions, and how much
closer the learned guess is to the solution than the same pipeline without
the network.  One JSON line per network coarsening.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1440)
    ap.add_argument("--ny", type=int, default=720)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--train", type=int, default=300)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--coarse", default="1,2,4", help="network coarsenings to try")
    ap.add_argument("--tiles", default="16x8")
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args(argv)
    import torch

    from . import build, problems as P
    from .solver import SevpSolver
    from .warmstart import LearnedWarmStart, evaluate, solve_sequence, train

    build.build()
    t0 = time.perf_counter()
    p = P.global_grid(args.nx, args.ny, seed=args.seed)
    wet = p.meta["wet"]
    rhs = [torch.from_numpy(np.where(wet, b, 0.0)).cuda()
           for _, b in P.eddy_rhs(args.nx, args.ny, range(args.steps), seed=args.seed + 2)]
    tm, th = (int(v) for v in args.tiles.split("x"))
    s = SevpSolver(p, tile_m=tm, tile_h=th)
    etas = solve_sequence(s, rhs)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    train_idx = list(range(2, args.train))
    test_idx = list(range(args.train + 2, args.steps))
    base = evaluate(s, None, etas, rhs, test_idx)
    for c in (int(v) for v in args.coarse.split(",")):
        t1 = time.perf_counter()
        w = LearnedWarmStart.create(s, seed=0, train=True, coarse=c)
        losses = train(w, etas, rhs, train_idx, epochs=args.epochs, lr=2e-3, lr_final=2e-4)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t1
        w = w.inference_copy()
        x = torch.zeros_like(etas[0])
        gain = []
        for n in test_idx:
            w.predict(etas[n - 1], etas[n - 2], rhs[n], x)
            gain.append(float((w.e + w.m - etas[n]).norm() / (x - etas[n]).norm()))
        w.attach()
        res = evaluate(s, w, etas, rhs, test_idx)
        w.close()
        out = {"grid": [args.nx, args.ny], "steps": args.steps, "train_steps": len(train_idx),
               "test_steps": len(test_idx), "epochs": args.epochs, "network_grid": [w.net.W, w.net.H],
               "coarse": c, "tiles": [tm, th], "train_seconds": round(train_s, 1),
               "loss_first_last": [losses[0][1], losses[-1][1]],
               "guess_error_ratio_without_over_with_network": float(np.median(gain)),
               "results": {**{k: v for k, v in base.items()}, "learned": res["learned"]},
               "setup_seconds": round(setup_s, 1)}
        print(json.dumps(out), flush=True)
    s.close()


if __name__ == "__main__":
    main()
