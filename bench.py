#!/usr/bin/env python
"""Benchmark: solves/s to 1e-12 relative residual at 3600x2400.

Workload (one "step" = one time step of a sequence of barotropic solves):
  * operator: the 3600x2400 periodic-in-x global grid (lat in [-78, 78],
    dx = R dlon cos(lat), seeded synthetic bathymetry with ~30 % land,
    dt = 60 s), symmetric 5-point FP32 coefficients;
  * right-hand sides: a seeded field of 300 Gaussian eddies (radius
    50-150 km) advected at 0.2 m/s with slow amplitude drift, one field per
    step (the sequence workload of the learned warm start, at 3600x2400);
  * a step solves A eta_n = b_n to ||b - A eta|| / ||b|| <= 1e-12 (FP64
    residual) on the GPU.

The first --train-steps steps of the sequence are solved in FP64 (untimed);
they are the history of the timed steps and the training set of the
warm-start U-Net, which is trained on them at start-up by the library's own
BF16 forward/backward kernels (untimed).

Arms reported in one JSON line:
  value        mixed precision (FP32 PCG + FP64 refinement) from the learned
               warm start (network inference inside the timing); inputs
               resident in HBM, device-timed
  linear_mixed the same steps from linear extrapolation 2 eta[n-1] - eta[n-2]
               (no network)
  fp64_plain   the plain FP64 SEVP-PCG from a zero guess on the same steps
  e2e          the value arm through the C ABI with host buffers (b_n,
               eta_{n-1}, eta_{n-2} in, eta_n out, copies inside the timing)
  roofline     the dominant kernel (tile SEVP pass B) against measured HBM
  cpu_baseline the CPU oracle (FP64 tile-SEVP PCG, OpenMP) on the host cores

Every vector is larger than the 126 MB L2 (69 MB per FP64 field; ~1 GB of
traffic per PCG iteration), so no explicit L2 flush is done between steps.

``--impl reference`` times the CPU implementation of the method (the oracle
port; the reference's own full-width REP1 needs > 60 GB of influence
matrices at 3600 columns and its unpreconditioned BiCGSTAB needs thousands
of iterations, so neither finishes in minutes) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s to 1e-12 rel. residual at 3600x2400: learned+mixed vs plain FP64 SEVP"
NX, NY = 3600, 2400
# tile shape of the CPU oracle arms; the GPU arm autotunes its own (16x8 is
# what the autotuner picks on a B200 at 3600x2400)
TILE_M, TILE_H, GROWTH = 16, 8, 1e10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precond-fp32", type=int, default=0,
                    help="FP32 influence matrices in the inner FP32 solve of the mixed arms")
    ap.add_argument("--train-steps", type=int, default=40,
                    help="leading steps of the sequence solved in FP64 and used to train the "
                         "warm-start network (untimed)")
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--coarse", type=int, default=8, choices=[1, 2, 4, 8],
                    help="the network runs on the grid averaged over coarse x coarse cells")
    ap.add_argument("--tiles", default="auto",
                    help="tile shape MxH of the GPU solver, or 'auto' (measured at start-up)")
    ap.add_argument("--precond", default="auto", choices=["auto", "bj", "schwarz"],
                    help="block-Jacobi tiles, the overlapping Schwarz sweep, or 'auto' (measured)")
    ap.add_argument("--inner-tol", default="auto",
                    help="relative reduction of each FP32 inner solve, or 'auto' (measured)")
    ap.add_argument("--no-fs", action="store_true",
                    help="skip the barotropic correction loop arm (3600x2400, 20 layers)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 64-member 720x360 ensemble arm")
    ap.add_argument("--no-learned", action="store_true",
                    help="value arm from linear extrapolation instead of the network")
    return ap.parse_args()


# ------------------------------------------------------------------ utils
class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(nx, ny, tiles, kernel="passb"):
    """Per-launch DRAM bytes from the committed ncu summaries (profiles/):
    the FP32 pass-B kernel ("passb") or the Schwarz stage kernel averaged
    over stages 2 and 3 ("couple"); None when the summary covers another
    grid or tile shape (they are 3600x2400 captures with 16x6 tiles)."""
    if (nx, ny, tuple(tiles)) != (3600, 2400, (16, 6)):
        return None
    name, key = {"passb": ("tile_pass_b_3600x2400.md", "traffic_bytes_per_launch_mixed:"),
                 "couple": ("schwarz_stages_3600x2400.md", "traffic_bytes_per_launch_avg:")}[kernel]
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith(key):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def make_sequence(nx, ny, nsteps):
    from musoc_solver_b200 import problems as P

    p = P.global_grid(nx, ny, seed=11)
    rhs = [b for _, b in P.eddy_rhs(nx, ny, range(nsteps), seed=3)]
    wet = p.meta["wet"]
    rhs = [np.where(wet, b, 0.0) for b in rhs]
    return p, rhs


def dist_setup(args):
    """One process per GPU (torchrun): NCCL on the GPU box; gloo on a host
    without a GPU, where only the CPU reference arm runs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def max_over_ranks(v, dist, device):
    """The largest v over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------ CPU oracle
def cpu_solve_seconds(p, b, threads, tile_nb=None, tiles=(TILE_M, TILE_H)):
    """One FP64 tile-SEVP PCG solve with the CPU oracle (setup excluded),
    with the same tile layout as the GPU solver."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from musoc_solver_b200.solver import tile_sub_blocks

    if tile_nb is None:
        tile_nb = tile_sub_blocks(p, tiles[0], tiles[1], GROWTH)
    pc = O.TilePC(p, tiles[0], tiles[1], tile_nb=tile_nb)
    t = time.perf_counter()
    x, it, rel = pc.pcg(b, tol=1e-12)
    dt = time.perf_counter() - t
    return dt, it, rel


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    p, rhs = make_sequence(args.nx, args.ny, args.warmup + args.steps)
    times, iters = [], []
    for n in range(args.warmup + args.steps):
        dt, it, rel = cpu_solve_seconds(p, rhs[n], cores)
        if n >= args.warmup:
            times.append(dt)
            iters.append(it)
    total = sum(times)
    value = len(times) / total
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.nx}x{args.ny} global grid, eddy right-hand-side sequence, "
                               f"FP64 tile-SEVP PCG ({TILE_M}x{TILE_H} tiles) to 1e-12, zero guess",
                   "grid": [args.nx, args.ny], "tol": 1e-12, "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": "one full FP64 tile-SEVP PCG solve per step with the C oracle "
                                   f"(OpenMP, {cores} threads), setup excluded; mean iterations "
                                   f"{float(np.mean(iters)):.1f}"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- ensemble
def run_ensemble(K, W, members=64, nx=720, ny=360, schwarz=False, inner_tol=1e-5):
    """64 members x 720x360 (independently perturbed depths and right-hand
    sides) stacked into one system: every kernel launch covers all members."""
    import torch

    from musoc_solver_b200 import problems as P
    from musoc_solver_b200.ensemble import EnsembleSolver

    t0 = time.perf_counter()
    ms = P.ensemble(members=members, nx=nx, ny=ny, seed=5)
    e = EnsembleSolver(ms)
    setup_s = time.perf_counter() - t0
    b = e.rhs()
    stream = e.solver.stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": f"{members} members x {nx}x{ny}, +-5% depth noise, own right-hand sides, "
                       f"stacked ({e.problem.nx}x{e.problem.ny}), tiles {e.solver.tile_m}x{e.solver.tile_h}",
           "setup_seconds": setup_s}
    arms = [("mixed", 1, False), ("fp64", 0, False)]
    if schwarz:
        arms += [("mixed_schwarz", 1, True), ("fp64_schwarz", 0, True)]
    for name, prec, sw in arms:
        if sw != bool(e.solver.schwarz_shift):
            e.solver.set_schwarz(-1 if sw else 0)
        x = torch.zeros_like(b)
        for _ in range(W):
            e.solve(b, x=x.zero_(), precision=prec, inner_tol=inner_tol)
        torch.cuda.synchronize()
        ev0.record(stream)
        res = None
        for _ in range(K):
            x.zero_()
            x, res, _ = e.solve(b, x=x, precision=prec, inner_tol=inner_tol)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3
        rel = e.member_residuals(b, x)
        out[name] = {"value": members * K / t, "unit": "member solves/s", "ms_per_ensemble": 1e3 * t / K,
                     "iterations": res.iterations, "max_member_rel_residual": float(rel.max())}
        if name == "mixed":
            xm = x.clone()
        if name == "fp64":
            x64 = x.clone()
    # per-member error of the mixed solve against the FP64 solve
    d = (xm - x64).reshape(members, -1).abs().amax(dim=1)
    ref = x64.reshape(members, -1).abs().amax(dim=1)
    out["mixed"]["max_member_rel_err_vs_fp64"] = float((d / ref).max())
    e.close()
    return out


# ------------------------------------------------ barotropic correction loop
def run_fs(nx, ny, k1, tiles, passes=3, peak=None, schwarz=False, inner_tol=1e-5):
    """The FS barotropic correction (ITMASK loop) on a layered state: one
    pass = land masking, continuity right-hand side, mixed solve, P0 and
    velocity correction of every layer."""
    import torch

    from musoc_solver_b200 import problems as P
    from musoc_solver_b200.barotropic import BarotropicCorrection

    st = P.fs_state(nx, ny, k1, seed=7)
    bc = BarotropicCorrection(st, tile_m=tiles[0], tile_h=tiles[1], schwarz=schwarz)
    u, v, p0, scr = bc.upload()
    stream = bc.solver.stream
    bc.run(u, v, p0, scr, tolerance=0.0, mxmask=1, inner_tol=inner_tol)  # warm-up pass
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    n_pass, vmax, iters = bc.run(u, v, p0, scr, tolerance=0.0, mxmask=passes, inner_tol=inner_tol)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_loop = ev0.elapsed_time(ev1) / n_pass

    def time_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / reps

    n = nx * ny
    t_rhs = time_ms(lambda: bc.rhs(u, v, b=bc.b))
    t_cor = time_ms(lambda: bc.correct(bc.x, u, v, p0, scr))
    # algorithmic bytes: rhs reads U and V of every layer, writes b; the
    # correction reads X and masks, reads and writes U, V, P0 and 4 SCR planes
    b_rhs = n * (8 * k1 + 8)
    b_cor = n * (8 + 12 * k1 + 8 + 8 + 16)
    gbs = lambda b, ms: b / (ms * 1e-3) / 1e9
    out = {"workload": f"{nx}x{ny} interior, {k1} layers, land masks from the synthetic depth; "
                       f"mixed solve to 1e-12, tiles {tiles[0]}x{tiles[1]}"
                       f"{', Schwarz preconditioner' if schwarz else ''}",
           "ms_per_pass": t_loop, "passes": n_pass, "pcg_iterations": iters,
           "land_velocity_after": vmax,
           "rhs_ms": t_rhs, "rhs_gbs": gbs(b_rhs, t_rhs), "correct_ms": t_cor,
           "correct_gbs": gbs(b_cor, t_cor)}
    if peak:
        out["rhs_frac"] = gbs(b_rhs, t_rhs) / peak
        out["correct_frac"] = gbs(b_cor, t_cor) / peak
    bc.close()
    return out


# ---------------------------------------------------------------- native
def run_native(args, world, rank, local, dist):
    import torch

    from musoc_solver_b200 import build, native as N
    from musoc_solver_b200.solver import SevpSolver

    build.build()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup

    T = max(args.train_steps, 4)
    nsteps = T + W + K
    p, rhs = make_sequence(args.nx, args.ny, nsteps)
    n = p.nx * p.ny
    # the leading T steps: FP64 solves from linear extrapolation (untimed);
    # they are the history of the timed steps and the network's training set
    # (block-Jacobi 16x6 tiles; the solutions do not depend on the solver
    # configuration beyond the 1e-12 tolerance)
    from musoc_solver_b200.autotune import CANDIDATES, SCHWARZ_MAX_ROWS, autotune
    from musoc_solver_b200.warmstart import LearnedWarmStart, solve_sequence, train

    b_dev = [torch.from_numpy(b).to(dev) for b in rhs]
    base = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH, precond_fp32=args.precond_fp32)
    eta = solve_sequence(base, b_dev[:T])

    # tile shape, preconditioner and inner tolerance: measured (untimed) on
    # step T-1 from the linear extrapolation of its history, the warm start
    # the timed arms use, unless all three are given
    tune_table = None
    cands = CANDIDATES if args.tiles == "auto" else (
        tuple(int(v) for v in args.tiles.lower().split("x")),)
    sw_opts = {"auto": (False, True), "bj": (False,), "schwarz": (True,)}[args.precond]
    itols = (1e-5, 1e-6) if args.inner_tol == "auto" else (float(args.inner_tol),)
    if len(cands) * len(sw_opts) * len(itols) > 1:
        best, tune_table = autotune(p, b_dev[T - 1], candidates=cands, precision=1,
                                    growth_limit=GROWTH, schwarz=sw_opts, inner_tols=itols,
                                    history=(eta[T - 2], eta[T - 3]))
        tiles, use_sw, itol = (best["tile_m"], best["tile_h"]), best["schwarz"], best["inner_tol"]
    else:
        tiles, use_sw, itol = cands[0], sw_opts[0], itols[0]
    if dist is not None:
        # every rank runs the same arms (and so the same collectives): rank
        # 0's choice holds for all
        choice = [(tuple(tiles), bool(use_sw), float(itol))]
        dist.broadcast_object_list(choice, src=0)
        tiles, use_sw, itol = choice[0]
    if use_sw and tiles[1] > SCHWARZ_MAX_ROWS:
        raise SystemExit(f"the Schwarz preconditioner needs tiles of at most {SCHWARZ_MAX_ROWS} rows")
    if tuple(tiles) == (16, 6) and not use_sw:
        solver = base
    else:
        base.close()
        solver = SevpSolver(p, tile_m=tiles[0], tile_h=tiles[1], growth_limit=GROWTH,
                            precond_fp32=args.precond_fp32, schwarz=use_sw)
    stream = solver.stream
    torch.cuda.synchronize()

    eta += [torch.zeros_like(eta[0]) for _ in range(W + K)]
    guess_mode, guess_name = N.GUESS_LINEAR, "linear extrapolation 2*eta[n-1]-eta[n-2]"
    warm, train_info = None, None
    if not args.no_learned:
        t0 = time.perf_counter()
        trainer = LearnedWarmStart.create(solver, seed=0, train=True, coarse=args.coarse)
        losses = train(trainer, eta, b_dev, list(range(2, T)), epochs=args.epochs, lr=2e-3,
                       lr_final=2e-4)
        warm = trainer.inference_copy()
        del trainer
        torch.cuda.synchronize()
        warm.attach(solver)
        guess_mode = N.GUESS_LEARNED
        guess_name = (f"learned: U-Net (4 levels, 32 base channels, BF16) on the "
                      f"{warm.net.H}x{warm.net.W} grid ({args.coarse}x{args.coarse} averages), "
                      "correction added to 2*eta[n-1]-eta[n-2] + one tile-SEVP solve")
        train_info = {"steps": T - 2, "epochs": args.epochs, "seconds": time.perf_counter() - t0,
                      "loss_first": losses[0][1], "loss_last": losses[-1][1],
                      "network_grid": [warm.net.W, warm.net.H]}

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()


    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timed = range(T + W, T + W + K)

    def run_arm(mode, hist):
        """Warm-up and timed steps of a sequence arm; hist holds the solutions."""
        for k in range(T, T + W):
            solver.solve_step(b_dev[k], hist[k - 1], hist[k - 2], hist[k], guess=mode, precision=1,
                              inner_tol=itol)
        barrier()
        reps = []
        l0 = solver.launches()
        ev0.record(stream)
        for k in timed:
            _, r = solver.solve_step(b_dev[k], hist[k - 1], hist[k - 2], hist[k], guess=mode,
                                     precision=1, inner_tol=itol)
            reps.append(r)
        ev1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist, dev), reps, solver.launches() - l0

    # ---- value arm: mixed precision + warm start, device-resident inputs
    with ClockSampler(local) as clk:
        t_value, reps, launches_value = run_arm(guess_mode, eta)
    # per-kernel device times of the same steps, from an untimed replay with
    # CUDA events around every launch (the events and the direct launches
    # they need would slow the timed arm)
    solver.profile(True)
    run_arm(guess_mode, eta)
    prof = solver.profile_read()
    solver.profile(False)
    relres = [r.rel_residual for r in reps]
    status = [r.status for r in reps]

    # ---- the same sequence from linear extrapolation (no network)
    eta_lin = eta[:T] + [torch.zeros_like(eta[0]) for _ in range(W + K)]
    t_lin, reps_lin, _ = run_arm(N.GUESS_LINEAR, eta_lin)
    del eta_lin

    # error of the value arm against an FP64 solve of the same steps
    ref_x = torch.zeros_like(eta[0])
    errs = []
    for k in (timed[0], timed[-1]):
        solver.solve(b_dev[k], x=ref_x.zero_(), precision=0)
        errs.append(float((eta[k] - ref_x).abs().max() / ref_x.abs().max()))

    # ---- plain FP64 SEVP-PCG from a zero guess (block-Jacobi tiles)
    def fp64_zero_arm():
        xz = torch.zeros_like(eta[0])
        for k in range(T, T + W):
            solver.solve(b_dev[k], x=xz.zero_(), precision=0)
        barrier()
        ev0.record(stream)
        its = []
        for k in timed:
            _, r = solver.solve(b_dev[k], x=xz.zero_(), precision=0)
            its.append(r.iterations)
        ev1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist, dev), its

    if use_sw:
        solver.set_schwarz(0)
    t_fp64, it64 = fp64_zero_arm()
    fp64_sw = None
    if use_sw:
        solver.set_schwarz(-1)
        t_sw, it_sw = fp64_zero_arm()
        fp64_sw = {"value": world * K / t_sw, "unit": "solves/s", "ms_per_step": 1e3 * t_sw / K,
                   "mean_iterations": float(np.mean(it_sw))}
    xz = torch.zeros_like(eta[0])

    # ---- mixed precision from a zero guess (isolates the precision gain)
    barrier()
    ev0.record(stream)
    itmz = []
    for k in timed:
        _, r = solver.solve(b_dev[k], x=xz.zero_(), precision=1, inner_tol=itol)
        itmz.append(r.iterations)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_mixed0 = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist, dev)

    # ---- e2e: the same value arm through the C ABI with host buffers.
    #      The context keeps the last two solutions in device memory, so a
    #      step copies b in and x out (pinned buffers).  Headline: the
    #      asynchronous steps (step n+1's b prefetched during step n's
    #      solve, x copied out on a copy stream); beside it the synchronous
    #      step, and the steps with the history copied in every step.
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    b_host = {k: pin(rhs[k]) for k in range(T, T + W + K)}
    eta_host = {k: pin(np.zeros((p.ny, p.nx))) for k in range(T - 2, T + W + K)}
    for k in (T - 2, T - 1):
        eta_host[k][:] = eta[k].cpu().numpy()
    solver.step_history(eta_host[T - 1], eta_host[T - 2])
    for k in range(T, T + W):
        solver.step_submit(b_host[k], eta_host[k], guess=guess_mode, precision=1, inner_tol=itol)
    solver.step_wait()
    barrier()
    t0 = time.perf_counter()
    l1 = solver.launches()
    solver.step_prefetch(b_host[timed[0]])
    for k in timed:
        if k + 1 in timed:
            solver.step_prefetch(b_host[k + 1])
        solver.step_submit(b_host[k], eta_host[k], guess=guess_mode, precision=1, inner_tol=itol)
    solver.step_wait()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, dist, dev)
    launches_e2e = solver.launches() - l1
    h2d = 8 * n
    d2h = 8 * n
    # the synchronous step (history on the device, copies not overlapped)
    solver.step_history(eta_host[timed[0] - 1], eta_host[timed[0] - 2])
    barrier()
    t0 = time.perf_counter()
    for k in timed:
        solver.step_host(b_host[k], eta_host[k], guess=guess_mode, precision=1, inner_tol=itol)
    torch.cuda.synchronize()
    t_e2e_sync = max_over_ranks(time.perf_counter() - t0, dist, dev)
    barrier()
    t0 = time.perf_counter()
    for k in timed:
        solver.solve_step_host(b_host[k], eta_host[k - 1], eta_host[k - 2], eta_host[k],
                               guess=guess_mode, precision=1, inner_tol=itol)
    torch.cuda.synchronize()
    t_e2e_hist = max_over_ranks(time.perf_counter() - t0, dist, dev)
    h2d_hist = 8 * n * (3 if guess_mode in (N.GUESS_LINEAR, N.GUESS_LEARNED) else 2)

    # ---- roofline of the dominant kernel (FP32 vectors): pass B with the
    #      block-Jacobi preconditioner, the Schwarz stage kernel otherwise
    peak, peak_kind = measured_peak_hbm()
    tile_ms, tile_n = prof["tile"]
    cpl_ms, cpl_n = prof["couple"]
    ncoef = 3 if solver.symmetric else 5
    scale = 0.5 if args.precond_fp32 else 1.0
    infl_a = int(solver.influence_bytes() * scale)
    infl_b = int(solver.schwarz_influence_bytes() * scale)
    # pass B: x,p,r,q in; x,r,z out (without r.z and z with the Schwarz
    # preconditioner: z1 out); coefficient planes; influence data
    b_passb = n * (4 * 4 + 3 * 4 + 4 * ncoef) + infl_a
    # Schwarz stages, per launch averaged over stage 2 (w in, z2 out) and
    # stage 3 (w, z1, r in, z out): halo rows of w (2 per tile row) and of
    # AT (symmetric storage), coefficient planes, the tiling's influence data
    halo = (2 * 4 + (4 if solver.symmetric else 0)) / tiles[1]
    b_stage2 = n * (4 + 4 + halo + 4 * ncoef) + infl_b
    b_stage3 = n * (4 + 4 + 4 + 4 + halo + 4 * ncoef) + infl_a
    b_couple = 0.5 * (b_stage2 + b_stage3)
    short_tiles = tiles[1] <= 6  # FP32 vectors with tiles up to 6 rows run the short-tile kernel
    passb_name = ("k_tile_short<float, update, dots>" if short_tiles
                  else "k_tile_apply<float, update, dots>") + " (PCG pass B)"
    if use_sw and cpl_n:
        dom_name = "k_tile_couple<float> (Schwarz stages 2 and 3, averaged per launch)"
        bytes_per_launch, avg_s, dom_n = b_couple, cpl_ms / 1e3 / cpl_n, cpl_n
        traffic = ncu_traffic(p.nx, p.ny, tiles, "couple")
    else:
        dom_name = passb_name
        bytes_per_launch, avg_s, dom_n = b_passb, tile_ms / 1e3 / max(tile_n, 1), tile_n
        traffic = ncu_traffic(p.nx, p.ny, tiles, "passb")
    achieved = bytes_per_launch / avg_s / 1e9 if dom_n else None

    # ---- 64-member ensemble (720x360 each), every launch over all members
    ens = None
    if not args.no_ensemble:
        ens = run_ensemble(max(2, K // 2), max(1, min(W, 2)), schwarz=True, inner_tol=itol)

    # ---- the barotropic correction loop around the solve (FS ITMASK loop)
    fs = None
    if not args.no_fs:
        fs = run_fs(p.nx, p.ny, 20, tiles, peak=peak, schwarz=use_sw, inner_tol=itol)

    # ---- CPU baseline (rank 0 at N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        dt, itc, relc = cpu_solve_seconds(p, rhs[timed[0]], cores, solver.tile_nb, tiles)
        cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": f"one full FP64 tile-SEVP PCG solve of step {timed[0]} with the C oracle "
                         f"(OpenMP, {cores} threads, {itc} iterations, rel. residual {relc:.2e}), "
                         "setup excluded"}

    value = world * K / t_value
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": 1e3 * t_value / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic",
        "config": {
            "workload": f"{p.nx}x{p.ny} global grid (lat +-78, ~30% land, dt=60 s), eddy "
                        "right-hand-side sequence; mixed FP32 tile-SEVP PCG + FP64 iterative "
                        f"refinement to 1e-12 from warm start: {guess_name}",
            "grid": [p.nx, p.ny], "tiles": list(tiles),
            "preconditioner": (f"overlapping Schwarz, second tiling shifted by "
                               f"{solver.schwarz_shift} columns" if use_sw else "block-Jacobi tiles"),
            "inner_tol": itol,
            "tile_autotune": None if tune_table is None else
            {f"{r['tile_m']}x{r['tile_h']}{' schwarz' if r['schwarz'] else ''} itol={r['inner_tol']:g}":
             round(r["ms"], 2) for r in tune_table},
            "tile_autotune_workload": "one warm-start step (linear extrapolation), mixed solve",
            "marching_growth_limit": GROWTH,
            "coefficient_planes": 3 if solver.symmetric else 5,
            "influence_fp32_in_inner_solve": bool(args.precond_fp32),
            "tol": 1e-12, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (69 MB per FP64 field), no flush",
        },
        "fp64_plain": {"value": world * K / t_fp64, "unit": "solves/s",
                       "ms_per_step": 1e3 * t_fp64 / K,
                       "mean_iterations": float(np.mean(it64)),
                       "preconditioner": "block-Jacobi tiles"},
        "fp64_schwarz_zero_guess": fp64_sw,
        "mixed_zero_guess": {"value": world * K / t_mixed0, "unit": "solves/s",
                             "mean_iterations": float(np.mean(itmz))},
        "linear_mixed": {"value": world * K / t_lin, "unit": "solves/s",
                         "ms_per_step": 1e3 * t_lin / K,
                         "mean_iterations": float(np.mean([r.iterations for r in reps_lin]))},
        "warm_start_training": train_info,
        "value_arm": {"mean_iterations": float(np.mean([r.iterations for r in reps])),
                      "mean_refinements": float(np.mean([r.refinements for r in reps])),
                      "max_rel_residual": float(max(relres)), "status": sorted(set(status)),
                      "max_rel_err_vs_fp64": float(max(errs))},
        "speedup_vs_fp64_plain": (K / t_value) / (K / t_fp64),
        "e2e": {"value": world * K / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "api": "sevp_step_prefetch / sevp_step_submit / sevp_step_wait (history of the "
                       "two previous solutions held in HBM; copies overlapped with the solves)"},
        "e2e_step_host": {"value": world * K / t_e2e_sync, "unit": "solves/s",
                          "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                          "api": "sevp_step_host (history in HBM, copies not overlapped)"},
        "e2e_history_from_host": {"value": world * K / t_e2e_hist, "unit": "solves/s",
                                  "h2d_bytes_per_step": h2d_hist, "d2h_bytes_per_step": d2h,
                                  "api": "sevp_solve_step_host (b, eta1, eta2 copied in)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": dom_name,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": avg_s * 1e3, "launches": dom_n,
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
        "kernels": {"tile_pass_b": {"launches": tile_n,
                                    "avg_ms": tile_ms / max(tile_n, 1),
                                    "hbm_frac": (b_passb / (tile_ms / 1e3 / tile_n) / 1e9 / peak)
                                    if tile_n else None},
                    "schwarz_stages": {"launches": cpl_n, "avg_ms": cpl_ms / max(cpl_n, 1),
                                       "hbm_frac": (b_couple / (cpl_ms / 1e3 / cpl_n) / 1e9 / peak)
                                       if cpl_n else None},
                    "stencil": {"launches": prof["stencil"][1],
                                "avg_ms": prof["stencil"][0] / max(prof["stencil"][1], 1)},
                    "precondition_start": {"launches": prof["precond"][1],
                                           "avg_ms": prof["precond"][0] / max(prof["precond"][1], 1)}},
        "ensemble_c5": ens,
        "fs_barotropic_loop": fs,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches_value),
        "gpu_launches_e2e": int(launches_e2e),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if warm is not None:
        warm.close()
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return rc
    return run_native(args, world, rank, local, dist)


if __name__ == "__main__":
    sys.exit(main())
