"""Learned warm start trained on solver-generated solutions of an eddy
right-hand-side sequence, checked on held-out steps.

What the network must show: its guess is closer to the FP64 solution than
the guess without it (the same pipeline with the network output set to
zero: linear extrapolation plus one tile-SEVP solve of its residual), and
solving from it still reaches 1e-12.  Iterations for the zero, previous,
linear and learned guesses are reported (printed) for the record.
"""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coarse", [1, 2, 4, 8])
def test_learned_warm_start_beats_no_network(torch_cuda_ws, coarse):
    torch = torch_cuda_ws
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver
    from musoc_solver_b200.warmstart import LearnedWarmStart, evaluate, solve_sequence, train

    nx, ny, nsteps = 240, 120, 48
    p = P.global_grid(nx, ny, seed=21)
    wet = p.meta["wet"]
    rhs = [torch.from_numpy(np.where(wet, b, 0.0)).cuda()
           for _, b in P.eddy_rhs(nx, ny, range(nsteps), seed=4)]
    s = SevpSolver(p, tile_m=16, tile_h=16)
    etas = solve_sequence(s, rhs)
    warm = LearnedWarmStart.create(s, seed=0, train=True, coarse=coarse)
    train_idx = list(range(2, 36))
    test_idx = list(range(38, nsteps))
    losses = train(warm, etas, rhs, train_idx, epochs=6, lr=2e-3, lr_final=2e-4)
    assert losses[-1][1] < losses[0][1]
    # guess error with and without the network on held-out steps
    x = torch.zeros_like(etas[0])
    gain = []
    warm = warm.inference_copy()
    for n in test_idx:
        warm.predict(etas[n - 1], etas[n - 2], rhs[n], x)
        err_net = float((x - etas[n]).norm())
        err_base = float((warm.e + warm.m - etas[n]).norm())
        gain.append(err_base / err_net)
    warm.attach()
    res = evaluate(s, warm, etas, rhs, test_idx)
    print(f"coarse={coarse} warm start (mean iterations, ms):",
          {k: (v["mean_iterations"], round(v["mean_ms"], 3)) for k, v in res.items()},
          "guess-error ratio (no network / network):", np.round(gain, 2))
    assert np.median(gain) > 1.0
    assert res["learned"]["max_rel_err_vs_fp64"] < 1e-9
    assert res["learned"]["mean_iterations"] <= res["previous"]["mean_iterations"]
    warm.close()


@pytest.fixture(scope="module")
def torch_cuda_ws():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


@pytest.mark.parametrize("coarse", [1, 4])
def test_features_match_numpy_restatement(torch_cuda_ws, oracle, coarse):
    """sevp_nn_features against numpy with the oracle's operator and tile
    preconditioner: e, d exact; m to the marching tolerance; scales (RMS of
    the coarse-cell averages) and the BF16 network input to BF16 rounding."""
    torch = torch_cuda_ws
    from musoc_solver_b200.solver import SevpSolver
    from musoc_solver_b200.warmstart import LearnedWarmStart

    nx, ny = 96, 48
    p = P.global_grid(nx, ny, seed=31)
    s = SevpSolver(p, tile_m=16, tile_h=8, growth_limit=1e6)
    rng = np.random.default_rng(32)
    eta1, eta2 = rng.standard_normal((2, ny, nx))
    b = p.b
    w = LearnedWarmStart.create(s, seed=0, train=False, coarse=coarse)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    e1, e2, bb = t(eta1), t(eta2), t(b)
    w.features(e1.data_ptr(), e2.data_ptr(), bb.data_ptr())
    torch.cuda.synchronize()
    e = 2.0 * eta1 - eta2
    d = eta1 - eta2
    assert np.array_equal(w.e.cpu().numpy(), e)
    assert np.array_equal(w.d.cpu().numpy(), d)
    r = b - oracle.apply(p, e)
    m = oracle.TilePC(p, 16, 8, tile_nb=s.tile_nb).apply(r)
    assert np.abs(w.m.cpu().numpy() - m).max() <= 1e-8 * np.abs(m).max()
    avg = lambda a: a.reshape(ny // coarse, coarse, nx // coarse, coarse).mean(axis=(1, 3))
    av = [avg(a) for a in (r, m, d)]
    sc = np.array([np.sqrt((a * a).mean()) for a in av])
    assert np.allclose(w.scales.cpu().numpy()[:3], sc, rtol=1e-5)
    H, W = w.net.H, w.net.W
    x = w.net.A["x"].float().cpu().numpy().reshape(H, W, -1)
    cy, cx = ny // coarse, nx // coarse
    for q in range(3):
        ref = av[q] / sc[q]
        got = x[:cy, :cx, q]
        assert np.abs(got - ref).max() <= 8e-3 * np.abs(ref).max() + 1e-6
        assert not x[cy:, :, q].any() and not x[:, cx:, q].any()
