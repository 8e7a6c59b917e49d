"""Batched ensemble solves (all members in every launch) and the CUDA-graph
replay of the FP32 inner iterations."""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda_e():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


def test_graph_replay_matches_direct_launches(torch_cuda_e):
    torch = torch_cuda_e
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=5)
    s = SevpSolver(p, tile_m=16, tile_h=16)
    b = torch.from_numpy(p.b).cuda()
    s.graphs(False)
    x0, r0 = s.solve(b, precision=1)
    s.graphs(True)
    x1, r1 = s.solve(b, precision=1)
    x2, r2 = s.solve(b, precision=1)  # replays the captured interval
    assert r0.status == r1.status == r2.status == 0
    assert r0.iterations == r1.iterations == r2.iterations
    assert torch.equal(x0, x1) and torch.equal(x1, x2)
    assert r1.rel_residual <= 1e-12


@pytest.mark.parametrize("schwarz", [False, True])
def test_ensemble_members_reach_tolerance_and_match_single_solves(torch_cuda_e, oracle, schwarz):
    torch = torch_cuda_e
    from musoc_solver_b200.ensemble import EnsembleSolver
    from musoc_solver_b200.solver import SevpSolver

    members = P.ensemble(members=4, nx=96, ny=48, seed=9)
    e = EnsembleSolver(members, schwarz=schwarz)
    assert bool(e.solver.schwarz_shift) == schwarz
    b = e.rhs()
    x, res, rel = e.solve(b, precision=1)
    assert res.status == 0
    assert rel.shape == (4,) and float(rel.max()) <= 1e-12
    xs = x.reshape(4, 48, 96)
    for k, m in enumerate(members):
        sk = SevpSolver(m, tile_m=16, tile_h=e.solver.tile_h)
        xk, rk = sk.solve(torch.from_numpy(m.b).cuda(), precision=0)
        err = float((xs[k] - xk).abs().max() / xk.abs().max())
        assert err < 1e-9, (k, err)
        sk.close()
    # one member against the CPU oracle's FP64 tile-SEVP PCG
    from musoc_solver_b200.solver import tile_sub_blocks

    m = members[2]
    pc = oracle.TilePC(m, 16, 16, tile_nb=tile_sub_blocks(m, 16, 16, 1e10))
    xo, it, relo = pc.pcg(m.b, tol=1e-12)
    assert relo <= 1e-12
    err = np.abs(xs[2].cpu().numpy() - xo).max() / np.abs(xo).max()
    assert err < 1e-9
    e.close()
