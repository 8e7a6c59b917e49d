"""Overlapping Schwarz preconditioner on the GPU against the oracle.

The library forms each stage's residual from the couplings across the
previous tiling's boundaries; the oracle (``SchwarzPC``) forms it in full,
r - A z, and builds the second tiling on the grid rolled by the same shift.
Both agree up to the marching rounding.

Tolerances (growth bound 1e6, as the block-Jacobi parity tests):
  * preconditioner z = M^-1 r: relative 1e-8 of max|z| with FP64 vectors,
    1e-5 with FP32 vectors;
  * solves: ||b - A x|| / ||b|| <= 1e-12 and max|x - x_oracle| <= 1e-8
    max|x_oracle|; FP64 iteration counts within 2 of the oracle's PCG.
"""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu

GROWTH = 1e6


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


def _pair(oracle, p, tm, th, shift=True, **kw):
    from musoc_solver_b200.solver import SevpSolver, tile_sub_blocks

    s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=GROWTH, schwarz=shift, **kw)
    xs = s.schwarz_shift
    assert 0 < xs < tm
    pc = oracle.SchwarzPC(p, tm, th, xs, s.tile_nb,
                          tile_sub_blocks(oracle.rolled_grid(p, xs), tm, th, GROWTH))
    assert pc.status == 0
    return s, pc


CASES = [
    ("global16x6", lambda: P.global_grid(180, 90, seed=2), 16, 6),
    ("ragged16x5", lambda: P.global_grid(100, 70, seed=3), 16, 5),
    ("basin16x8", lambda: P.basin(0), 16, 8),
    ("global8x8", lambda: P.global_grid(120, 64, seed=4), 8, 8),
    ("ragged32x6", lambda: P.global_grid(150, 77, seed=5), 32, 6),
    # nx mod tm == tm / 2: the half-tile shift would put a tile edge on the
    # seam, so another shift is chosen
    ("seam184", lambda: P.global_grid(184, 60, seed=6), 16, 6),
]


@pytest.mark.parametrize("name,mk,tm,th", CASES)
def test_schwarz_precondition_matches_oracle(torch_cuda, oracle, name, mk, tm, th):
    torch = torch_cuda
    p = mk()
    s, pc = _pair(oracle, p, tm, th)
    if name == "seam184":
        assert s.schwarz_shift != tm // 2
    rng = np.random.default_rng(7)
    r = rng.standard_normal((p.ny, p.nx))
    z = s.precondition(torch.from_numpy(r).cuda()).cpu().numpy()
    zo = pc.apply(r)
    assert np.isfinite(z).all()
    assert np.abs(z - zo).max() <= 1e-8 * np.abs(zo).max()
    z32 = s.precondition(torch.from_numpy(r.astype(np.float32)).cuda()).cpu().numpy()
    assert np.abs(z32 - zo).max() <= 1e-5 * np.abs(zo).max()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,mk,tm,th", CASES[:4])
def test_schwarz_solve_matches_oracle(torch_cuda, oracle, name, mk, tm, th, precision):
    torch = torch_cuda
    p = mk()
    s, pc = _pair(oracle, p, tm, th)
    x, rep = s.solve(torch.from_numpy(p.b).cuda(), precision=precision, tol=1e-12)
    assert rep.status == 0 and rep.rel_residual <= 1e-12
    xg = x.cpu().numpy()
    res = np.linalg.norm(p.b - P.apply_operator(p, xg)) / np.linalg.norm(p.b)
    assert res <= 2e-12
    xo, it, rel = pc.pcg(p.b, tol=1e-12)
    assert rel <= 1e-12
    assert np.abs(xg - xo).max() <= 1e-8 * np.abs(xo).max()
    if precision == 0:
        assert abs(rep.iterations - it) <= 2


def test_schwarz_needs_fewer_iterations(torch_cuda):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(360, 180, seed=8)
    b = torch.from_numpy(p.b).cuda()
    bj = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH)
    sw = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH, schwarz=True)
    for prec in (0, 1):
        _, rb = bj.solve(b, precision=prec)
        _, rs = sw.solve(b, precision=prec)
        assert rb.status == 0 and rs.status == 0
        assert rs.iterations * 2 <= rb.iterations
    # back to block-Jacobi: the same iterations as a block-Jacobi context
    sw.set_schwarz(0)
    assert sw.schwarz_shift == 0
    _, r0 = sw.solve(b, precision=0)
    _, rb0 = bj.solve(b, precision=0)
    assert r0.iterations == rb0.iterations


def test_schwarz_graph_replay_identical(torch_cuda):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=9)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH, schwarz=True)
    b = torch.from_numpy(p.b).cuda()
    s.graphs(False)
    x1, r1 = s.solve(b, precision=1)
    s.graphs(True)
    x2, r2 = s.solve(b, precision=1)
    x3, r3 = s.solve(b, precision=1)
    assert r1.iterations == r2.iterations == r3.iterations
    assert torch.equal(x1, x2) and torch.equal(x2, x3)


def test_schwarz_full_planes_and_fp32_influence(torch_cuda, oracle):
    torch = torch_cuda
    p = P.global_grid(180, 90, seed=10)
    s, pc = _pair(oracle, p, 16, 6, full_coefficients=True)
    assert not s.symmetric
    rng = np.random.default_rng(11)
    r = rng.standard_normal((p.ny, p.nx))
    z = s.precondition(torch.from_numpy(r).cuda()).cpu().numpy()
    zo = pc.apply(r)
    assert np.abs(z - zo).max() <= 1e-8 * np.abs(zo).max()
    from musoc_solver_b200.solver import SevpSolver

    s32 = SevpSolver(p, tile_m=16, tile_h=6, schwarz=True, precond_fp32=True)
    x, rep = s32.solve(torch.from_numpy(p.b).cuda(), precision=1, tol=1e-12)
    assert rep.status == 0 and rep.rel_residual <= 1e-12


def test_schwarz_rejects_bad_shapes(torch_cuda):
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(180, 90, seed=12)
    s = SevpSolver(p, tile_m=16, tile_h=16, growth_limit=GROWTH)
    with pytest.raises(N.SevpError):
        s.set_schwarz(-1)          # tiles higher than 8 rows
    assert s.schwarz_shift == 0
    s2 = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH)
    with pytest.raises(N.SevpError):
        s2.set_schwarz(16)         # shift must be inside a tile
    s2.set_schwarz(5)
    assert s2.schwarz_shift == 5


@pytest.mark.parametrize("schwarz", [False, True])
def test_condition_estimate_matches_dense_spectrum(torch_cuda, oracle, schwarz):
    """Ritz values from the recorded PCG coefficients against the dense
    spectrum of M^-1 A built with the oracle's preconditioner (small grid)."""
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver, tile_sub_blocks

    p = P.global_grid(48, 24, seed=13)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=GROWTH, schwarz=schwarz)
    rng = np.random.default_rng(14)
    b = rng.standard_normal((p.ny, p.nx))
    est = s.condition_estimate(torch.from_numpy(b).cuda())
    if schwarz:
        pc = oracle.SchwarzPC(p, 16, 6, s.schwarz_shift, s.tile_nb,
                              tile_sub_blocks(oracle.rolled_grid(p, s.schwarz_shift), 16, 6, GROWTH))
    else:
        pc = oracle.TilePC(p, 16, 6, tile_nb=s.tile_nb)
    n = p.nx * p.ny
    MA = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        MA[:, j] = pc.apply(oracle.apply(p, e.reshape(p.ny, p.nx))).ravel()
    ev = np.sort(np.linalg.eigvals(MA).real)
    assert abs(est["lambda_max"] - ev[-1]) <= 1e-3 * ev[-1]
    assert abs(est["lambda_min"] - ev[0]) <= 1e-2 * ev[0]
    assert est["iterations"] >= 2
