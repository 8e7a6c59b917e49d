"""Parity of the native sm_100a SEVP-PCG path against the CPU oracle.

Tolerances:
  * operator apply: relative 1e-13 (FP64; the GPU fuses multiply-adds);
  * tile preconditioner z = M^-1 r: relative 1e-8 of max|z| (marching
    amplifies rounding by at most the growth bound used to pick sub-block
    heights, 1e6, on top of ~1e-16);
  * solves: ||b - A x|| / ||b|| <= 1e-12 (FP64), and max|x - x_oracle| <=
    1e-8 max|x_oracle| (both satisfy the same residual bound).
"""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


def _solver(p, tm, th, srow=None):
    from musoc_solver_b200.solver import SevpSolver

    # growth bound 1e6: marching rounding stays ~1e-10, so the GPU and the
    # oracle preconditioners agree tightly
    return SevpSolver(p, tile_m=tm, tile_h=th, sub_rows=srow, growth_limit=1e6)


CASES = [
    ("basin", lambda: P.basin(0), 24, 24),
    ("basin16", lambda: P.basin(1), 16, 16),
    ("global_small", lambda: P.global_grid(180, 90, seed=2), 16, 16),
    ("ragged", lambda: P.global_grid(100, 70, seed=3), 12, 9),
    ("ragged32", lambda: P.global_grid(150, 77, seed=4), 32, 20),
    # short tiles (FP32 vectors run the all-rows-in-registers kernel)
    ("short6", lambda: P.global_grid(180, 90, seed=5), 16, 6),
    ("short4ragged", lambda: P.global_grid(100, 70, seed=6), 16, 4),
    ("tiny", lambda: P.basin(2, n=7), 8, 3),
]


@pytest.mark.parametrize("name,mk,tm,th", CASES)
def test_apply_matches_oracle(torch_cuda, oracle, name, mk, tm, th):
    torch = torch_cuda
    p = mk()
    s = _solver(p, tm, th)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((p.ny, p.nx))
    y = s.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    yo = oracle.apply(p, x)
    assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()


@pytest.mark.parametrize("name,mk,tm,th", CASES)
def test_precondition_matches_oracle(torch_cuda, oracle, name, mk, tm, th):
    torch = torch_cuda
    p = mk()
    s = _solver(p, tm, th)
    pc = oracle.TilePC(p, tm, th, tile_nb=s.tile_nb)
    assert pc.status == 0
    rng = np.random.default_rng(1)
    r = rng.standard_normal((p.ny, p.nx))
    z = s.precondition(torch.from_numpy(r).cuda()).cpu().numpy()
    zo = pc.apply(r)
    assert np.isfinite(z).all()
    assert np.abs(z - zo).max() <= 1e-8 * np.abs(zo).max()
    # FP32 vectors, FP64 marching: rounding of r and z only
    z32 = s.precondition(torch.from_numpy(r.astype(np.float32)).cuda()).cpu().numpy()
    assert np.abs(z32 - zo).max() <= 1e-5 * np.abs(zo).max()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,mk,tm,th", CASES[:-1])
def test_solve_matches_oracle(torch_cuda, oracle, name, mk, tm, th, precision):
    torch = torch_cuda
    p = mk()
    s = _solver(p, tm, th)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=precision, tol=1e-12)
    assert rep.status == 0
    assert rep.rel_residual <= 1e-12
    xg = x.cpu().numpy()
    # independent FP64 residual on the host
    res = np.linalg.norm(p.b - P.apply_operator(p, xg)) / np.linalg.norm(p.b)
    assert res <= 2e-12
    pc = oracle.TilePC(p, tm, th, tile_nb=s.tile_nb)
    xo, it, rel = pc.pcg(p.b, tol=1e-12)
    assert rel <= 1e-12
    assert np.abs(xg - xo).max() <= 1e-8 * np.abs(xo).max()
    if precision == 0:
        # same method, same arithmetic up to reduction order: same iteration count +-2
        assert abs(rep.iterations - it) <= 2


def test_solve_host_and_guess(torch_cuda, oracle):
    p = P.global_grid(180, 90, seed=5)
    s = _solver(p, 16, 16)
    x, rep = s.solve_host(p.b, precision=1)
    assert rep.rel_residual <= 1e-12
    # warm start from the solution converges immediately
    x2, rep2 = s.solve_host(p.b, x=x, precision=0)
    assert rep2.iterations == 0 and rep2.rel_residual <= 1e-12
    # warm start from a perturbed solution needs fewer iterations than zero
    xp = x * (1.0 + 1e-6 * np.random.default_rng(0).standard_normal(x.shape))
    x3, rep3 = s.solve_host(p.b, x=xp, precision=0)
    _, rep0 = s.solve_host(p.b, precision=0)
    assert rep3.rel_residual <= 1e-12 and rep3.iterations < rep0.iterations


def test_relative_residual_and_zero_rhs(torch_cuda):
    torch = torch_cuda
    p = P.basin(3)
    s = _solver(p, 24, 24)
    b = torch.zeros((p.ny, p.nx), dtype=torch.float64, device="cuda")
    x, rep = s.solve(b, precision=0)
    assert rep.status == 0 and rep.iterations == 0
    assert float(x.abs().max()) == 0.0


def test_nonfinite_rhs_reports_status(torch_cuda):
    torch = torch_cuda
    from musoc_solver_b200 import native as N

    p = P.basin(4)
    s = _solver(p, 24, 24)
    b = torch.from_numpy(p.b).cuda()
    b[5, 5] = float("nan")
    with pytest.raises(N.SevpError) as e:
        s.solve(b, precision=0)
    assert e.value.status == N.SEVP_NONFINITE
    # context stays usable
    x, rep = s.solve(torch.from_numpy(p.b).cuda(), precision=0)
    assert rep.status == 0


def test_max_iter_status(torch_cuda):
    torch = torch_cuda
    p = P.global_grid(180, 90, seed=6)
    s = _solver(p, 16, 16)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=0, max_iter=3)
    assert rep.status == 1 and rep.iterations == 3 and rep.rel_residual > 1e-12


def test_symmetric_storage_matches_full(torch_cuda, oracle):
    """The 3-plane kernels (exactly symmetric operators) give the same apply,
    preconditioner and solve as the 5-plane kernels."""
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(180, 90, seed=12)
    s3 = SevpSolver(p, tile_m=16, tile_h=16, growth_limit=1e6)
    s5 = SevpSolver(p, tile_m=16, tile_h=16, growth_limit=1e6, full_coefficients=True)
    assert s3.symmetric and not s5.symmetric
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal((p.ny, p.nx))).cuda()
    a3, a5 = s3.apply(x).cpu().numpy(), s5.apply(x).cpu().numpy()
    assert np.abs(a3 - a5).max() <= 1e-14 * np.abs(a5).max()
    z3, z5 = s3.precondition(x).cpu().numpy(), s5.precondition(x).cpu().numpy()
    assert np.abs(z3 - z5).max() <= 1e-12 * np.abs(z5).max()
    b = torch.from_numpy(p.b).cuda()
    for prec in (0, 1):
        x3, r3 = s3.solve(b, precision=prec)
        x5, r5 = s5.solve(b, precision=prec)
        assert r3.rel_residual <= 1e-12 and r5.rel_residual <= 1e-12
        assert np.abs((x3 - x5).cpu().numpy()).max() <= 1e-9 * float(x5.abs().max())


def test_nonsymmetric_operator_uses_full_planes(torch_cuda, oracle):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.basin(5, n=64)
    rng = np.random.default_rng(5)
    p.al *= (1.0 + 0.01 * rng.random(p.al.shape)).astype(np.float32)  # break symmetry
    s = SevpSolver(p, tile_m=16, tile_h=16, growth_limit=1e6)
    assert not s.symmetric
    x = rng.standard_normal((p.ny, p.nx))
    y = s.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    yo = oracle.apply(p, x)
    assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()
    pc = oracle.TilePC(p, 16, 16, tile_nb=s.tile_nb)
    z = s.precondition(torch.from_numpy(x).cuda()).cpu().numpy()
    zo = pc.apply(x)
    assert np.abs(z - zo).max() <= 1e-8 * np.abs(zo).max()


def test_mixed_with_fp32_influence(torch_cuda):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=13)
    s = SevpSolver(p, tile_m=16, tile_h=16, precond_fp32=True)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=1, tol=1e-12)
    assert rep.status == 0 and rep.rel_residual <= 1e-12
    res = np.linalg.norm(p.b - P.apply_operator(p, x.cpu().numpy())) / np.linalg.norm(p.b)
    assert res <= 2e-12


def test_step_host_keeps_history_on_device(torch_cuda):
    """sevp_step_host (history in device memory, b in and x out per step)
    gives the same solutions as device steps with the history passed in."""
    torch = torch_cuda
    from musoc_solver_b200 import native as N

    p = P.global_grid(180, 90, seed=7)
    rhs = [np.ascontiguousarray(b) for _, b in P.eddy_rhs(180, 90, range(6), seed=2)]
    s1, s2 = _solver(p, 16, 6), _solver(p, 16, 6)
    etas = []
    for n, b in enumerate(rhs):
        mode = N.GUESS_ZERO if n == 0 else (N.GUESS_PREVIOUS if n == 1 else N.GUESS_LINEAR)
        x = torch.zeros((p.ny, p.nx), dtype=torch.float64, device="cuda")
        s1.solve_step(torch.from_numpy(b).cuda(), etas[-1] if n >= 1 else None,
                      etas[-2] if n >= 2 else None, x, guess=mode, precision=1)
        etas.append(x)
    for n, b in enumerate(rhs):
        xh = np.zeros_like(b)
        _, rep = s2.step_host(b, xh, guess=N.GUESS_LINEAR, precision=1)
        assert rep.status == 0 and rep.rel_residual <= 1e-12
        assert np.array_equal(xh, etas[n].cpu().numpy()), n
    # a history loaded from the host
    e1, e2 = etas[-1].cpu().numpy(), etas[-2].cpu().numpy()
    s2.step_history(e1, e2)
    xh = np.zeros_like(rhs[0])
    s2.step_host(rhs[0], xh, guess=N.GUESS_LINEAR, precision=1)
    x = torch.zeros_like(etas[0])
    s1.solve_step(torch.from_numpy(rhs[0]).cuda(), etas[-1], etas[-2], x, guess=N.GUESS_LINEAR,
                  precision=1)
    assert np.array_equal(xh, x.cpu().numpy())


def test_step_submit_overlapped_copies_match_step_host(torch_cuda):
    """Asynchronous steps (next b prefetched before each submit, x copied out
    on a copy stream) give the same solutions as synchronous steps."""
    torch = torch_cuda
    from musoc_solver_b200 import native as N

    p = P.global_grid(180, 90, seed=8)
    rhs = [np.ascontiguousarray(b) for _, b in P.eddy_rhs(180, 90, range(7), seed=5)]
    pin = lambda a: torch.from_numpy(np.array(a)).pin_memory().numpy()
    bs = [pin(b) for b in rhs]
    xs = [pin(np.zeros_like(b)) for b in rhs]
    s1, s2 = _solver(p, 16, 6), _solver(p, 16, 6)
    ref = []
    for b in rhs:
        xh = np.zeros_like(b)
        s1.step_host(b, xh, guess=N.GUESS_LINEAR, precision=1)
        ref.append(xh)
    s2.step_prefetch(bs[0])
    for n in range(len(bs)):
        if n + 1 < len(bs):
            s2.step_prefetch(bs[n + 1])
        rep = s2.step_submit(bs[n], xs[n], guess=N.GUESS_LINEAR, precision=1)
        assert rep.status == 0 and rep.rel_residual <= 1e-12
    s2.step_wait()
    for n in range(len(bs)):
        assert np.array_equal(xs[n], ref[n]), n
    # a step submitted without a prefetch stages its own b
    s2.step_history(ref[-1], ref[-2])
    s1.step_history(ref[-1], ref[-2])
    xa, xb = pin(np.zeros_like(rhs[0])), np.zeros_like(rhs[0])
    s2.step_submit(bs[0], xa, guess=N.GUESS_LINEAR, precision=1)
    s2.step_wait()
    s1.step_host(rhs[0], xb, guess=N.GUESS_LINEAR, precision=1)
    assert np.array_equal(xa, xb)


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_at_the_1440x720_grid_matches_oracle(torch_cuda, oracle, precision):
    """Parity at a configuration's own size: the 1440x720 global grid (c2,
    16x6 tiles, growth bound 1e10), FP64 and mixed, against the oracle's
    FP64 tile PCG on all host cores; the residual recomputed on the host."""
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(1440, 720, seed=11)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e10)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=precision, tol=1e-12)
    assert rep.status == 0 and rep.rel_residual <= 1e-12
    xg = x.cpu().numpy()
    res = np.linalg.norm(p.b - P.apply_operator(p, xg)) / np.linalg.norm(p.b)
    assert res <= 2e-12
    pc = oracle.TilePC(p, 16, 6, tile_nb=s.tile_nb)
    xo, it, rel = pc.pcg(p.b, tol=1e-12)
    assert rel <= 1e-12
    assert np.abs(xg - xo).max() <= 1e-9 * np.abs(xo).max()
    if precision == 0:
        assert abs(rep.iterations - it) <= 2
