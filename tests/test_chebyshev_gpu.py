"""The one-launch Chebyshev iteration (SEVP_METHOD_CHEB) against the CPU
oracle.

Each iteration is one kernel launch: the operator is applied inside the tile
kernel to the previous launch's direction (its halo read from global
memory), then the tile SEVP solve runs.  It is a mixed-precision method
(FP32 vectors inside FP64 iterative refinement), so the bars are those of
the two-pass mixed solve:
  * one launch against the same step written with numpy and the oracle's
    A and M^-1: 1e-5 of the largest value (FP32 vectors);
  * ||b - A x|| / ||b|| <= 1e-12, recomputed on the host with the oracle's
    operator apply;
  * max|x - x_oracle| <= 1e-8 max|x_oracle| against the oracle's own
    Chebyshev iteration (or_cheb) on the same bounds;
  * the bounds from the library's CG-Lanczos estimate within 2e-3 of a numpy
    CG-Lanczos run with the oracle preconditioner (both are Ritz values of a
    finished solve, converged to a few digits).
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


CASES = [
    ("global16x6", lambda: P.global_grid(240, 120, seed=7), 16, 6),
    ("global16x8", lambda: P.global_grid(180, 90, seed=2), 16, 8),
    ("basin_closed", lambda: P.basin(1), 16, 6),
    ("ragged", lambda: P.global_grid(100, 70, seed=3), 12, 5),
    ("narrow8", lambda: P.global_grid(96, 64, seed=8), 8, 8),
    ("wide32", lambda: P.global_grid(150, 77, seed=4), 32, 6),
]


def _residual(p, x):
    return np.linalg.norm(p.b - P.apply_operator(p, x)) / np.linalg.norm(p.b)


def _solve(torch, s, p, method, **kw):
    from musoc_solver_b200 import native as N

    s.set_method(method)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=1, **kw)
    assert rep.status == 0, rep
    return x.cpu().numpy(), rep


@pytest.mark.parametrize("name,mk,tm,th", CASES[:4])
def test_single_chebyshev_launch_matches_numpy(torch_cuda, oracle, name, mk, tm, th):
    import ctypes as C

    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = mk()
    s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=1e6)
    pc = oracle.TilePC(p, tm, th, tile_nb=s.tile_nb)
    A = P.sparse_matrix(p)
    rng = np.random.default_rng(3)
    shape = (p.ny, p.nx)
    f32 = lambda: rng.standard_normal(shape).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    close = lambda got, ref: np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    theta, delta = 0.6, 0.45
    for it in (0, 1):
        d, r, x = f32(), f32(), f32()
        rho = delta / theta
        bd, br, bx, bo = dev(d), dev(r), dev(x), dev(np.zeros_like(d))
        rr = C.c_double()
        st = N.lib().sevp_cheb_step(s.h, it, theta, delta, rho, N.ptr(bd), N.ptr(bo), N.ptr(bx),
                                    N.ptr(br), C.byref(rr))
        torch.cuda.synchronize()
        assert st == 0
        dd = d.astype(np.float64) if it else np.zeros(shape)
        rn = r - (A @ dd.ravel()).reshape(shape)
        z = pc.apply(rn)
        if it:
            rho1 = 1.0 / (2.0 * theta / delta - rho)
            dn = rho1 * rho * dd + 2.0 * rho1 / delta * z
        else:
            dn = z / theta
        assert close(br.cpu().numpy(), rn) and close(bx.cpu().numpy(), x + dd), (name, it)
        assert close(bo.cpu().numpy(), dn), (name, it)
        assert abs(rr.value - (rn * rn).sum()) <= 1e-5 * (rn * rn).sum()
    s.close()


@pytest.mark.parametrize("name,mk,tm,th", CASES)
def test_fused_chebyshev_matches_oracle(torch_cuda, oracle, name, mk, tm, th):
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = mk()
    s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=1e6)
    b = torch.from_numpy(p.b).cuda()
    lo, hi = s.chebyshev_setup(b)
    assert 0 < lo < hi
    x, rep = _solve(torch, s, p, N.METHOD_CHEB)
    assert rep.rel_residual <= 1e-12 and _residual(p, x) <= 2e-12
    pc = oracle.TilePC(p, tm, th, tile_nb=s.tile_nb)
    xc, itc, relc = pc.cheb(p.b, lo * 0.98, hi * 1.02, tol=1e-12)
    assert relc <= 1e-12
    assert np.abs(x - xc).max() <= 1e-8 * np.abs(xc).max()
    s.close()


def test_bounds_match_numpy_lanczos(torch_cuda, oracle):
    from musoc_solver_b200.solver import SevpSolver

    from test_oracle_cpu import _lanczos_bounds

    torch = torch_cuda
    p = P.global_grid(160, 80, seed=3)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    lo, hi, it = s.estimate_bounds(torch.from_numpy(p.b).cuda())
    pc = oracle.TilePC(p, 16, 6, tile_nb=s.tile_nb)
    lo2, hi2 = _lanczos_bounds(p, pc)
    assert abs(lo - lo2) <= 2e-3 * lo2 and abs(hi - hi2) <= 2e-3 * hi2, (lo, hi, lo2, hi2)
    s.close()


def test_chebyshev_graph_replay_is_bit_identical(torch_cuda):
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(240, 120, seed=9)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e10)
    b = torch.from_numpy(p.b).cuda()
    s.chebyshev_setup(b)
    s.set_method(1)
    xg, rg = s.solve(b, precision=1)
    s.graphs(False)
    xd, rd = s.solve(b, precision=1)
    assert rg.iterations == rd.iterations
    assert torch.equal(xg, xd)
    s.close()


def test_fused_five_plane_and_fp32_influence(torch_cuda, oracle):
    """The 5-plane (full-storage) kernels and the FP32 influence data, on a
    small grid where FP32 influence data is accurate enough."""
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(180, 90, seed=2)
    for kw in (dict(full_coefficients=True), dict(precond_fp32=True)):
        s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e4, **kw)
        b = torch.from_numpy(p.b).cuda()
        s.chebyshev_setup(b)
        x, rep = _solve(torch, s, p, N.METHOD_CHEB)
        assert rep.rel_residual <= 1e-12 and _residual(p, x) <= 2e-12, kw
        s.close()


def test_chebyshev_refuses_unsupported_settings(torch_cuda):
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(96, 64, seed=1)
    b = torch.from_numpy(p.b).cuda()
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    s.set_method(N.METHOD_CHEB)
    with pytest.raises(N.SevpError, match="bounds"):
        s.solve(b, precision=1)  # no bounds yet
    o = s.opts(precision=0, method=N.METHOD_CHEB)
    import ctypes as C

    rep = N.Report()
    x = torch.zeros_like(b)
    assert N.lib().sevp_solve(s.h, N.ptr(b), N.ptr(x), C.byref(o), C.byref(rep)) == N.SEVP_BAD_ARG
    s.chebyshev_setup(b)
    s.set_schwarz(-1)
    with pytest.raises(N.SevpError, match="Schwarz"):
        s.solve(b, precision=1)
    s.close()
    s = SevpSolver(p, tile_m=16, tile_h=12, growth_limit=1e6)
    s.chebyshev_setup(b)
    s.set_method(N.METHOD_CHEB)
    with pytest.raises(N.SevpError, match="8 rows"):
        s.solve(b, precision=1)
    s.close()



def test_chebyshev_continues_across_residual_replacements(torch_cuda):
    """Mixed Chebyshev solves that continue the recurrence on each replaced
    FP64 residual (the default) and ones that restart it: both reach the
    tolerance, the continued one in at most one more iteration (odd and
    even check intervals, so the direction's buffer parity is exercised)."""
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(360, 180, seed=21)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    b = torch.from_numpy(p.b).cuda()
    s.chebyshev_setup(b)
    s.set_method(N.METHOD_CHEB)
    for ce in (3, 4):
        out = {}
        for restart in (False, True):
            s.restart_inner = restart
            x, rep = s.solve(b, precision=1, tol=1e-12, inner_tol=1e-4, check_every=ce)
            assert rep.status == 0 and rep.rel_residual <= 1e-12, (ce, restart, rep)
            assert _residual(p, x.cpu().numpy()) <= 2e-12
            out[restart] = rep
        s.restart_inner = False
        assert out[False].refinements >= 2
        assert out[False].iterations <= out[True].iterations + 1, (ce, out)
    s.close()
