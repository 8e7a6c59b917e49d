"""Influence data with the precision chosen per warp group of tiles
(sevp_set_influence_fp32) in the FP32 inner iterations of mixed solves.

The two ends of the choice are exact: with every group FP32 the solve is the
all-FP32 (precond_fp32) solve bit for bit, and with none it is the FP64
influence-data solve bit for bit.  In between, the solve still reaches the
FP64 tolerance and agrees with the CPU oracle.
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


def _solve(s, b, **kw):
    x, rep = s.solve(b, precision=1, tol=1e-12, **kw)
    assert rep.status == 0 and rep.rel_residual <= 1e-12, rep
    return x.cpu().numpy(), rep


@pytest.mark.parametrize("tm,th", [(16, 16), (16, 6)])
def test_all_fp32_groups_equal_fp32_influence(torch_cuda, tm, th):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=13)
    b = torch.from_numpy(p.b).cuda()
    s32 = SevpSolver(p, tile_m=tm, tile_h=th, precond_fp32=True)
    x32, r32 = _solve(s32, b)
    s = SevpSolver(p, tile_m=tm, tile_h=th)
    s.set_influence_fp32(1e300)
    f, g, nbytes = s.influence_fp32_groups()
    assert f == g > 0
    assert nbytes < s.influence_bytes()
    xm, rm = _solve(s, b)
    assert rm.iterations == r32.iterations
    assert np.array_equal(xm, x32)


@pytest.mark.parametrize("tm,th", [(16, 16), (16, 6)])
def test_no_fp32_groups_equal_fp64_influence(torch_cuda, tm, th):
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=14)
    b = torch.from_numpy(p.b).cuda()
    s64 = SevpSolver(p, tile_m=tm, tile_h=th)
    x64, r64 = _solve(s64, b)
    s = SevpSolver(p, tile_m=tm, tile_h=th)
    # a limit just above 1: no tile with row growth z > 1 qualifies
    s.set_influence_fp32(1.0 + 1e-9)
    f, g, nbytes = s.influence_fp32_groups()
    assert f == 0 and g > 0
    xm, rm = _solve(s, b)
    assert rm.iterations == r64.iterations
    assert np.array_equal(xm, x64)
    # switched off again: the FP64 influence data
    s.set_influence_fp32(0.0)
    assert s.influence_fp32_groups()[0] == 0
    xo, _ = _solve(s, b)
    assert np.array_equal(xo, x64)


def test_partial_fp32_groups_solve_matches_oracle(torch_cuda, oracle):
    """A growth limit that splits the groups: the mixed solve reaches 1e-12
    in about the iterations of the FP64-influence solve and agrees with the
    oracle's FP64 PCG; the choice survives a new operator."""
    torch = torch_cuda
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(360, 180, seed=15)
    b = torch.from_numpy(p.b).cuda()
    s64 = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    _, r64 = _solve(s64, b)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    s.set_influence_fp32(1e4)
    f, g, nbytes = s.influence_fp32_groups()
    assert 0 < f < g
    assert nbytes < s.influence_bytes()
    x, rep = _solve(s, b)
    assert rep.iterations <= r64.iterations + 2
    res = np.linalg.norm(p.b - P.apply_operator(p, x)) / np.linalg.norm(p.b)
    assert res <= 2e-12
    pc = oracle.TilePC(p, 16, 6, tile_nb=s.tile_nb)
    xo, _, _ = pc.pcg(p.b, tol=1e-12)
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()


def test_chebyshev_reads_the_chosen_precision(torch_cuda):
    """The one-launch Chebyshev iteration with every group FP32 equals its
    all-FP32 (precond_fp32) solve bit for bit, and with a splitting limit
    still reaches the tolerance."""
    torch = torch_cuda
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    p = P.global_grid(240, 120, seed=16)
    b = torch.from_numpy(p.b).cuda()
    out = {}
    for key, kw, lim in (("all32", dict(precond_fp32=True), None), ("mix_all", {}, 1e300),
                         ("mix_part", {}, 1e4)):
        s = SevpSolver(p, tile_m=16, tile_h=6, **kw)
        s.chebyshev_setup(b)
        s.set_method(N.METHOD_CHEB)
        if lim is not None:
            s.set_influence_fp32(lim)
        out[key] = _solve(s, b)
    assert out["mix_all"][1].iterations == out["all32"][1].iterations
    assert np.array_equal(out["mix_all"][0], out["all32"][0])
    x = out["mix_part"][0]
    res = np.linalg.norm(p.b - P.apply_operator(p, x)) / np.linalg.norm(p.b)
    assert res <= 2e-12
