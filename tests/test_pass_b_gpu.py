"""The FP32 PCG tile pass (pass B: x += alpha p, r -= alpha q, z = M^-1 r,
r.z, r.r) with tensor-copied shared-memory task stages, against the
register kernel.

The staged kernel runs the register kernel's arithmetic on the same values
and on the same grid, so its x, r and z, and its sums r.z and r.r, agree bit
for bit: whole mixed solves through the two kernels must then give the same
solution bit for bit, in the same iterations.  Cases cover full tasks (one
sub-block, matrices staged), tasks with several sub-blocks (matrices read
from global memory), a last tile narrower than the others, a last tile row
shorter than the others, 8- and 32-column tiles, and tilings the staged
kernel does not take (12-column tiles, nx not a multiple of 4), where the
register kernel runs.
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


# (name, problem, tile columns, tile rows, growth limit, staged kernel taken)
CASES = [
    ("global320x160", lambda: P.global_grid(320, 160, seed=6), 16, 6, 1e10, True),
    ("subblocks", lambda: P.global_grid(320, 160, seed=6), 16, 6, 1e3, True),
    ("ragged248x124", lambda: P.global_grid(248, 124, seed=8), 16, 6, 1e6, True),
    ("basin96", lambda: P.basin(1), 16, 6, 1e10, True),
    ("tiles8x6", lambda: P.global_grid(240, 120, seed=7), 8, 6, 1e10, True),
    ("tiles32x4", lambda: P.global_grid(256, 96, seed=5), 32, 4, 1e10, True),
    ("tiles12x6", lambda: P.global_grid(240, 120, seed=7), 12, 6, 1e10, False),
    ("nx_not_mult4", lambda: P.global_grid(102, 66, seed=9), 16, 6, 1e10, False),
]


@pytest.mark.parametrize("name,mk,tm,th,growth,staged", CASES)
def test_staged_pass_b_solves_bit_identical(torch_cuda, name, mk, tm, th, growth, staged):
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = mk()
    s = SevpSolver(p, tile_m=tm, tile_h=th, growth_limit=growth)
    b = torch.from_numpy(p.b).cuda()
    res = {}
    for kind in (N.PASS_B_REGISTERS, N.PASS_B_STAGED):
        s.set_pass_b_kernel(kind)
        x, rep = s.solve(b, precision=1, tol=1e-12)
        torch.cuda.synchronize()
        used = s.pass_b_kernel_used()
        if kind == N.PASS_B_STAGED:
            assert used == (N.PASS_B_STAGED if staged else N.PASS_B_REGISTERS), (name, used)
        else:
            assert used == N.PASS_B_REGISTERS, (name, used)
        assert rep.status == 0 and rep.rel_residual <= 1e-12, (name, kind, rep)
        res[kind] = (x.cpu().numpy(), rep.iterations, rep.rel_residual)
    (x1, i1, r1), (x2, i2, r2) = res[N.PASS_B_STAGED], res[N.PASS_B_REGISTERS]
    assert i1 == i2 and r1 == r2, (name, i1, i2, r1, r2)
    assert np.array_equal(x1, x2), (name, np.abs(x1 - x2).max())
    r = np.linalg.norm(p.b - P.apply_operator(p, x1)) / np.linalg.norm(p.b)
    assert r <= 2e-12, (name, r)
    s.close()


def test_staged_pass_b_without_graphs_and_from_a_guess(torch_cuda):
    """Direct launches (no CUDA-graph replay) and a warm start: the two
    kernels still agree bit for bit."""
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(320, 160, seed=11)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e10)
    s.graphs(False)
    b = torch.from_numpy(p.b).cuda()
    x0, _ = s.solve(b, precision=0, tol=1e-6)
    guess = (x0 * 0.97).contiguous()
    out = {}
    for kind in (N.PASS_B_REGISTERS, N.PASS_B_STAGED):
        s.set_pass_b_kernel(kind)
        x, rep = s.solve(b, guess.clone(), precision=1, tol=1e-12)
        assert rep.status == 0 and rep.rel_residual <= 1e-12, (kind, rep)
        out[kind] = (x.cpu().numpy(), rep.iterations)
    assert out[N.PASS_B_STAGED][1] == out[N.PASS_B_REGISTERS][1]
    assert np.array_equal(out[N.PASS_B_STAGED][0], out[N.PASS_B_REGISTERS][0])
    s.close()
