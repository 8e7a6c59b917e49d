"""Resumed inner runs of the mixed-precision PCG (reliable updates).

After each FP64 residual the stopped FP32 run resumes with the
preconditioned residual of its last pass when its recursive residual is
close to the replaced one; otherwise the replaced residual is preconditioned
afresh.  A tile that covers the whole closed basin makes the preconditioner
exact: every run then ends after one iteration with a recursive residual at
FP32 rounding level, unrelated to the replaced one, and resuming on it would
diverge.  The check must catch that case, and on an ordinary grid the
resumed solve must reach the same solution as the one that never resumes.
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


def test_exact_preconditioner_does_not_resume_on_rounding_noise(torch_cuda):
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.basin(3, n=32)
    s = SevpSolver(p, tile_m=32, tile_h=32)
    b = torch.from_numpy(p.b).cuda()
    x, rep = s.solve(b, precision=1, tol=1e-12)
    assert rep.status == 0 and rep.rel_residual <= 1e-12, rep
    assert rep.iterations <= 8, rep
    xr = x.cpu().numpy()
    r = np.linalg.norm(p.b - P.apply_operator(p, xr)) / np.linalg.norm(p.b)
    assert r <= 2e-12
    s.close()


@pytest.mark.parametrize("tiles", [(16, 6), (16, 16)])
def test_resumed_and_restarted_continuations_agree(torch_cuda, tiles):
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(320, 160, seed=12)
    s = SevpSolver(p, tile_m=tiles[0], tile_h=tiles[1])
    b = torch.from_numpy(p.b).cuda()
    out = {}
    for dev in (0.0, 0.3):
        s.set_resume_check(dev)
        x, rep = s.solve(b, precision=1, tol=1e-12, inner_tol=1e-4)
        assert rep.status == 0 and rep.rel_residual <= 1e-12, (dev, rep)
        out[dev] = (x.cpu().numpy(), rep.iterations)
    (x0, i0), (x1, i1) = out[0.0], out[0.3]
    assert abs(i0 - i1) <= max(3, i0 // 10), (i0, i1)
    assert np.abs(x0 - x1).max() <= 1e-9 * np.abs(x0).max()
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_profiled_tile_passes_are_the_iterations(torch_cuda, precision):
    """Per-kernel profiling counts the pass-B launches that ran an iteration:
    the launches of a check interval after the run finished return at once
    and are left out, so the count equals the solve's iterations."""
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(320, 160, seed=12)
    s = SevpSolver(p, tile_m=16, tile_h=6)
    b = torch.from_numpy(p.b).cuda()
    s.profile(True)
    x, rep = s.solve(b, precision=precision, tol=1e-12, check_every=4)
    prof = s.profile_read()
    s.profile(False)
    assert rep.status == 0 and rep.rel_residual <= 1e-12
    assert prof["tile"][1] == rep.iterations, (prof, rep.iterations)
    assert prof["tile"][0] > 0.0
    s.close()
