"""The PCG stencil pass (pass A: p = z + beta p_old, q = A p, p.q) on
tensor-copied shared-memory tiles, against the column-walking kernel and
numpy.

Both kernels form p and q with the same operations in the same order, so
p and q must agree bit for bit; p.q is summed in a different order (per tile
instead of per column strip), so it agrees to 1e-12 relative.  Against numpy
(float64 on the FP32 values): p to 1 ulp of FP32 (the fused multiply-add),
q to 1e-5 of max|q| in FP32 and 1e-13 in FP64.  Cases cover the periodic
seam (the wrapped halo column of the first and last tile), closed basins,
grids that do not fill the last tile in x or y, a nonsymmetric operator
(five coefficient planes read), the first iteration (beta = 0, p = z) and a
grid the tensor copies cannot take (nx not a multiple of 4: the column
kernel runs instead).
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


def _nonsymmetric(p, seed=5):
    rng = np.random.default_rng(seed)
    q = P.Problem(*(a.copy() for a in (p.al, p.ab, p.ac, p.ar, p.at, p.b)), periodic=p.periodic,
                  name=p.name + "_nonsym")
    q.al *= (1.0 + 0.2 * rng.random(q.al.shape)).astype(np.float32)
    q.ab *= (1.0 + 0.2 * rng.random(q.ab.shape)).astype(np.float32)
    return q


CASES = [
    ("global240x120", lambda: P.global_grid(240, 120, seed=7)),
    ("global_ragged", lambda: P.global_grid(100, 70, seed=3)),
    ("global_one_tile", lambda: P.global_grid(48, 40, seed=2)),
    ("basin96", lambda: P.basin(1)),
    ("nonsym", lambda: _nonsymmetric(P.global_grid(200, 90, seed=4))),
    ("nx_not_mult4", lambda: P.global_grid(102, 66, seed=9)),
]


@pytest.mark.parametrize("name,mk", CASES)
@pytest.mark.parametrize("fp64", [False, True])
def test_pass_a_tiles_match_columns_and_numpy(torch_cuda, name, mk, fp64):
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = mk()
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    rng = np.random.default_rng(11)
    dt = np.float64 if fp64 else np.float32
    z = rng.standard_normal((p.ny, p.nx)).astype(dt)
    pold = rng.standard_normal((p.ny, p.nx)).astype(dt)
    dz, dp = torch.from_numpy(z).cuda(), torch.from_numpy(pold).cuda()
    for beta in (0.0, 0.37):
        out = {}
        for kind in (N.PASS_A_TILES, N.PASS_A_COLUMNS):
            s.set_pass_a_kernel(kind)
            pn, q, pq = s.pass_a(dz, dp, beta)
            torch.cuda.synchronize()
            out[kind] = (pn.cpu().numpy(), q.cpu().numpy(), pq)
        (p1, q1, pq1), (p2, q2, pq2) = out[N.PASS_A_TILES], out[N.PASS_A_COLUMNS]
        assert np.array_equal(p1, p2) and np.array_equal(q1, q2), (name, beta)
        assert abs(pq1 - pq2) <= 1e-12 * abs(pq2), (name, beta, pq1, pq2)
        pref = z.astype(np.float64) + beta * pold.astype(np.float64)
        mag = np.abs(z.astype(np.float64)) + abs(beta) * np.abs(pold.astype(np.float64))
        ulp = mag * (2.0 ** -23 if not fp64 else 2.0 ** -51) + 1e-300
        assert np.all(np.abs(p1 - pref) <= ulp), (name, beta)
        qref = P.apply_operator(p, p1.astype(np.float64))
        tol = (1e-13 if fp64 else 1e-5) * np.abs(qref).max()
        assert np.abs(q1 - qref).max() <= tol, (name, beta)
        pqref = float((p1.astype(np.float64) * q1.astype(np.float64)).sum())
        assert abs(pq1 - pqref) <= 1e-12 * abs(pqref)
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_with_either_pass_a_kernel(torch_cuda, precision):
    """Solves through both kernels reach the same FP64 residual bar and the
    same solution (p.q differs in its last bits, so the iteration counts may
    differ by a few)."""
    from musoc_solver_b200 import native as N
    from musoc_solver_b200.solver import SevpSolver

    torch = torch_cuda
    p = P.global_grid(320, 160, seed=6)
    s = SevpSolver(p, tile_m=16, tile_h=6, growth_limit=1e6)
    b = torch.from_numpy(p.b).cuda()
    res = {}
    for kind in (N.PASS_A_TILES, N.PASS_A_COLUMNS):
        s.set_pass_a_kernel(kind)
        x, rep = s.solve(b, precision=precision, tol=1e-12)
        assert rep.status == 0 and rep.rel_residual <= 1e-12, (kind, rep)
        xr = x.cpu().numpy()
        r = np.linalg.norm(p.b - P.apply_operator(p, xr)) / np.linalg.norm(p.b)
        assert r <= 2e-12
        res[kind] = (xr, rep.iterations)
    (x1, i1), (x2, i2) = res[N.PASS_A_TILES], res[N.PASS_A_COLUMNS]
    assert abs(i1 - i2) <= max(2, i2 // 20), (i1, i2)
    assert np.abs(x1 - x2).max() <= 1e-9 * np.abs(x2).max()
    s.close()
