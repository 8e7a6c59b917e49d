"""CPU checks of the Schwarz preconditioner's oracle and shift rule."""
import numpy as np

from musoc_solver_b200 import problems as P
from musoc_solver_b200.solver import tile_sub_blocks


def _pc(oracle, p, tm, th, shift):
    return oracle.SchwarzPC(p, tm, th, shift, tile_sub_blocks(p, tm, th, 1e10),
                            tile_sub_blocks(oracle.rolled_grid(p, shift), tm, th, 1e10))


def test_rolled_grid_cuts_closed_seam(oracle):
    p = P.basin(1, n=40)
    g = oracle.rolled_grid(p, 5)
    assert np.all(g.al[:, 40 - 5] == 0) and np.all(g.ar[:, 40 - 5 - 1] == 0)
    assert np.array_equal(g.ac, np.roll(p.ac, -5, axis=1))
    q = P.global_grid(64, 32, seed=1)
    gq = oracle.rolled_grid(q, 5)
    assert np.array_equal(gq.al, np.roll(q.al, -5, axis=1))


def test_schwarz_oracle_symmetric_and_faster(oracle):
    for p in (P.global_grid(160, 80, seed=3), P.basin(2, n=64)):
        pc = _pc(oracle, p, 16, 6, 8)
        assert pc.status == 0
        rng = np.random.default_rng(0)
        u, v = rng.standard_normal((2, p.ny, p.nx))
        a, b = float((u * pc.apply(v)).sum()), float((v * pc.apply(u)).sum())
        assert abs(a - b) <= 1e-8 * abs(a)
        bj = oracle.TilePC(p, 16, 6, tile_nb=tile_sub_blocks(p, 16, 6, 1e10))
        _, itb, _ = bj.pcg(p.b, tol=1e-12)
        x, its, rel = pc.pcg(p.b, tol=1e-12)
        assert rel <= 1e-12 and its < itb
        res = np.linalg.norm(p.b - oracle.apply(p, x)) / np.linalg.norm(p.b)
        assert res <= 2e-12
