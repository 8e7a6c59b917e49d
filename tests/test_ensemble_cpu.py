"""Stacking ensemble members: the stacked operator is block-diagonal and
open member edges are rejected (host logic, no GPU)."""
import numpy as np
import pytest

from musoc_solver_b200 import problems as P
from musoc_solver_b200.ensemble import member_tile_height


def test_stack_is_block_diagonal():
    ms = P.ensemble(members=3, nx=48, ny=24, seed=3)
    s = P.stack(ms)
    assert (s.ny, s.nx) == (72, 48) and s.meta["members"] == 3
    x = np.random.default_rng(0).standard_normal((s.ny, s.nx))
    y = P.apply_operator(s, x)
    for k, m in enumerate(ms):
        rows = slice(24 * k, 24 * (k + 1))
        assert np.array_equal(y[rows], P.apply_operator(m, x[rows]))
    assert np.array_equal(s.b[24:48], ms[1].b)


def test_members_differ_and_stack_rejects_open_edges():
    ms = P.ensemble(members=2, nx=48, ny=24, seed=3)
    assert not np.array_equal(ms[0].ac, ms[1].ac)  # perturbed depths
    bad = P.idealised(48, 24)
    bad.at[-1] = -0.25  # an open north edge would couple two members
    with pytest.raises(ValueError):
        P.stack([bad, bad])


def test_member_tile_height_divides_rows():
    for ny in (24, 48, 360, 180, 90):
        h = member_tile_height(ny)
        assert ny % h == 0 and 6 <= h <= 24
    assert member_tile_height(360) == 6
    assert member_tile_height(45) == 15
