"""The oracle of the barotropic correction loop (host only): masking zeroes
land faces only, a resting ocean has no right-hand side, and a zero or
constant correction field changes no velocity."""
import numpy as np

from musoc_solver_b200 import problems as P


def test_fs_oracle_sanity(oracle):
    st = P.fs_state(24, 12, 4, seed=2)
    u, v = st.u.copy(), st.v.copy()
    oracle.fs_mask(u, v, st.iu0, st.iv0)
    i0, j0, k0 = st.dims
    land = (st.iu0[1:-1, 1:-2] == 0)
    assert np.all(u[0, 1:-1, 1:-2][land] == 0)
    assert np.array_equal(u[0, 1:-1, 1:-2][~land], st.u[0, 1:-1, 1:-2][~land])
    assert np.array_equal(u[1:], st.u[1:])  # lower layers untouched
    s = oracle.fs_rhs(np.zeros_like(u), np.zeros_like(v), st.odx, st.ody, st.ocs, st.csv, st.odz)
    assert not s.any()
    p0, scr = st.p0.copy(), st.scr.copy()
    u2, v2 = u.copy(), v.copy()
    vm = oracle.fs_correct(np.full((j0 - 2, i0 - 2), 3.0), st.odt, st.odx, st.odyv, st.iu, st.iv,
                           st.iu0, st.iv0, p0, u2, v2, scr)
    # a constant X has no gradient: velocities unchanged, P0 = 3 ODT inside
    assert np.array_equal(u2, u) and np.array_equal(v2, v)
    assert np.allclose(p0[1:-1, 1:-1], np.float32(3.0 * st.odt))
    assert vm == 0.0  # land faces were zeroed and receive no correction
