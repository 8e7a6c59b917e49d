"""p_sevp_pcg_: the tile-SEVP preconditioned CG behind p_bicgstab_le's
argument list (M/sevp.f90:443), called through the C ABI with the
reference's layouts: PREP's nonsymmetric REAL*4 planes as assembled by
P/prep_GLOBAL.f90:170-244 (the oracle's restatement, or_assemble), a REAL*4
right-hand side and the padded REAL*8 X in and out.

Checks against the oracle:
* the relative residual ||S - A X|| / ||S|| <= 1e-12, recomputed on the host
  with the oracle's p_sqprod (M/sevp.f90:696-713) on the returned padded X;
* the solution within 1e-9 (max norm, relative) of scipy's sparse direct
  solve of the same system, boundary data included;
* the reference harness's known answer (M/fs_GLOBAL.f90:1835-1858): with
  S = A 0 on the singular idealised stencil and a guess of 1 on
  X(3:I2-1, 3:J2-1), the absolute rule ends at a constant field;
* an operator that no row scaling symmetrises is refused (status 8) and X
  is left untouched.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from musoc_solver_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build, native

    build.build()
    lib = native.lib()
    yield lib
    lib.sevp_fs_release()
    lib.sevp_set_periodic_we(1)


def _opts(L, **kw):
    from musoc_solver_b200 import native as N

    o = N.FsOptions()
    L.sevp_fs_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    assert L.sevp_fs_set_options(C.byref(o)) == 0
    return o


def _call(L, planes, b, x, cplanes=None):
    """p_sevp_pcg_ with host arrays; returns (status, report)."""
    from musoc_solver_b200 import native as N

    f32 = [np.ascontiguousarray(a, np.float32) for a in planes]
    cp = f32 if cplanes is None else [np.ascontiguousarray(a, np.float32) for a in cplanes]
    b32 = np.ascontiguousarray(b, np.float32)
    j2, i2 = b32.shape
    args = [a.ctypes.data_as(C.c_void_p) for a in f32] + [b32.ctypes.data_as(C.c_void_p),
                                                         x.ctypes.data_as(C.c_void_p)]
    args += [a.ctypes.data_as(C.c_void_p) for a in cp]
    args += [C.byref(C.c_int(i2)), C.byref(C.c_int(j2))]
    L.p_sevp_pcg_(*args)
    rep = N.Report()
    L.sevp_fs_last_report(C.byref(rep))
    return L.sevp_last_status(), rep


def _residual(oracle, planes, b, x, periodic):
    """||S - A X|| / ||S|| with the oracle's p_sqprod on the padded X (its
    periodic ghost columns as returned)."""
    xp = x.copy()
    if periodic:
        xp[1:-1, 0] = xp[1:-1, -2]
        xp[1:-1, -1] = xp[1:-1, 1]
    r = b - oracle.sqprod(*planes, xp)[1:-1, 1:-1]
    return np.linalg.norm(r) / np.linalg.norm(b)


def _direct(p, b, xpad):
    """scipy solve of the interior system with X's ghost values as boundary data."""
    al, ab, ac, ar, at = (a.astype(np.float64) for a in p.coeffs())
    rhs = b.copy()
    rhs[0, :] -= ab[0, :] * xpad[0, 1:-1]
    rhs[-1, :] -= at[-1, :] * xpad[-1, 1:-1]
    if not p.periodic:
        rhs[:, 0] -= al[:, 0] * xpad[1:-1, 0]
        rhs[:, -1] -= ar[:, -1] * xpad[1:-1, -1]
    return spla.spsolve(P.sparse_matrix(p).tocsc(), rhs.ravel()).reshape(b.shape)


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("precision", [0, 1])
def test_prep_coefficients_solve_to_1e12(L, oracle, periodic, precision):
    p = P.prep_grid(120, 60, k1=5, seed=4, periodic=periodic)
    m = p.meta
    planes = oracle.assemble(p.nx, p.ny, m["k1"], m["odx"], m["ody"], m["csv"], m["ocs"],
                             m["odyv"], m["odz"], m["iu"], m["iv"], m["nbir"], float(m["gamma"]), 0)
    assert all(np.array_equal(a, b) for a, b in zip(planes, p.coeffs()))
    al, ab, ac, ar, at = planes
    assert not np.array_equal(at[:-1], ab[1:])  # PREP's operator is not symmetric
    L.sevp_set_periodic_we(int(periodic))
    _opts(L, precision=precision)
    rng = np.random.default_rng(7)
    x = np.zeros((p.ny + 2, p.nx + 2))
    # Dirichlet data in the ghost rows (and columns when closed)
    x[0, 1:-1] = rng.standard_normal(p.nx)
    x[-1, 1:-1] = rng.standard_normal(p.nx)
    if not periodic:
        x[1:-1, 0] = rng.standard_normal(p.ny)
        x[1:-1, -1] = rng.standard_normal(p.ny)
    x0 = x.copy()
    st, rep = _call(L, planes, p.b, x)
    assert st == 0, (st, L.sevp_last_error())
    assert rep.rel_residual <= 1e-12
    assert _residual(oracle, planes, p.b, x, periodic) <= 2e-12
    xd = _direct(p, p.b, x0)
    err = np.abs(x[1:-1, 1:-1] - xd).max() / np.abs(xd).max()
    assert err <= 1e-9, err
    # ghost rows keep the caller's boundary data; periodic ghost columns refreshed
    assert np.array_equal(x[0], x0[0]) and np.array_equal(x[-1], x0[-1])
    if periodic:
        assert np.array_equal(x[1:-1, 0], x[1:-1, -2]) and np.array_equal(x[1:-1, -1], x[1:-1, 1])
    else:
        assert np.array_equal(x[1:-1, 0], x0[1:-1, 0])


def test_cached_operator_follows_changed_coefficients(L, oracle):
    """A second call with the same arrays reuses the device operator; after
    the caller changes AC in place, the hash check rebuilds it."""
    p = P.prep_grid(96, 48, k1=4, seed=9, periodic=True)
    planes = [np.ascontiguousarray(a) for a in p.coeffs()]
    L.sevp_set_periodic_we(1)
    _opts(L, precision=1)
    for scale in (1.0, 1.0, 1.5):
        planes[2][:] = p.ac * np.float32(scale)
        x = np.zeros((p.ny + 2, p.nx + 2))
        st, rep = _call(L, planes, p.b, x)
        assert st == 0
        assert _residual(oracle, planes, p.b, x, True) <= 2e-12, scale


def test_reference_absolute_rule_harness_known_answer(L):
    """FS_SOLVER's test (M/fs_GLOBAL.f90:1835-1858) with the reference's
    absolute rule: S = A 0 = 0 on the idealised stencil (singular: constants
    in the null space), guess 1 on X(3:I2-1, 3:J2-1); after removing the
    value at (10, 10) the solution is zero."""
    p = P.idealised(180, 90)
    L.sevp_set_periodic_we(1)
    for precision in (0, 1):
        _opts(L, precision=precision, tol_abs=1, tol=1e-10)
        x = np.zeros((92, 182))
        x[2:89, 2:179] = 1.0
        st, rep = _call(L, p.coeffs(), p.b, x)
        assert st == 0, (precision, st)
        assert rep.abs_residual <= 1e-10
        xs = x[1:-1, :] - x[9, 9]
        assert np.abs(xs).max() <= 1e-7, (precision, np.abs(xs).max())


def test_operator_without_symmetrising_scaling_is_refused(L):
    p = P.prep_grid(64, 32, k1=3, seed=2, periodic=True)
    planes = [np.array(a) for a in p.coeffs()]
    planes[4][10, 7] *= np.float32(1.5)  # AT(8, 11) alone: the row ratio varies
    _opts(L)
    x = np.full((p.ny + 2, p.nx + 2), 3.0)
    st, _ = _call(L, planes, p.b, x)
    assert st == 8  # SEVP_NONSYMMETRIC
    assert "I=8, J=11" in L.sevp_last_error().decode()
    assert (x == 3.0).all()
