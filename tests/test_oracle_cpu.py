"""The CPU oracle pinned against the reference's own known answers and
independent solvers (no GPU needed).

The reference ships no golden vectors and no tests; its only check is the
harness in FS_SOLVER (M/fs_GLOBAL.f90:1806-2050): S = A*0 on the idealised
stencil (P/prep_GLOBAL.f90:246-261), an initial guess of 1 on
X(3:I2-1,3:J2-1), and a comparison after removing the arbitrary constant
(the value at (10,10)).  Those known answers are checked here, together with
scipy's sparse direct solve on the same assembled matrices.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from musoc_solver_b200 import problems as P


def _harness_guess(i2=180, j2=90):
    x0 = np.zeros((j2 + 2, i2 + 2))
    x = x0.copy()
    x[2:j2 - 1, 2:i2 - 1] = 1.0  # X(3:I2-1, 3:J2-1) = 1, 1-based
    return x0, x


def test_block_partition_matches_reference_rule(oracle):
    ie, ok = oracle.block_partition(90, 15)
    assert ok and list(ie) == [7 + 6 * k for k in range(14)] + [91]
    ie, ok = oracle.block_partition(96, 12)
    assert ok and ie[-1] == 97
    # J2=90, NB0=22: NN = ANINT(4.09) = 4, last block takes the remainder
    ie, ok = oracle.block_partition(90, 22)
    assert ie[-2] == 85 and ie[-1] == 91


@pytest.mark.parametrize("nb0", [45, 90])
def test_rep1_harness_constant(oracle, nb0):
    p = P.idealised()
    ie, _ = oracle.block_partition(90, nb0)
    rinv, rinv1, st = oracle.pre1(*p.coeffs(), ie)
    assert st == 0
    x0, x = _harness_guess()
    xr = oracle.rep1(*p.coeffs(), rinv, rinv1, np.zeros((90, 180), np.float32), x, ie)
    xr = xr - (xr[9, 9] - x0[9, 9])
    assert np.abs(xr[1:-1] - x0[1:-1]).max() < 1e-10


def test_bicgstab_harness_constant(oracle):
    p = P.idealised()
    x0, x = _harness_guess()
    xb, it, res = oracle.bicgstab(*p.coeffs(), np.zeros((90, 180), np.float32), x)
    xb = xb - (xb[9, 9] - x0[9, 9])
    assert res <= 1e-8 * 1.0001 and it < 1000
    assert np.abs(xb[1:-1] - x0[1:-1]).max() < 1e-6


def test_rep_basin_matches_scipy(oracle):
    p = P.basin(0)
    f = p.b.astype(np.float32)
    A = P.sparse_matrix(p).tocsc()
    xs = spla.spsolve(A, f.astype(np.float64).ravel()).reshape(p.ny, p.nx)
    for n0, tol in ((4, 1e-11), (6, 1e-9)):
        ie, _ = oracle.block_partition(96, 96 // n0)
        rinv, rinv1, st = oracle.pre(*p.coeffs(), ie)
        assert st == 0
        xr = oracle.rep(*p.coeffs(), rinv, rinv1, f, np.zeros((98, 98)), ie)[1:-1, 1:-1]
        assert np.abs(xr - xs).max() <= tol * np.abs(xs).max()


def test_rep1_periodic_matches_scipy(oracle):
    p = P.idealised(60, 30)
    p.ac[:] += np.float32(0.05)
    ie, _ = oracle.block_partition(30, 10)
    rinv, rinv1, st = oracle.pre1(*p.coeffs(), ie)
    rng = np.random.default_rng(2)
    f = rng.standard_normal((30, 60)).astype(np.float32)
    xr = oracle.rep1(*p.coeffs(), rinv, rinv1, f, np.zeros((32, 62)), ie)
    xs = spla.spsolve(P.sparse_matrix(p).tocsc(), f.astype(np.float64).ravel()).reshape(30, 60)
    assert np.abs(xr[1:-1, 1:-1] - xs).max() <= 1e-11 * np.abs(xs).max()
    # ghost columns are the periodic copies
    assert np.array_equal(xr[1:-1, 0], xr[1:-1, -2]) and np.array_equal(xr[1:-1, -1], xr[1:-1, 1])


def test_matinv_matches_numpy(oracle):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((40, 40)) + 40 * np.eye(40)
    for pivot in (False, True):
        b, st = oracle.matinv(a, pivot=pivot)
        assert st == 0
        assert np.abs(b - np.linalg.inv(a)).max() < 1e-13
    b, st = oracle.matinv(np.array([[0.0, 1.0], [1.0, 0.0]]))
    assert st == 1  # the reference divides by the zero pivot
    b, st = oracle.matinv(np.array([[0.0, 1.0], [1.0, 0.0]]), pivot=True)
    assert st == 0 and np.allclose(b, [[0, 1], [1, 0]])


def test_ratqr_figi_match_numpy(oracle):
    rng = np.random.default_rng(7)
    n = 10
    d = 4.0 + rng.random(n)
    e = rng.random(n)
    t = np.zeros((3, n))  # column-major T(n,3) == C (3, n)
    t[0, 1:] = e[1:]
    t[1, :] = d
    t[2, :-1] = e[1:]
    L = oracle.lib()
    dd, ee, e2 = np.zeros(n), np.zeros(n), np.zeros(n)
    assert L.or_figi(n, np.ascontiguousarray(t), dd, ee, e2) == 0
    import ctypes as C
    mn = C.c_double()
    assert L.or_ratqr(n, 1e-10, dd, ee, C.byref(mn)) == 0
    T = np.diag(d) + np.diag(e[1:], 1) + np.diag(e[1:], -1)
    assert abs(mn.value - np.linalg.eigvalsh(T).min()) < 1e-8


def _spd_basin():
    """The basin operator negated: symmetric positive definite, non-uniform
    (the reference's start vector of ones is not an eigenvector)."""
    p = P.basin(0, n=32)
    for name in ("al", "ab", "ac", "ar", "at"):
        setattr(p, name, -getattr(p, name))
    return p


def test_lanczos_bounds_bracket_spectrum(oracle):
    p = _spd_basin()
    mn, mx, ierr, alpha, sigma = oracle.lanczos(*p.coeffs())
    ev = np.linalg.eigvalsh(P.sparse_matrix(p).toarray())
    assert ierr == 0
    assert mx >= ev.max() * 0.95
    assert 0.0 <= mn <= ev.max()


def test_lanczos_breakdown_terminates(oracle):
    """On the shifted idealised stencil the start vector of ones is an exact
    eigenvector: the two-sided Lanczos recurrence breaks down and the
    reference's RATQR loop would not terminate; the restatement returns."""
    p = P.idealised(40, 20)
    p.ac[:] += np.float32(0.1)
    mn, mx, ierr, alpha, sigma = oracle.lanczos(*p.coeffs())
    assert abs(alpha[0] - 0.1) < 1e-6


def test_csi_converges_with_bracketing_bounds(oracle):
    p = P.idealised(60, 30)
    p.ac[:] += np.float32(0.05)
    rng = np.random.default_rng(3)
    b = rng.standard_normal((30, 60)).astype(np.float32)
    x, it, res = oracle.csi(*p.coeffs(), 0.05, 2.05, b, np.zeros((32, 62)))
    assert res <= 1e-7 and it < 1000
    xs = spla.spsolve(P.sparse_matrix(p).tocsc(), b.astype(np.float64).ravel()).reshape(30, 60)
    assert np.abs(x[1:-1, 1:-1] - xs).max() <= 1e-6 * np.abs(xs).max()


def _bir_case(oracle):
    p = P.idealised(48, 30)
    p.ac[:] += np.float32(0.05)
    c = [np.ascontiguousarray(a, np.float32) for a in p.coeffs()]
    i2, j2, nbir = 48, 30, 4
    ibir = 2 * i2 // nbir
    ie, _ = oracle.block_partition(j2, 6)
    nb0 = len(ie)
    L = oracle.lib()
    ro = np.zeros((nbir, nb0, ibir * ibir))
    r1o = np.zeros((nbir, nb0 - 1, ibir * ibir))
    ws = [np.zeros((j2, ibir), np.float32) for _ in range(5)]
    assert L.or_pre_strips(*c, ro.reshape(-1), r1o.reshape(-1), np.zeros((j2 + 2, ibir + 2)), ie,
                           i2, j2, nb0, nbir, *ws) == 0
    rng = np.random.default_rng(4)
    s = rng.standard_normal((j2, i2)).astype(np.float32)
    xs = spla.spsolve(P.sparse_matrix(p).tocsc(), s.astype(np.float64).ravel()).reshape(j2, i2)

    def sweeps(n, fix):
        x = np.zeros((j2 + 2, i2 + 2))
        xx = np.zeros((j2 + 2, ibir + 2))
        errs = []
        for _ in range(n):
            wsrc = [np.zeros((j2, ibir), np.float32) for _ in range(6)]
            L.or_bir_sweeps(*c, s, ro.reshape(-1), r1o.reshape(-1), x, xx,
                            np.zeros((j2 + 2, ibir + 2)), *wsrc, np.zeros((nb0 - 1, ibir)),
                            np.zeros(ibir), np.zeros(ibir), ie, i2, j2, nb0, nbir, 1, 1, fix)
            errs.append(np.abs(x[1:-1, 1:-1] - xs).max())
        return errs

    return sweeps


def test_bir_sweeps_reference_wrap_rows(oracle):
    """The reference refreshes the wrapped strip's side boundaries for rows
    1..J2 only (M/fs_GLOBAL.f90:1925-1926): its top interior row keeps a
    zero boundary and the Schwarz sweeps stall at an O(1) error.  With the
    rows refreshed (opt-in fix_wrap) the sweeps converge."""
    sweeps = _bir_case(oracle)
    ref = sweeps(5, 0)
    assert ref[-1] > 0.5 and abs(ref[-1] - ref[-2]) < 1e-3
    fixed = sweeps(6, 1)
    assert fixed[1] < 1e-2 * fixed[0] and fixed[-1] < 1e-10


def test_assemble_idealised_override(oracle):
    i2, j2, k1 = 12, 8, 3
    odx = np.ones(j2 + 2, np.float32) * 1e-5
    ody = np.ones(j2 + 2, np.float32) * 1e-5
    csv = np.ones(j2 + 2, np.float32)
    ocs = np.ones(j2 + 2, np.float32)
    odyv = np.ones(j2 + 2, np.float32) * 1e-5
    odz = np.ones(k1, np.float32) * 1e-3
    iu = np.ones((k1 + 1, j2 + 2, i2 + 2), np.int32)
    iv = np.ones((k1 + 1, j2 + 2, i2 + 2), np.int32)
    al, ab, ac, ar, at = oracle.assemble(i2, j2, k1, odx, ody, csv, ocs, odyv, odz, iu, iv, 6, 0.0, 1)
    assert (al == -0.25).all() and (ar == -0.25).all()
    assert (ab[0] == 0).all() and (at[-1] == 0).all() and (ac[0] == 0.75).all()
    # rows sum to zero: constants are in the null space
    assert np.allclose(al + ab + ac + ar + at, 0.0)
    al, ab, ac, ar, at = oracle.assemble(i2, j2, k1, odx, ody, csv, ocs, odyv, odz, iu, iv, 1, 0.5, 0)
    assert (al[:, 0] == 0).all() and (ar[:, -1] == 0).all() and (ab[0, :][np.arange(i2) != i2 // 2 - 1] == 0).all()
    assert np.allclose(ac, -(al + ar + ab + at) - 0.5)


@pytest.mark.parametrize("tm,th", [(24, 24), (16, 16), (12, 9)])
def test_tile_pcg_matches_scipy(oracle, tm, th):
    from musoc_solver_b200.solver import default_sub_rows

    for p in (P.basin(0), P.global_grid(100, 70, seed=3)):
        pc = oracle.TilePC(p, tm, th, default_sub_rows(p, th, 1e6))
        assert pc.status == 0
        x, it, rel = pc.pcg(p.b, tol=1e-12)
        assert rel <= 1e-12
        xs = spla.spsolve(P.sparse_matrix(p).tocsc(), p.b.ravel()).reshape(p.ny, p.nx)
        assert np.abs(x - xs).max() <= 1e-9 * np.abs(xs).max()


def test_tile_preconditioner_is_exact_tile_inverse(oracle):
    """Each tile block of M^-1 is the inverse of the tile's block of A."""
    from musoc_solver_b200.solver import default_sub_rows

    p = P.global_grid(40, 24, seed=8)
    tm, th = 10, 8
    pc = oracle.TilePC(p, tm, th, default_sub_rows(p, th, 1e6))
    A = P.sparse_matrix(p).toarray()
    rng = np.random.default_rng(0)
    r = rng.standard_normal((p.ny, p.nx))
    z = pc.apply(r)
    for b in range(3):
        for a in range(4):
            idx = np.arange(p.nx * p.ny).reshape(p.ny, p.nx)[b * th:(b + 1) * th, a * tm:(a + 1) * tm].ravel()
            zt = np.linalg.solve(A[np.ix_(idx, idx)], r.ravel()[idx])
            assert np.abs(z.ravel()[idx] - zt).max() <= 1e-9 * np.abs(zt).max()


def _lanczos_bounds(p, pc, tol=1e-12):
    """Extreme Ritz values of M^-1 A from the CG-Lanczos tridiagonal of a
    numpy PCG run with the oracle preconditioner."""
    A = P.sparse_matrix(p)
    b = p.b.ravel()
    x = np.zeros_like(b)
    r = b.copy()
    z = pc.apply(r.reshape(p.ny, p.nx)).ravel()
    pv = z.copy()
    rz = r @ z
    al, be = [], []
    for _ in range(500):
        q = A @ pv
        a = rz / (pv @ q)
        x += a * pv
        r -= a * q
        al.append(a)
        if np.linalg.norm(r) <= tol * np.linalg.norm(b):
            break
        z = pc.apply(r.reshape(p.ny, p.nx)).ravel()
        rz2 = r @ z
        be.append(rz2 / rz)
        rz = rz2
        pv = z + be[-1] * pv
    k = len(al)
    d = np.array([1 / al[j] + (be[j - 1] / al[j - 1] if j else 0.0) for j in range(k)])
    e = np.array([np.sqrt(be[j]) / al[j] for j in range(k - 1)])
    ev = np.linalg.eigvalsh(np.diag(d) + np.diag(e, 1) + np.diag(e, -1))
    return ev[0], ev[-1]


@pytest.mark.parametrize("grid", ["global", "basin"])
def test_tile_chebyshev_matches_scipy(oracle, grid):
    """The oracle's preconditioned Chebyshev iteration (or_cheb) with bounds
    from CG-Lanczos converges to the scipy direct solution."""
    from musoc_solver_b200.solver import tile_sub_blocks

    p = P.global_grid(160, 80, seed=3) if grid == "global" else P.basin(1)
    pc = oracle.TilePC(p, 16, 6, tile_nb=tile_sub_blocks(p, 16, 6, 1e10))
    lo, hi = _lanczos_bounds(p, pc)
    assert 0 < lo < hi
    x, it, rel = pc.cheb(p.b, lo * 0.98, hi * 1.02, tol=1e-12)
    assert rel <= 1e-12, (it, rel)
    xd = spla.spsolve(P.sparse_matrix(p).tocsc(), p.b.ravel()).reshape(p.b.shape)
    assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()
    # Chebyshev with exact bounds takes no more than about the CG bound
    _, it_cg, _ = pc.pcg(p.b, tol=1e-12)
    assert it <= 3 * it_cg + 10, (it, it_cg)


def test_repbir_period_equals_rep1_full_width(oracle):
    """REPBIR_PERIOD (M/sevp.f90:109-217) at full width (M0 = I0, M2 = I2)
    marches the same equations with the same periodic ghost refresh as REP1
    (M/sevp.f90:11-107): equal results bit for bit."""
    p = P.idealised(120, 60)
    p.ac[:] += np.float32(0.01)
    c = p.coeffs()
    ie, ok = oracle.block_partition(60, 10)
    rinv, rinv1, st = oracle.pre1(*c, ie)
    assert st == 0
    rng = np.random.default_rng(4)
    f = rng.standard_normal((60, 120)).astype(np.float32)
    x = np.zeros((62, 122))
    x[0] = rng.standard_normal(122)
    x1 = oracle.rep1(*c, rinv, rinv1, f, x, ie)
    xp, st = oracle.repbir_period(*c, rinv, rinv1, f, x, ie)
    assert st == 0
    assert np.array_equal(x1, xp)


def test_repbir_strip_satisfies_its_equations(oracle):
    """REPBIR (M/sevp.f90:218-328) on a strip of M2 columns with Dirichlet
    side columns: the solution satisfies the strip's equations."""
    p = P.idealised(120, 60)
    p.ac[:] += np.float32(0.01)
    c = p.coeffs()
    m2 = 40
    ie, ok = oracle.block_partition(60, 10)
    rinv, rinv1, st = oracle.pre(*c, ie, m2=m2)
    assert st == 0
    rng = np.random.default_rng(5)
    f = rng.standard_normal((60, m2)).astype(np.float32)
    x = np.zeros((62, m2 + 2))
    x[:, 0] = rng.standard_normal(62)
    x[:, -1] = rng.standard_normal(62)
    xs, _ = oracle.repbir(*c, rinv, rinv1, f, x, ie, m2)
    al, ab, ac, ar, at = (a[:, :m2].astype(np.float64) for a in c)
    lhs = (ab * xs[:-2, 1:-1] + al * xs[1:-1, :-2] + ac * xs[1:-1, 1:-1] + ar * xs[1:-1, 2:]
           + at * xs[2:, 1:-1])
    assert np.abs(lhs - f).max() <= 1e-8 * np.abs(f).max()
