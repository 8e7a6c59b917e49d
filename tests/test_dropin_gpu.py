"""Parity of the Fortran-compatible drop-ins (C ABI, host arrays) with the
CPU oracle's restatement of the reference routines.

The marching routines (REP1, REP, REPBIR, PRE1, PRE, MATINV, the BIR strip
sweeps) and the operator applies use explicitly rounded FP64 steps in the
reference's order on the GPU, so they must match the oracle BIT FOR BIT.
The Krylov drop-ins (BiCGSTAB, CSI, Lanczos) sum their dot products in a
parallel tree, so they match within tolerances stated per test.
"""
import ctypes as C

import numpy as np
import pytest

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
    lib.sevp_set_periodic_we(1)
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _i(v):
    return C.byref(C.c_int(int(v)))


def _coeffs(p):
    return [np.ascontiguousarray(a, np.float32) for a in p.coeffs()]


def _shifted_idealised(i2=180, j2=90, shift=0.01):
    p = P.idealised(i2, j2)
    p.ac[:] += np.float32(shift)
    return p


def test_pre1_rep1_bit_exact(L, oracle):
    p = _shifted_idealised()
    c = _coeffs(p)
    j2, i2 = p.ac.shape
    ie, ok = oracle.block_partition(j2, 15)
    assert ok
    nb = len(ie)
    rinv = np.zeros((nb, i2, i2))
    rinv1 = np.zeros((nb - 1, i2, i2))
    h = np.zeros((j2 + 2, i2 + 2))
    L.pre1_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(h), _p(ie), _i(i2 + 2), _i(i2), _i(nb))
    assert L.sevp_last_status() == 0
    r_o, r1_o, st = oracle.pre1(*c, ie)
    assert st == 0
    assert np.array_equal(rinv, r_o)
    assert np.array_equal(rinv1, r1_o[: nb - 1])
    # REP1 with those matrices, random F and boundary data
    rng = np.random.default_rng(0)
    f = rng.standard_normal((j2, i2)).astype(np.float32)
    x = np.zeros((j2 + 2, i2 + 2))
    x[0] = rng.standard_normal(i2 + 2)
    d0 = np.zeros((nb - 1, i2))
    d1 = np.zeros(i2)
    d2 = np.zeros(i2)
    hh = np.zeros((j2 + 2, i2 + 2))
    xg = x.copy()
    L.rep1_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(d0), _p(d1), _p(d2), _p(f), _p(hh), _p(xg),
            _p(ie), _i(i2 + 2), _i(i2), _i(nb))
    assert L.sevp_last_status() == 0
    xo = oracle.rep1(*c, r_o, r1_o, f, x, ie)
    assert np.array_equal(xg, xo)
    res = f - P.apply_operator(p, xg[1:-1, 1:-1])
    assert np.linalg.norm(res) <= 1e-8 * np.linalg.norm(f)


def test_pre1_evp_file_rep1(L, oracle, tmp_path):
    """PREP -> MAIN through the EVP file: influence data computed by the GPU
    pre1_ is written in PREP's record, read back as MAIN reads it, and the
    GPU rep1_ on the read matrices equals the oracle's REP1 bit for bit."""
    from musoc_solver_b200 import evp

    p = _shifted_idealised(120, 60)
    c = _coeffs(p)
    j2, i2 = p.ac.shape
    ie, ok = oracle.block_partition(j2, 6)
    assert ok
    nb = len(ie)
    rinv = np.zeros((nb, i2, i2))
    rinv1 = np.zeros((nb - 1, i2, i2))
    h = np.zeros((j2 + 2, i2 + 2))
    L.pre1_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(h), _p(ie), _i(i2 + 2), _i(i2), _i(nb))
    assert L.sevp_last_status() == 0
    al, ab, ac, ar, at = c
    evp.write(tmp_path / "EVP", al, ar, ab, at, ac, rinv, rinv1, ie)
    r = evp.read(tmp_path / "EVP", i2, j2, rinv.shape, rinv1.shape, nb)
    assert r["oac"] is None
    rng = np.random.default_rng(3)
    f = rng.standard_normal((j2, i2)).astype(np.float32)
    x = np.zeros((j2 + 2, i2 + 2))
    x[0] = rng.standard_normal(i2 + 2)
    d0, d1, d2 = np.zeros((nb - 1, i2)), np.zeros(i2), np.zeros(i2)
    hh = np.zeros((j2 + 2, i2 + 2))
    xg = x.copy()
    c2 = [np.ascontiguousarray(r[k]) for k in ("al", "ab", "ac", "ar", "at")]
    L.rep1_(*[_p(a) for a in c2], _p(r["rinv"]), _p(r["rinv1"]), _p(d0), _p(d1), _p(d2), _p(f),
            _p(hh), _p(xg), _p(r["ie"]), _i(i2 + 2), _i(i2), _i(nb))
    assert L.sevp_last_status() == 0
    r_o, r1_o, st = oracle.pre1(*c, ie)
    xo = oracle.rep1(*c, r_o, r1_o, f, x, ie)
    assert np.array_equal(xg, xo)


def test_rep1_known_answer_constant(L, oracle):
    """FS_SOLVER's harness (M/fs_GLOBAL.f90:1814-1858): S = A*0 on the
    singular idealised stencil; SEVP returns a constant, i.e. x0 after the
    shift by the value at (10,10).  Holds with 2-row blocks (the near
    singular last block amplifies rounding with taller blocks)."""
    p = P.idealised(180, 90)
    c = _coeffs(p)
    ie, _ = oracle.block_partition(90, 45)
    nb = len(ie)
    rinv = np.zeros((nb, 180, 180))
    rinv1 = np.zeros((nb - 1, 180, 180))
    h = np.zeros((92, 182))
    L.pre1_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(h), _p(ie), _i(182), _i(180), _i(nb))
    x0 = np.zeros((92, 182))
    x = x0.copy()
    x[2:89, 2:179] = 1.0
    s = np.zeros((90, 180), np.float32)
    d0, d1, d2, hh = np.zeros((nb - 1, 180)), np.zeros(180), np.zeros(180), np.zeros((92, 182))
    L.rep1_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(d0), _p(d1), _p(d2), _p(s), _p(hh), _p(x),
            _p(ie), _i(182), _i(180), _i(nb))
    x = x - (x[9, 9] - x0[9, 9])
    assert np.abs(x[1:-1] - x0[1:-1]).max() < 1e-10


@pytest.mark.parametrize("n0", [4, 8])
def test_pre_rep_basin_bit_exact(L, oracle, n0):
    p = P.basin(0)
    c = _coeffs(p)
    ie, _ = oracle.block_partition(96, 96 // n0)
    nb = len(ie)
    rinv = np.zeros((nb, 96, 96))
    rinv1 = np.zeros((nb - 1, 96, 96))
    h = np.zeros((98, 98))
    L.pre_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(h), _p(ie), _i(96), _i(98), _i(96), _i(nb))
    assert L.sevp_last_status() == 0
    r_o, r1_o, _ = oracle.pre(*c, ie)
    assert np.array_equal(rinv, r_o) and np.array_equal(rinv1, r1_o[: nb - 1])
    f = p.b.astype(np.float32)
    x = np.zeros((98, 98))
    d0, d1, d2, hh = np.zeros((nb - 1, 96)), np.zeros(96), np.zeros(96), np.zeros((98, 98))
    L.rep_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(d0), _p(d1), _p(d2), _p(f), _p(hh), _p(x),
           _p(ie), _i(98), _i(96), _i(nb))
    assert L.sevp_last_status() == 0
    xo = oracle.rep(*c, r_o, r1_o, f, np.zeros((98, 98)), ie)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("n", [1, 7, 64, 333])
def test_matinv_bit_exact(L, oracle, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = np.asfortranarray(a.copy())
    L.matinv_(b.ctypes.data_as(C.c_void_p), _i(n))
    assert L.sevp_last_status() == 0
    bo, st = oracle.matinv(a)
    assert st == 0
    assert np.array_equal(np.asarray(b), bo)
    assert np.allclose(np.asarray(b) @ a, np.eye(n), atol=1e-10)


def test_matinv_zero_pivot_status(L):
    b = np.asfortranarray(np.array([[0.0, 1.0], [1.0, 0.0]]))
    L.matinv_(b.ctypes.data_as(C.c_void_p), _i(2))
    assert L.sevp_last_status() == 7  # SEVP_SINGULAR


def test_bir_strips_bit_exact(L, oracle):
    """PRE for the NBIR strips (P/prep_GLOBAL.f90:272-318) and the 5
    multiplicative Schwarz sweeps of FS_SOLVER (M/fs_GLOBAL.f90:1904-1966)."""
    p = _shifted_idealised(48, 30, 0.05)
    c = _coeffs(p)
    i2, j2, nbir = 48, 30, 4
    ibir = 2 * i2 // nbir
    ie, _ = oracle.block_partition(j2, 6)
    nb0 = len(ie)
    L_ = oracle.lib()
    rg = np.zeros((nbir, nb0, ibir * ibir))
    r1g = np.zeros((nbir, nb0 - 1, ibir * ibir))
    L.sevp_pre_strips_(*[_p(a) for a in c], _p(rg), _p(r1g), _p(ie), _i(i2), _i(j2), _i(nb0), _i(nbir))
    assert L.sevp_last_status() == 0
    ro = np.zeros_like(rg)
    r1o = np.zeros_like(r1g)
    ws = [np.zeros((j2, ibir), np.float32) for _ in range(5)]
    h = np.zeros((j2 + 2, ibir + 2))
    st = L_.or_pre_strips(*c, ro.reshape(-1), r1o.reshape(-1), h, ie, i2, j2, nb0, nbir, *ws)
    assert st == 0
    assert np.array_equal(rg, ro) and np.array_equal(r1g, r1o)
    rng = np.random.default_rng(3)
    s = rng.standard_normal((j2, i2)).astype(np.float32)
    for fix in (0, 1):
        x = np.zeros((j2 + 2, i2 + 2))
        xx = np.zeros((j2 + 2, ibir + 2))
        xg, xxg = x.copy(), xx.copy()
        L.sevp_bir_sweeps_(*[_p(a) for a in c], _p(s), _p(rg), _p(r1g), _p(xg), _p(xxg), _p(ie),
                           _i(i2), _i(j2), _i(nb0), _i(nbir), _i(5), _i(fix))
        assert L.sevp_last_status() == 0
        wsrc = [np.zeros((j2, ibir), np.float32) for _ in range(6)]
        hw = np.zeros((j2 + 2, ibir + 2))
        d0, d1, d2 = np.zeros((nb0 - 1, ibir)), np.zeros(ibir), np.zeros(ibir)
        L_.or_bir_sweeps(*c, s, ro.reshape(-1), r1o.reshape(-1), x, xx, hw, *wsrc, d0, d1, d2, ie,
                         i2, j2, nb0, nbir, 5, 1, fix)
        assert np.array_equal(xg, x) and np.array_equal(xxg, xx), fix


def test_sqprod_bit_exact_and_inprod(L, oracle):
    p = P.global_grid(90, 45, seed=9)
    c = _coeffs(p)
    j2, i2 = p.ac.shape
    rng = np.random.default_rng(4)
    x = rng.standard_normal((j2 + 2, i2 + 2))
    for name, ref in (("p_sqprod_", oracle.sqprod), ("p_sqprod_t_", oracle.sqprod_t)):
        r = rng.standard_normal((j2 + 2, i2 + 2))
        rg = r.copy()
        getattr(L, name)(*[_p(a) for a in c], _p(x), _p(rg), _i(i2), _i(j2))
        ro = ref(*c, x)
        ro[0, :], ro[-1, :], ro[:, 0], ro[:, -1] = r[0, :], r[-1, :], r[:, 0], r[:, -1]
        assert np.array_equal(rg, ro), name
    y = rng.standard_normal((j2 + 2, i2 + 2))
    tp = C.c_double()
    L.p_inprod_(_p(x), _p(y), C.byref(tp), _i(i2), _i(j2))
    to = oracle.inprod(x, y)
    assert abs(tp.value - to) <= 1e-13 * np.abs(x[1:-1, 1:-1] * y[1:-1, 1:-1]).sum()


def test_bicgstab_known_answer_and_oracle(L, oracle):
    """p_bicgstab_le on the harness problem converges to a constant; on a
    nonsingular problem it matches the oracle's solution within the
    stopping tolerance."""
    p = P.idealised(180, 90)
    c = _coeffs(p)
    x0 = np.zeros((92, 182))
    x = x0.copy()
    x[2:89, 2:179] = 1.0
    b = np.zeros((90, 180), np.float32)
    xg = x.copy()
    L.p_bicgstab_le_(*[_p(a) for a in c], _p(b), _p(xg), *[_p(a) for a in c], _i(180), _i(90))
    assert L.sevp_last_status() == 0
    xg = xg - (xg[9, 9] - x0[9, 9])
    assert np.abs(xg[1:-1] - x0[1:-1]).max() < 1e-6
    q = _shifted_idealised(120, 60, 0.02)
    c = _coeffs(q)
    rng = np.random.default_rng(5)
    b = rng.standard_normal((60, 120)).astype(np.float32)
    xg = np.zeros((62, 122))
    L.p_bicgstab_le_(*[_p(a) for a in c], _p(b), _p(xg), *[_p(a) for a in c], _i(120), _i(60))
    xo, it, res = oracle.bicgstab(*c, b, np.zeros((62, 122)))
    assert np.abs(xg - xo).max() <= 1e-6 * np.abs(xo).max()


def test_lanczos_csi(L, oracle):
    sp = P.basin(0, n=48)
    cs = [-np.ascontiguousarray(a, np.float32) for a in sp.coeffs()]  # SPD
    mn, mx = C.c_double(), C.c_double()
    L.lanczos_(*[_p(a) for a in cs], C.byref(mn), C.byref(mx), _i(48), _i(48))
    assert L.sevp_last_status() == 0
    mno, mxo, ierr, _, _ = oracle.lanczos(*cs)
    assert ierr == 0
    assert abs(mn.value - mno) <= 1e-6 * abs(mxo) and abs(mx.value - mxo) <= 1e-8 * abs(mxo)
    q = _shifted_idealised(120, 60, 0.02)
    c = _coeffs(q)
    rng = np.random.default_rng(6)
    b = rng.standard_normal((60, 120)).astype(np.float32)
    # Chebyshev with bounds that enclose the spectrum (the reference's own
    # bounds from 10 Lanczos steps may not)
    lo, hi = 0.02, 2.03
    xg = np.zeros((62, 122))
    L.p_csi_(*[_p(a) for a in c], C.byref(C.c_double(lo)), C.byref(C.c_double(hi)), _p(b), _p(xg),
             *[_p(a) for a in c], _i(120), _i(60))
    assert L.sevp_last_status() == 0
    xo, it, res = oracle.csi(*c, lo, hi, b, np.zeros((62, 122)))
    assert res <= 1e-7
    assert np.abs(xg - xo).max() <= 1e-6 * np.abs(xo).max()


def test_dropin_bad_args(L):
    L.matinv_(None, _i(3))
    assert L.sevp_last_status() == 5
    x = np.zeros((4, 5))
    L.p_inprod_(_p(x), _p(x), None, _i(3), _i(2))
    assert L.sevp_last_status() == 5


def test_repbir_period_and_repbir_bit_exact(L, oracle):
    """REPBIR_PERIOD (full width, M/sevp.f90:109-217) and REPBIR on a strip
    of M2 columns (M/sevp.f90:218-328) equal the oracle bit for bit."""
    p = _shifted_idealised(120, 60)
    c = _coeffs(p)
    j2, i2 = p.ac.shape
    ie, ok = oracle.block_partition(j2, 10)
    nb = len(ie)
    rng = np.random.default_rng(6)
    # full width, periodic
    rinv, rinv1, st = oracle.pre1(*c, ie)
    f = rng.standard_normal((j2, i2)).astype(np.float32)
    x = np.zeros((j2 + 2, i2 + 2))
    x[0] = rng.standard_normal(i2 + 2)
    xg = x.copy()
    d0, d1, d2 = np.zeros((nb - 1, i2)), np.zeros(i2), np.zeros(i2)
    hh = np.zeros((j2 + 2, i2 + 2))
    L.repbir_period_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(d0), _p(d1), _p(d2), _p(f),
                     _p(hh), _p(xg), _p(ie), _i(i2 + 2), _i(i2), _i(i2 + 2), _i(i2), _i(nb))
    assert L.sevp_last_status() == 0
    xo, st = oracle.repbir_period(*c, rinv, rinv1, f, x, ie)
    assert st == 0 and np.array_equal(xg, xo)
    # strip of m2 columns with Dirichlet side columns
    m2 = 40
    rinv, rinv1, st = oracle.pre(*c, ie, m2=m2)
    f = rng.standard_normal((j2, m2)).astype(np.float32)
    x = np.zeros((j2 + 2, m2 + 2))
    x[:, 0] = rng.standard_normal(j2 + 2)
    x[:, -1] = rng.standard_normal(j2 + 2)
    xg = x.copy()
    d0, d1, d2 = np.zeros((nb - 1, m2)), np.zeros(m2), np.zeros(m2)
    hh = np.zeros((j2 + 2, m2 + 2))
    L.repbir_(*[_p(a) for a in c], _p(rinv), _p(rinv1), _p(d0), _p(d1), _p(d2), _p(f), _p(hh),
              _p(xg), _p(ie), _i(m2 + 2), _i(i2), _i(m2 + 2), _i(m2), _i(nb))
    assert L.sevp_last_status() == 0
    xo, _ = oracle.repbir(*c, rinv, rinv1, f, x, ie, m2)
    assert np.array_equal(xg, xo)
