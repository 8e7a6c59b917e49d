"""Host-side pieces of the fast drop-in p_sevp_pcg_ (no GPU):

* ``problems.prep_assemble`` restates PREP's coefficient assembly
  (P/prep_GLOBAL.f90:170-244) in numpy float32; it equals the oracle's C
  restatement (or_assemble) bit for bit;
* ``sevp_row_symmetrize`` (the library's host row scaling) finds weights
  w_J proportional to 1 / (OCS(J+1) ODY(J+1)) -- the factor PREP puts in
  row J of AB and AT -- and returns exactly symmetric planes within FP32
  rounding of W A;
* operators that no row scaling symmetrises are refused.
"""
import ctypes as C

import numpy as np
import pytest

from musoc_solver_b200 import problems as P


@pytest.fixture(scope="module")
def L():
    from musoc_solver_b200 import build, native

    build.build()
    return native.lib()


def _sym(L, planes, periodic):
    j2, i2 = planes[2].shape
    f32 = [np.ascontiguousarray(a, np.float32) for a in planes]
    w = np.zeros(j2)
    sym = np.zeros((5, j2, i2), np.float32)
    st = L.sevp_row_symmetrize(*[a.ctypes.data_as(C.c_void_p) for a in f32], i2, j2, int(periodic),
                               w.ctypes.data_as(C.c_void_p), sym.ctypes.data_as(C.c_void_p))
    return st, w, sym


@pytest.mark.parametrize("periodic", [True, False])
def test_prep_assemble_matches_oracle(oracle, periodic):
    p = P.prep_grid(50, 30, k1=5, seed=1, periodic=periodic)
    m = p.meta
    ref = oracle.assemble(p.nx, p.ny, m["k1"], m["odx"], m["ody"], m["csv"], m["ocs"], m["odyv"],
                          m["odz"], m["iu"], m["iv"], m["nbir"], float(m["gamma"]), 0)
    for a, b in zip(ref, p.coeffs()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("periodic", [True, False])
def test_row_weights_undo_prep_row_factor(L, periodic):
    p = P.prep_grid(64, 40, k1=4, seed=5, periodic=periodic)
    st, w, sym = _sym(L, p.coeffs(), periodic)
    assert st == 0
    m = p.meta
    factor = m["ocs"][1:p.ny + 1].astype(np.float64) * m["ody"][1:p.ny + 1]  # OCS(J+1) ODY(J+1)
    ratio = w * factor
    assert np.abs(ratio / ratio[0] - 1).max() <= 1e-6
    sl, sb, sc, sr, st_ = sym
    # exact symmetry of the returned planes
    assert np.array_equal(sr[:, :-1], sl[:, 1:])
    assert np.array_equal(st_[:-1], sb[1:])
    if periodic:
        assert np.array_equal(sr[:, -1], sl[:, 0])
    else:
        assert (sl[:, 0] == 0).all() and (sr[:, -1] == 0).all()
    assert (sb[0] == 0).all() and (st_[-1] == 0).all()
    # the planes are W A up to FP32 rounding
    al, ab, ac, ar, at = (a.astype(np.float64) for a in p.coeffs())
    wc = w[:, None]
    assert np.abs(sc - wc * ac).max() <= 1e-6 * np.abs(wc * ac).max()
    assert np.abs(st_[:-1] - wc[:-1] * at[:-1]).max() <= 1e-6 * np.abs(wc * at).max()
    assert np.abs(sb[1:] - wc[1:] * ab[1:]).max() <= 1e-6 * np.abs(wc * ab).max()
    assert np.isclose(np.abs(sc).max(), 1.0, rtol=1e-6)


def test_symmetric_input_keeps_unit_ratios(L):
    p = P.idealised(40, 20)
    st, w, sym = _sym(L, p.coeffs(), True)
    assert st == 0 and np.allclose(w, w[0])
    assert np.array_equal(sym[2], p.ac * np.float32(w[0]))


def test_unsymmetrisable_operator_refused(L):
    p = P.prep_grid(32, 16, k1=3, seed=2, periodic=True)
    planes = [np.array(a) for a in p.coeffs()]
    planes[3][4, 5] *= np.float32(1.01)  # AR(6, 5) != AL(7, 5)
    st, _, _ = _sym(L, planes, True)
    assert st == 8
    assert "AR(I,J) differs from AL(I+1,J)" in L.sevp_last_error().decode()


def test_block_partition_matches_oracle(L, oracle):
    """sevp_block_partition (host code in the library) against the oracle's
    restatement of P/prep_GLOBAL.f90:148-168, valid and invalid partitions,
    including quotients that round half away from zero."""
    seen_bad = seen_ok = 0
    for dimen in (2, 3):
        for j2 in (1, 2, 3, 5, 7, 10, 15, 24, 25, 90, 92, 181, 2398, 2400):
            for nb0 in (2, 3, 4, 5, 6, 8, 12, 15, 16, 50, 400):
                ie = np.zeros(nb0, np.int32)
                st = L.sevp_block_partition(j2, nb0, dimen, ie.ctypes.data_as(C.c_void_p))
                ref, ok = oracle.block_partition(j2, nb0, dimen)
                assert np.array_equal(ie, ref), (j2, nb0, dimen)
                assert (st == 0) == ok, (j2, nb0, dimen, st)
                if ok:
                    seen_ok += 1
                else:
                    seen_bad += 1
                    assert "not properly defined" in L.sevp_last_error().decode()
    assert seen_ok > 20 and seen_bad > 20
    # the reference's 182 x 92 grid with 15 blocks (I2 = 180, J2 = 90)
    ie = np.zeros(15, np.int32)
    assert L.sevp_block_partition(90, 15, 3, ie.ctypes.data_as(C.c_void_p)) == 0
    assert ie.tolist() == [7, 13, 19, 25, 31, 37, 43, 49, 55, 61, 67, 73, 79, 85, 91]
    assert L.sevp_block_partition(90, 1, 3, ie.ctypes.data_as(C.c_void_p)) == 5
