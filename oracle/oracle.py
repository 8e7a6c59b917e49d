"""ctypes binding of the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by the smoke check and by
the CPU-baseline leg of ``bench.py``.  The product library never uses it.

Each wrapper names the reference routine it restates; arrays follow the
reference layout (column-major (I, J) == C-order (J, I) numpy arrays).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(_HERE, "sevp_oracle.c")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        c5 = [f32p] * 5
        L.or_rep1.argtypes = c5 + [f64p, f64p, f64p, f64p, f64p, f32p, f64p, f64p, i32p] + [C.c_int] * 3
        L.or_rep.argtypes = L.or_rep1.argtypes
        L.or_repbir.argtypes = c5 + [f64p, f64p, f64p, f64p, f64p, f32p, f64p, f64p, i32p] + [C.c_int] * 5
        L.or_repbir_period.argtypes = L.or_repbir.argtypes
        L.or_repbir_period.restype = C.c_int
        L.or_pre1.argtypes = c5 + [f64p, f64p, f64p, i32p] + [C.c_int] * 3
        L.or_pre1.restype = C.c_int
        L.or_pre.argtypes = c5 + [f64p, f64p, f64p, i32p] + [C.c_int] * 4
        L.or_pre.restype = C.c_int
        L.or_matinv.argtypes = [f64p, C.c_int]
        L.or_matinv.restype = C.c_int
        L.or_matinv_pivot.argtypes = [f64p, C.c_int]
        L.or_matinv_pivot.restype = C.c_int
        L.or_block_partition.argtypes = [C.c_int, C.c_int, C.c_int, i32p]
        L.or_block_partition.restype = C.c_int
        L.or_sqprod.argtypes = c5 + [f64p, f64p, C.c_int, C.c_int]
        L.or_sqprod_t.argtypes = L.or_sqprod.argtypes
        L.or_inprod.argtypes = [f64p, f64p, C.c_int, C.c_int]
        L.or_inprod.restype = C.c_double
        L.or_bicgstab_le.argtypes = c5 + [f32p, f64p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.or_bicgstab_le.restype = C.c_int
        L.or_csi.argtypes = c5 + [C.c_double, C.c_double, f32p, f64p, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_double)]
        L.or_csi.restype = C.c_int
        L.or_lanczos.argtypes = c5 + [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      f64p, f64p]
        L.or_lanczos.restype = C.c_int
        L.or_figi.argtypes = [C.c_int, f64p, f64p, f64p, f64p]
        L.or_figi.restype = C.c_int
        L.or_ratqr.argtypes = [C.c_int, C.c_double, f64p, f64p, C.POINTER(C.c_double)]
        L.or_ratqr.restype = C.c_int
        L.or_bir_sweeps.argtypes = (c5 + [f32p, f64p, f64p, f64p, f64p, f64p] + [f32p] * 6
                                    + [f64p, f64p, f64p, i32p] + [C.c_int] * 7)
        L.or_pre_strips.argtypes = c5 + [f64p, f64p, f64p, i32p] + [C.c_int] * 4 + [f32p] * 5
        L.or_pre_strips.restype = C.c_int
        L.or_assemble.argtypes = ([C.c_int] * 3 + [f32p] * 6 + [i32p, i32p, C.c_int, C.c_float, C.c_int]
                                  + [f32p] * 5)
        L.or_assemble_dim.argtypes = ([C.c_int] * 4 + [f32p] * 6
                                      + [i32p, i32p, C.c_int, C.c_float, C.c_int] + [f32p] * 5)
        L.or_tile_setup.argtypes = c5 + [C.c_int] * 4 + [i32p, C.POINTER(C.c_int)]
        L.or_tile_setup.restype = C.c_void_p
        L.or_tile_free.argtypes = [C.c_void_p]
        L.or_tile_count.argtypes = [C.c_void_p]
        L.or_tile_count.restype = C.c_int
        L.or_tile_get.argtypes = [C.c_void_p, C.c_int, i32p, C.c_void_p, C.c_void_p]
        L.or_tile_apply.argtypes = [C.c_void_p] + c5 + [f64p, f64p]
        L.or_apply.argtypes = c5 + [C.c_int] * 3 + [f64p, f64p]
        L.or_dot.argtypes = [f64p, f64p, C.c_int, C.c_int]
        L.or_dot.restype = C.c_double
        L.or_pcg.argtypes = [C.c_void_p] + c5 + [C.c_int, f64p, f64p, C.c_double, C.c_int,
                                                 C.POINTER(C.c_double)]
        L.or_pcg.restype = C.c_int
        L.or_cheb.argtypes = [C.c_void_p] + c5 + [C.c_int, f64p, f64p, C.c_double, C.c_double,
                                                  C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.or_cheb.restype = C.c_int
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def block_partition(j2: int, nb0: int, dimen: int = 3):
    """IE of P/prep_GLOBAL.f90:148-168; returns (ie, ok)."""
    ie = np.zeros(nb0, np.int32)
    st = lib().or_block_partition(j2, nb0, dimen, ie)
    return ie, st == 0


def pre1(al, ab, ac, ar, at, ie):
    """PRE1 (P/prep_GLOBAL.f90:327-386): RINV (NB0,I2,I2), RINV1 (NB0-1,I2,I2)
    as C arrays whose last two axes are the Fortran (I2, I2) column-major."""
    j2, i2 = ac.shape
    nb = len(ie)
    rinv = np.zeros((nb, i2, i2))
    rinv1 = np.zeros((max(nb - 1, 1), i2, i2))
    h = np.zeros((j2 + 2, i2 + 2))
    st = lib().or_pre1(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], rinv, rinv1, h,
                       _c(ie, np.int32), i2 + 2, i2, nb)
    return rinv, rinv1, st


def pre(al, ab, ac, ar, at, ie, i2_ld=None, m2=None):
    """PRE (P/prep_GLOBAL.f90:457-513) on the first m2 columns."""
    j2, i2 = ac.shape
    m2 = m2 or i2
    nb = len(ie)
    rinv = np.zeros((nb, m2, m2))
    rinv1 = np.zeros((max(nb - 1, 1), m2, m2))
    h = np.zeros((j2 + 2, m2 + 2))
    st = lib().or_pre(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], rinv, rinv1, h,
                      _c(ie, np.int32), i2, m2 + 2, m2, nb)
    return rinv, rinv1, st


def _rep_common(fn, al, ab, ac, ar, at, rinv, rinv1, f, x, ie):
    j2, i2 = ac.shape
    nb = len(ie)
    i0 = i2 + 2
    x = _c(x, np.float64).copy()
    dum0 = np.zeros((max(nb - 1, 1), i2))
    dum1 = np.zeros(i2)
    dum2 = np.zeros(i2)
    h = np.zeros_like(x)
    fn(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], _c(rinv, np.float64), _c(rinv1, np.float64),
       dum0, dum1, dum2, _c(f, np.float32), h, x, _c(ie, np.int32), i0, i2, nb)
    return x


def rep1(al, ab, ac, ar, at, rinv, rinv1, f, x, ie):
    """REP1 (M/sevp.f90:11-107); x is the padded (J0, I0) field, returned."""
    return _rep_common(lib().or_rep1, al, ab, ac, ar, at, rinv, rinv1, f, x, ie)


def rep(al, ab, ac, ar, at, rinv, rinv1, f, x, ie):
    """REP (M/sevp.f90:335-438)."""
    return _rep_common(lib().or_rep, al, ab, ac, ar, at, rinv, rinv1, f, x, ie)


def _strip_common(fn, al, ab, ac, ar, at, rinv, rinv1, f, x, ie, m2):
    """REPBIR-style call on the first m2 columns: coefficients keep the full
    leading dimension I2, F and RINV have m2 columns, X and H have m2 + 2."""
    j2, i2 = ac.shape
    nb = len(ie)
    i0 = x.shape[1]
    m0 = m2 + 2
    x = _c(x, np.float64).copy()
    dum0 = np.zeros((max(nb - 1, 1), m2))
    dum1 = np.zeros(m2)
    dum2 = np.zeros(m2)
    h = np.zeros((x.shape[0], m0))
    st = fn(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], _c(rinv, np.float64),
            _c(rinv1, np.float64), dum0, dum1, dum2, _c(f, np.float32), h, x, _c(ie, np.int32),
            i0, i2, m0, m2, nb)
    return x, st


def repbir(al, ab, ac, ar, at, rinv, rinv1, f, x, ie, m2):
    """REPBIR (M/sevp.f90:218-328) on the first m2 columns; x is (J0, m2+2)
    or wider (leading dimension I0 = x.shape[1])."""
    return _strip_common(lib().or_repbir, al, ab, ac, ar, at, rinv, rinv1, f, x, ie, m2)


def repbir_period(al, ab, ac, ar, at, rinv, rinv1, f, x, ie):
    """REPBIR_PERIOD (M/sevp.f90:109-217), defined for M0 == I0 (full width)."""
    j2, i2 = ac.shape
    return _strip_common(lib().or_repbir_period, al, ab, ac, ar, at, rinv, rinv1, f, x, ie, i2)


def matinv(b, pivot=False):
    b = np.array(b, dtype=np.float64, order="C")
    # the C routine is column-major: pass the transpose buffer and transpose back
    bt = np.ascontiguousarray(b.T)
    st = (lib().or_matinv_pivot if pivot else lib().or_matinv)(bt, b.shape[0])
    return np.ascontiguousarray(bt.T), st


def sqprod(al, ab, ac, ar, at, x):
    j2, i2 = ac.shape
    r = np.zeros((j2 + 2, i2 + 2))
    lib().or_sqprod(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], _c(x, np.float64), r, i2, j2)
    return r


def sqprod_t(al, ab, ac, ar, at, x):
    j2, i2 = ac.shape
    r = np.zeros((j2 + 2, i2 + 2))
    lib().or_sqprod_t(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], _c(x, np.float64), r, i2, j2)
    return r


def inprod(r, p):
    j0, i0 = r.shape
    return lib().or_inprod(_c(r, np.float64), _c(p, np.float64), i0 - 2, j0 - 2)


def bicgstab(al, ab, ac, ar, at, b, x, periodic=True):
    j2, i2 = ac.shape
    x = _c(x, np.float64).copy()
    res = C.c_double()
    it = lib().or_bicgstab_le(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], _c(b, np.float32), x,
                              i2, j2, int(periodic), C.byref(res))
    return x, it, res.value


def csi(al, ab, ac, ar, at, mineig, maxeig, b, x, periodic=True):
    j2, i2 = ac.shape
    x = _c(x, np.float64).copy()
    res = C.c_double()
    it = lib().or_csi(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], mineig, maxeig,
                      _c(b, np.float32), x, i2, j2, int(periodic), C.byref(res))
    return x, it, res.value


def lanczos(al, ab, ac, ar, at):
    j2, i2 = ac.shape
    mn, mx = C.c_double(), C.c_double()
    alpha = np.zeros(10)
    sigma = np.zeros(11)
    ierr = lib().or_lanczos(*[_c(a, np.float32) for a in (al, ab, ac, ar, at)], i2, j2, C.byref(mn),
                            C.byref(mx), alpha, sigma)
    return mn.value, mx.value, ierr, alpha, sigma


def assemble(i2, j2, k1, odx, ody, csv, ocs, odyv, odz, iu, iv, nbir, gamma, idealised):
    out = [np.zeros((j2, i2), np.float32) for _ in range(5)]
    lib().or_assemble(i2, j2, k1, *[_c(a, np.float32) for a in (odx, ody, csv, ocs, odyv, odz)],
                      _c(iu, np.int32), _c(iv, np.int32), nbir, gamma, int(idealised), *out)
    al, ar, ab, at, ac = out
    return al, ab, ac, ar, at


def assemble_dim(i2, j2, k1, dimen, odx, ody, csv, ocs, odyv, odz, iu, iv, nbir, gamma, idealised):
    """PREP's assembly with the DIMEN switch of P/prep_GLOBAL.f90:170-212;
    iu, iv are int32 masks of shape (K, J0, I0)."""
    out = [np.zeros((j2, i2), np.float32) for _ in range(5)]
    lib().or_assemble_dim(i2, j2, k1, dimen,
                          *[_c(a, np.float32) for a in (odx, ody, csv, ocs, odyv, odz)],
                          _c(iu, np.int32), _c(iv, np.int32), nbir, gamma, int(idealised), *out)
    al, ar, ab, at, ac = out
    return al, ab, ac, ar, at


class TilePC:
    """Oracle of the block-Jacobi tile SEVP preconditioner (new method)."""

    def __init__(self, p, tm, th, srow=None, tile_nb=None):
        """srow: sub-block height per tile row (scalar or ty values), or
        tile_nb: sub-blocks per tile, shape (ty, tx)."""
        self.p = p
        self.c = [_c(a, np.float32) for a in p.coeffs()]
        ty = (p.ny + th - 1) // th
        tx = (p.nx + tm - 1) // tm
        if tile_nb is None:
            srow = np.broadcast_to(np.asarray(srow, np.int64), (ty,))
            hh = np.minimum(th, p.ny - th * np.arange(ty))
            nb_row = -(-hh // np.maximum(srow, 1))
            tile_nb = np.repeat(nb_row[:, None], tx, axis=1)
        tile_nb = np.ascontiguousarray(np.asarray(tile_nb).reshape(ty, tx), np.int32)
        self.tile_nb = tile_nb
        st = C.c_int()
        self.h = lib().or_tile_setup(*self.c, p.nx, p.ny, tm, th, tile_nb, C.byref(st))
        self.status = st.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_tile_free(self.h)
            self.h = None

    def ntiles(self):
        return lib().or_tile_count(self.h)

    def tile(self, t):
        g = np.zeros(5, np.int32)
        lib().or_tile_get(self.h, t, g, None, None)
        mw, nb = int(g[2]), int(g[4])
        rinv = np.zeros((nb, mw, mw))
        rinv1 = np.zeros((max(nb - 1, 1), mw, mw))
        lib().or_tile_get(self.h, t, g, rinv.ctypes.data, rinv1.ctypes.data)
        return g, rinv, rinv1

    def apply(self, r):
        z = np.zeros_like(r, dtype=np.float64)
        lib().or_tile_apply(self.h, *self.c, _c(r, np.float64), z)
        return z

    def pcg(self, b, x0=None, tol=1e-12, maxit=10000):
        x = np.zeros(b.shape) if x0 is None else _c(x0, np.float64).copy()
        rel = C.c_double()
        it = lib().or_pcg(self.h, *self.c, int(self.p.periodic), _c(b, np.float64), x, tol, maxit,
                          C.byref(rel))
        return x, it, rel.value


    def cheb(self, b, lmin, lmax, x0=None, tol=1e-12, maxit=10000):
        """Preconditioned Chebyshev iteration on [lmin, lmax] (or_cheb)."""
        x = np.zeros(b.shape) if x0 is None else _c(x0, np.float64).copy()
        rel = C.c_double()
        it = lib().or_cheb(self.h, *self.c, int(self.p.periodic), _c(b, np.float64), x,
                           float(lmin), float(lmax), tol, maxit, C.byref(rel))
        return x, it, rel.value


class _Grid:
    """Coefficient planes of one operator (the fields TilePC reads)."""

    def __init__(self, al, ab, ac, ar, at, periodic):
        self.al, self.ab, self.ac, self.ar, self.at = al, ab, ac, ar, at
        self.periodic = periodic

    @property
    def nx(self):
        return int(self.ac.shape[1])

    @property
    def ny(self):
        return int(self.ac.shape[0])

    def coeffs(self):
        return self.al, self.ab, self.ac, self.ar, self.at


def rolled_grid(p, shift):
    """The operator of ``p`` on the grid rolled west by ``shift`` columns
    (column c of the result is column (c + shift) mod nx of ``p``).  On a
    closed grid the couplings across the original seam are zero, so the
    rolled tile that contains the seam falls into two independent pieces."""
    R = lambda a: np.ascontiguousarray(np.roll(np.asarray(a, np.float32), -shift, axis=1))
    al, ab, ac, ar, at = (R(a) for a in p.coeffs())
    if not p.periodic and shift:
        nx = al.shape[1]
        al[:, nx - shift] = 0.0      # original column 0: no west neighbour
        ar[:, nx - shift - 1] = 0.0  # original column nx-1: no east neighbour
    return _Grid(al, ab, ac, ar, at, p.periodic)


class SchwarzPC:
    """Oracle of the two-tiling overlapping Schwarz preconditioner (new
    method).  The reference's BIR solve (``M/fs_GLOBAL.f90:1902-1966``)
    sweeps 50 %-overlapping strips multiplicatively as a stand-alone solver;
    here two tilings, the second rolled west by ``shift`` columns, make one
    symmetric multiplicative sweep that serves as the PCG preconditioner:

        z1 = Ma r,  z2 = Mb (r - A z1),  z = z1 + z2 + Ma (r - A (z1 + z2)),

    with the residuals formed in full (the library forms them from the
    tile-boundary couplings, which is the same in exact arithmetic).
    tile_nb / tile_nb_b: sub-blocks per tile of the two tilings."""

    def __init__(self, p, tm, th, shift, tile_nb, tile_nb_b):
        self.p, self.shift = p, int(shift)
        self.a = TilePC(p, tm, th, tile_nb=tile_nb)
        self.b = TilePC(rolled_grid(p, self.shift), tm, th, tile_nb=tile_nb_b)
        self.status = self.a.status | self.b.status

    def _mb(self, r):
        s = self.shift
        return np.roll(self.b.apply(np.roll(r, -s, axis=1)), s, axis=1)

    def apply(self, r):
        r = np.asarray(r, np.float64)
        z = self.a.apply(r)
        z = z + self._mb(r - apply(self.p, z))
        return z + self.a.apply(r - apply(self.p, z))

    def pcg(self, b, tol=1e-12, maxit=10000):
        """Plain PCG with this preconditioner from x = 0; returns (x,
        iterations, relative residual of the recursion)."""
        b = np.asarray(b, np.float64)
        x = np.zeros_like(b)
        r = b.copy()
        bn = np.linalg.norm(b)
        if bn == 0.0:
            return x, 0, 0.0
        z = self.apply(r)
        pv = z.copy()
        rz = float((r * z).sum())
        for it in range(1, maxit + 1):
            q = apply(self.p, pv)
            a = rz / float((pv * q).sum())
            x += a * pv
            r -= a * q
            rel = np.linalg.norm(r) / bn
            if rel <= tol:
                return x, it, rel
            z = self.apply(r)
            rz2 = float((r * z).sum())
            pv = z + (rz2 / rz) * pv
            rz = rz2
        return x, maxit, np.linalg.norm(r) / bn


def apply(p, x):
    y = np.zeros_like(x, dtype=np.float64)
    lib().or_apply(*[_c(a, np.float32) for a in p.coeffs()], p.nx, p.ny, int(p.periodic),
                   _c(x, np.float64), y)
    return y


# ------------------------------------------------ barotropic correction of FS
def _fs_sigs():
    L = lib()
    if getattr(L, "_fs_sigs", False):
        return L
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    i16p = np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS")
    L.or_fs_mask.argtypes = [C.c_int, C.c_int, f32p, f32p, i16p, i16p, C.c_int]
    L.or_fs_mask.restype = None
    L.or_fs_rhs.argtypes = [C.c_int, C.c_int, C.c_int] + [f32p] * 8
    L.or_fs_rhs.restype = None
    L.or_fs_correct.argtypes = [C.c_int, C.c_int, C.c_int, f64p, C.c_float, f32p, f32p, i16p, i16p,
                                i16p, i16p, f32p, f32p, f32p, f32p, C.c_int]
    L.or_fs_correct.restype = C.c_float
    L._fs_sigs = True
    return L


def fs_mask(u, v, iu0, iv0, periodic=True):
    """In place on u (K1,J0,I0) and v (K1,J1,I0) (M/fs_GLOBAL.f90:1158-1171)."""
    k1, j0, i0 = u.shape
    _fs_sigs().or_fs_mask(i0, j0, u, v, iu0, iv0, int(periodic))


def fs_rhs(u, v, odx, ody, ocs, csv, odz):
    """S (J2,I2) from continuity (M/fs_GLOBAL.f90:1177-1192)."""
    k1, j0, i0 = u.shape
    s = np.zeros((j0 - 2, i0 - 2), np.float32)
    _fs_sigs().or_fs_rhs(i0, j0, k1 + 1, u, v, odx, ody, ocs, csv, odz, s)
    return s


def fs_correct(x_interior, odt, odx, odyv, iu, iv, iu0, iv0, p0, u, v, scr, periodic=True):
    """In place on p0, u, v, scr (4,J0,I0); x_interior is the (J2,I2) solution.
    Returns the largest top-layer land velocity (M/fs_GLOBAL.f90:1216-1276)."""
    k1, j0, i0 = u.shape
    x = np.zeros((j0, i0))
    x[1:-1, 1:-1] = x_interior
    return float(_fs_sigs().or_fs_correct(i0, j0, k1 + 1, x, np.float32(odt), odx, odyv, iu, iv,
                                          iu0, iv0, p0, u, v, scr, int(periodic)))
