"""Seeded synthetic elliptic problems for the barotropic-pressure solve.

The reference model (TIMCOM) assembles its 5-point coefficients from grid
metrics, layer thicknesses and land masks (``P/prep_GLOBAL.f90:170-261``) and
regularises the operator by treating the top layer as all water
(``P/prep_GLOBAL.f90:184-196``), so every marched north coefficient is
nonzero.  No data files travel here, so the problems below are generated from
a seed with the shapes and value ranges of the five workloads:

* ``basin``      96x96 closed basin, 10 km spacing, 12 Gaussian seamounts
* ``global_grid``  periodic-in-x latitude-longitude grid (1440x720, 3600x2400)
* ``eddy_rhs``   advected Gaussian-eddy right-hand sides for a time sequence
* ``ensemble``   members with +-5 % multiplicative depth noise
* ``idealised``  the constant test stencil of ``P/prep_GLOBAL.f90:246-261``

The operator is ``div(H grad eta) - eta / (g dt^2)`` in finite-volume form,
multiplied by the cell area so that the matrix is symmetric:

    AL*eta_W + AB*eta_S + AC*eta_C + AR*eta_E + AT*eta_N = b

with ``AL, AR`` = face depth x face length / centre distance on the x faces,
``AB, AT`` likewise on the y faces, and ``AC = -(AL+AR+AB+AT) - area/(g dt^2)``
(the sign convention of ``P/prep_GLOBAL.f90:240-244``).  Face depths are the
mean of the two cells, floored at 50 m: that floor is the regularisation (land
cells stay in the system; the right-hand side is zero there).

Arrays are float32 coefficient planes and a float64 right-hand side of shape
``(ny, nx)`` in C order, which is the memory layout of the reference's
column-major ``(I2, J2)`` arrays.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

G = 9.81
EARTH_R = 6.371e6
DEPTH_FLOOR = 50.0


@dataclass
class Problem:
    """One elliptic problem: coefficients, right-hand side and metadata."""

    al: np.ndarray
    ab: np.ndarray
    ac: np.ndarray
    ar: np.ndarray
    at: np.ndarray
    b: np.ndarray
    periodic: bool
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nx(self) -> int:
        return int(self.ac.shape[1])

    @property
    def ny(self) -> int:
        return int(self.ac.shape[0])

    def coeffs(self):
        return self.al, self.ab, self.ac, self.ar, self.at


def smooth_field(ny: int, nx: int, scale: float, rng: np.random.Generator) -> np.ndarray:
    """Zero-mean, unit-variance random field with Gaussian spectral falloff.

    ``scale`` is the correlation length in grid cells.  Periodic in both axes.
    """
    w = rng.standard_normal((ny, nx))
    f = np.fft.rfft2(w)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    f *= np.exp(-((kx**2 + ky**2) * (np.pi * scale) ** 2))
    out = np.fft.irfft2(f, s=(ny, nx))
    out -= out.mean()
    sd = out.std()
    return out / (sd if sd > 0 else 1.0)


def _coefficients(depth, dx_c, dx_f, dy, dt, periodic):
    """Symmetric area-weighted coefficients from cell depths.

    depth: (ny, nx) cell depths (m, land <= 0); dx_c: (ny,) x spacing at cell
    centres; dx_f: (ny+1,) x spacing at the y faces; dy: scalar.
    """
    ny, nx = depth.shape
    hpos = np.maximum(depth, 0.0)
    # x faces: between i and i+1 (last column wraps when periodic)
    hx = 0.5 * (hpos + np.roll(hpos, -1, axis=1))
    hx = np.maximum(hx, DEPTH_FLOOR)
    kx = hx * (dy / dx_c)[:, None]
    ar = kx.copy()
    al = np.roll(kx, 1, axis=1)
    if not periodic:
        ar[:, -1] = 0.0
        al[:, 0] = 0.0
    # y faces: between j and j+1
    hy = 0.5 * (hpos[:-1] + hpos[1:])
    hy = np.maximum(hy, DEPTH_FLOOR)
    ky = hy * (dx_f[1:-1] / dy)[:, None]
    at = np.zeros_like(depth)
    ab = np.zeros_like(depth)
    at[:-1] = ky
    ab[1:] = ky
    area = (dx_c * dy)[:, None] * np.ones((1, nx))
    gamma = area / (G * dt * dt)
    al32, ar32, ab32, at32 = (a.astype(np.float32) for a in (al, ar, ab, at))
    ac = -(al32.astype(np.float64) + ar32 + ab32 + at32) - gamma
    return al32, ab32, ac.astype(np.float32), ar32, at32, area


def basin(seed: int = 0, n: int = 96, dx: float = 10e3, dt: float = 60.0) -> Problem:
    """Closed basin: H = 4000 m minus 12 Gaussian seamounts, land where H<50 m,
    right-hand side i.i.d. N(0, 1e-6) on wet points (times the cell area)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:n, 0:n].astype(np.float64) * dx
    depth = np.full((n, n), 4000.0)
    for _ in range(12):
        cx, cy = rng.uniform(0, n * dx, size=2)
        h = rng.uniform(500.0, 3000.0)
        r = rng.uniform(20e3, 80e3)
        depth -= h * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / r**2)
    wet = depth >= 50.0
    dxc = np.full(n, dx)
    dxf = np.full(n + 1, dx)
    al, ab, ac, ar, at, area = _coefficients(depth, dxc, dxf, dx, dt, periodic=False)
    f = rng.normal(0.0, 1e-6, size=(n, n)) * wet
    b = f * area
    return Problem(al, ab, ac, ar, at, b, periodic=False, name=f"basin{n}",
                   meta=dict(depth=depth, wet=wet, dx=dx, dt=dt, area=area))


def _global_geometry(nx, ny, lat_max):
    dlat = 2.0 * lat_max / ny
    lat_c = -lat_max + (np.arange(ny) + 0.5) * dlat
    lat_f = -lat_max + np.arange(ny + 1) * dlat
    dlon = np.deg2rad(360.0 / nx)
    dx_c = EARTH_R * dlon * np.cos(np.deg2rad(lat_c))
    dx_f = EARTH_R * dlon * np.cos(np.deg2rad(lat_f))
    dy = EARTH_R * np.deg2rad(dlat)
    return lat_c, dx_c, dx_f, dy


def _gaussians_separable(lon, lat, centers_lon, centers_lat, radii_km, amps):
    """Sum of Gaussians exp(-d^2/R^2) with d in a local planar metric at each
    centre's latitude; separable in (lat, lon), so the sum is one GEMM."""
    km_per_deg = EARTH_R * np.pi / 180.0 / 1e3
    dlon = (lon[None, :] - centers_lon[:, None] + 180.0) % 360.0 - 180.0
    gx = np.exp(-((dlon * km_per_deg * np.cos(np.deg2rad(centers_lat))[:, None]) ** 2)
                / radii_km[:, None] ** 2)
    gy = np.exp(-(((lat[None, :] - centers_lat[:, None]) * km_per_deg) ** 2) / radii_km[:, None] ** 2)
    return (gy.T * amps[None, :]) @ gx


def global_depth(nx, ny, seed, lat_max=78.0, land_frac=0.3, n_gauss=200):
    """Synthetic bathymetry: 4000 m plus 200 seeded Gaussians, continents from a
    thresholded smooth random field covering ``land_frac`` of the cells."""
    rng = np.random.default_rng(seed)
    lat_c, _, _, _ = _global_geometry(nx, ny, lat_max)
    lon = (np.arange(nx) + 0.5) * 360.0 / nx
    c_lon = rng.uniform(0, 360, n_gauss)
    c_lat = rng.uniform(-lat_max, lat_max, n_gauss)
    rad = rng.uniform(100.0, 800.0, n_gauss)
    amp = rng.uniform(-1800.0, 1800.0, n_gauss)
    depth = 4000.0 + _gaussians_separable(lon, lat_c, c_lon, c_lat, rad, amp)
    depth = np.clip(depth, 200.0, 6500.0)
    # continents: correlation length ~ 1/12 of the zonal extent
    cont = smooth_field(ny, nx, max(nx / 12.0, 2.0), rng)
    thresh = np.quantile(cont, land_frac)
    land = cont < thresh
    depth = np.where(land, 0.0, depth)
    return depth, lat_c, lon


def global_grid(nx: int = 1440, ny: int = 720, seed: int = 1, dt: float = 60.0,
                lat_max: float = 78.0, rhs: str = "divergence") -> Problem:
    """Periodic-in-x grid, lat in [-lat_max, lat_max], dx = R dlon cos(lat).

    The right-hand side is the flux divergence of a seeded smooth velocity
    field through wet faces (the analogue of the reference's surface W from
    continuity, ``M/fs_GLOBAL.f90:1178-1193``)."""
    depth, lat_c, lon = global_depth(nx, ny, seed, lat_max)
    _, dx_c, dx_f, dy = _global_geometry(nx, ny, lat_max)
    al, ab, ac, ar, at, area = _coefficients(depth, dx_c, dx_f, dy, dt, periodic=True)
    wet = depth > 0.0
    rng = np.random.default_rng(seed + 7919)
    if rhs == "divergence":
        b = divergence_rhs(depth, dx_c, dx_f, dy, rng, scale=max(nx / 60.0, 2.0))
    else:
        b = rng.normal(0.0, 1e-6, size=depth.shape) * wet * area
    return Problem(al, ab, ac, ar, at, b, periodic=True, name=f"global{nx}x{ny}",
                   meta=dict(depth=depth, wet=wet, dt=dt, lat=lat_c, lon=lon, dx=dx_c,
                             dy=dy, area=area, dxf=dx_f))


def divergence_rhs(depth, dx_c, dx_f, dy, rng, scale, speed=0.1):
    """Volume-flux divergence of a smooth random velocity through wet faces."""
    ny, nx = depth.shape
    wet = depth > 0.0
    hpos = np.maximum(depth, 0.0)
    u = speed * smooth_field(ny, nx, scale, rng)
    v = speed * smooth_field(ny, nx, scale, rng)
    wet_e = wet & np.roll(wet, -1, axis=1)
    hx = 0.5 * (hpos + np.roll(hpos, -1, axis=1))
    fx = np.where(wet_e, hx * u * dy, 0.0)  # flux through the east face of (i, j)
    wet_n = np.zeros_like(wet)
    wet_n[:-1] = wet[:-1] & wet[1:]
    hy = np.zeros_like(hpos)
    hy[:-1] = 0.5 * (hpos[:-1] + hpos[1:])
    fy = np.where(wet_n, hy * v * dx_f[1:, None], 0.0)  # through the north face
    div = fx - np.roll(fx, 1, axis=1)
    div += fy
    div[1:] -= fy[:-1]
    return div


def eddy_rhs(nx: int, ny: int, steps, seed: int = 3, n_eddies: int = 300,
             lat_max: float = 78.0, dt: float = 60.0, speed: float = 0.2,
             amp_scale: float = 1e-6):
    """Right-hand sides of a time sequence: 300 Gaussian eddies (radius
    50-150 km) advected at 0.2 m/s with a slow sinusoidal amplitude drift.

    Yields (n, b_n) for n in ``steps``; b_n = area * sum of eddies.  The eddy
    centres move by speed*dt per step along a seeded heading."""
    rng = np.random.default_rng(seed)
    lat_c, dx_c, _, dy = _global_geometry(nx, ny, lat_max)
    lon = (np.arange(nx) + 0.5) * 360.0 / nx
    c_lon0 = rng.uniform(0, 360, n_eddies)
    c_lat0 = rng.uniform(-0.9 * lat_max, 0.9 * lat_max, n_eddies)
    rad = rng.uniform(50.0, 150.0, n_eddies)
    amp0 = rng.normal(0.0, 1.0, n_eddies)
    heading = rng.uniform(0, 2 * np.pi, n_eddies)
    period = rng.uniform(200.0, 800.0, n_eddies)  # amplitude drift period in steps
    phase = rng.uniform(0, 2 * np.pi, n_eddies)
    area = (dx_c * dy)[:, None]
    deg_per_m = 180.0 / (np.pi * EARTH_R)
    for n in steps:
        dist = speed * dt * n
        c_lat = np.clip(c_lat0 + np.sin(heading) * dist * deg_per_m, -lat_max, lat_max)
        c_lon = c_lon0 + np.cos(heading) * dist * deg_per_m / np.cos(np.deg2rad(c_lat))
        amp = amp0 * (1.0 + 0.3 * np.sin(2 * np.pi * n / period + phase))
        f = _gaussians_separable(lon, lat_c, c_lon % 360.0, c_lat, rad, amp)
        yield n, amp_scale * f * area


def ensemble(members: int = 64, nx: int = 720, ny: int = 360, seed: int = 5,
             noise: float = 0.05, dt: float = 60.0):
    """Ensemble members sharing one base bathymetry, each with independently
    seeded +-5 % multiplicative depth noise and its own right-hand side."""
    base, lat_c, lon = global_depth(nx, ny, seed)
    _, dx_c, dx_f, dy = _global_geometry(nx, ny, 78.0)
    out = []
    for m in range(members):
        rng = np.random.default_rng(seed * 1000 + m)
        depth = base * (1.0 + noise * rng.uniform(-1.0, 1.0, size=base.shape))
        al, ab, ac, ar, at, area = _coefficients(depth, dx_c, dx_f, dy, dt, periodic=True)
        b = divergence_rhs(depth, dx_c, dx_f, dy, rng, scale=max(nx / 60.0, 2.0))
        out.append(Problem(al, ab, ac, ar, at, b, periodic=True, name=f"member{m}",
                           meta=dict(depth=depth, dt=dt)))
    return out


@dataclass
class FSState:
    """A layered ocean state for the barotropic correction loop of FS, in the
    reference's array shapes (C-order with I fastest): u (K1,J0,I0),
    v (K1,J1,I0), p0 (J0,I0), scr (4,J0,I0); masks iu0 / iv0 (J0,I0),
    iu (K1,J0,I0), iv (K1,J1,I0) int16; metrics odx / ody / ocs (J0),
    csv / odyv (J1), odz (K1) float32; odt; and the symmetric (row-scaled)
    operator with its row scale (J2) for the solve."""

    u: np.ndarray
    v: np.ndarray
    p0: np.ndarray
    scr: np.ndarray
    iu0: np.ndarray
    iv0: np.ndarray
    iu: np.ndarray
    iv: np.ndarray
    odx: np.ndarray
    ody: np.ndarray
    ocs: np.ndarray
    csv: np.ndarray
    odyv: np.ndarray
    odz: np.ndarray
    odt: float
    problem: Problem
    rscale: np.ndarray

    @property
    def dims(self):
        k1, j0, i0 = self.u.shape
        return i0, j0, k1 + 1


def fs_state(nx: int = 96, ny: int = 48, k1: int = 6, seed: int = 0, dt: float = 60.0,
             lat_max: float = 78.0, speed: float = 0.1) -> FSState:
    """Seeded layered state on the periodic global grid (interior nx x ny,
    k1 layers of 4000 m in total).  Cells are wet in layer k where the
    synthetic depth reaches the layer's top (the top layer counts as water
    everywhere, as in the reference's solver coefficients); a face is wet
    where both of its cells are.  The operator is the FLAG_FS form
    div(sum_k dz_k mask_k grad) - 1/(g dt^2) with the reference's metric
    factors (the assembly of P/prep_GLOBAL.f90:170-261), multiplied per row
    by 1/(OCS(J) ODY(J)) so that it is symmetric; rscale is that factor."""
    i2, j2 = nx, ny
    i0, j0 = i2 + 2, j2 + 2
    rng = np.random.default_rng(seed)
    dlat = 2.0 * lat_max / ny
    lat_c = -lat_max + (np.arange(j0) - 0.5) * dlat          # cell J = 1..J0
    lat_v = -lat_max + np.arange(j0 - 1) * dlat              # V face J = 1..J1
    dlon = np.deg2rad(360.0 / nx)
    dy = EARTH_R * np.deg2rad(dlat)
    odx = (1.0 / (EARTH_R * dlon * np.cos(np.deg2rad(lat_c)))).astype(np.float32)
    ody = np.full(j0, 1.0 / dy, np.float32)
    ocs = (1.0 / np.cos(np.deg2rad(lat_c))).astype(np.float32)
    csv = np.cos(np.deg2rad(lat_v)).astype(np.float32)
    odyv = np.full(j0 - 1, 1.0 / dy, np.float32)
    dz = 4000.0 * np.linspace(1.0, 3.0, k1) / np.linspace(1.0, 3.0, k1).sum()
    odz = (1.0 / dz).astype(np.float32)
    ztop = np.concatenate([[0.0], np.cumsum(dz)[:-1]])
    depth, _, _ = global_depth(nx, ny, seed)
    dpad = np.zeros((j0, i0))
    dpad[1:-1, 1:-1] = depth
    dpad[:, 0], dpad[:, -1] = dpad[:, -2], dpad[:, 1]          # periodic ghost columns
    wet = np.stack([dpad > ztop[k] + 1.0 for k in range(k1)])  # (K1, J0, I0)
    wet[0] = dpad > 0.0
    iu = np.zeros((k1, j0, i0), np.int16)
    iu[:, :, :-1] = (wet[:, :, :-1] & wet[:, :, 1:])
    iv = (wet[:, :-1, :] & wet[:, 1:, :]).astype(np.int16)
    iu0, iv0 = iu[0].copy(), np.zeros((j0, i0), np.int16)
    iv0[:-1] = iv[0]
    u = (speed * rng.standard_normal((k1, j0, i0))).astype(np.float32)
    v = (speed * rng.standard_normal((k1, j0 - 1, i0))).astype(np.float32)
    p0 = np.zeros((j0, i0), np.float32)
    scr = np.zeros((4, j0, i0), np.float32)
    # face coefficients, one value per face, so the operator is exactly symmetric
    w_row = (1.0 / (ocs[1:-1].astype(np.float64) * ody[1:-1]))  # rscale, J = 2..J1
    hx = np.einsum("k,kji->ji", dz, np.where(np.arange(k1)[:, None, None] == 0, 1, iu))
    hy = np.einsum("k,kji->ji", dz, np.where(np.arange(k1)[:, None, None] == 0, 1, iv))
    cx = (hx[1:-1, :] * (odx[1:-1, None].astype(np.float64) ** 2) * w_row[:, None]).astype(np.float32)
    cy = (hy * (csv[:, None].astype(np.float64) * odyv[:, None])).astype(np.float32)
    ar = cx[:, 1:-1].copy()            # face east of cell I = 2..I1
    al = cx[:, 0:-2].copy()            # face west of cell I (periodic through the ghost)
    at = cy[1:, 1:-1].copy()
    ab = cy[:-1, 1:-1].copy()
    at[-1] = 0.0                       # closed north and south edges
    ab[0] = 0.0
    gamma = 1.0 / (9.81 * dt * dt)
    ac = (-(al.astype(np.float64) + ar + ab + at) - gamma * w_row[:, None]).astype(np.float32)
    prob = Problem(al, ab, ac, ar, at, np.zeros((j2, i2)), periodic=True, name=f"fs{nx}x{ny}x{k1}",
                   meta=dict(gamma=gamma))
    return FSState(u, v, p0, scr, iu0, iv0, iu, iv, odx, ody, ocs, csv, odyv, odz, np.float32(1.0 / dt),
                   prob, w_row.astype(np.float32))


def stack(members) -> Problem:
    """Members of one grid size stacked along y into one block-diagonal
    problem.  Each member's north and south edge faces are closed (AT of its
    last row and AB of its first row are zero), so no equation couples two
    members; each row stays periodic in x with itself."""
    ny, nx = members[0].ny, members[0].nx
    for m in members:
        if (m.ny, m.nx) != (ny, nx) or m.periodic != members[0].periodic:
            raise ValueError("members must share grid size and periodicity")
        if np.any(m.at[-1] != 0) or np.any(m.ab[0] != 0):
            raise ValueError("member edges must be closed (AT of the last row, AB of the first)")
    cat = lambda k: np.ascontiguousarray(np.concatenate([getattr(m, k) for m in members], axis=0))
    return Problem(cat("al"), cat("ab"), cat("ac"), cat("ar"), cat("at"), cat("b"),
                   periodic=members[0].periodic, name=f"stack{len(members)}x{nx}x{ny}",
                   meta=dict(members=len(members), member_ny=ny))


def idealised(i2: int = 180, j2: int = 90) -> Problem:
    """The reference's test stencil (``P/prep_GLOBAL.f90:246-261``):
    AL=AB=AR=AT=-0.25, AC=1, Neumann rows on the north and south edges,
    periodic in x.  Rows sum to zero, so constants span the null space."""
    al = np.full((j2, i2), -0.25, np.float32)
    ab = al.copy()
    ar = al.copy()
    at = al.copy()
    ac = np.ones((j2, i2), np.float32)
    ac[-1] += at[-1]
    at[-1] = 0.0
    ac[0] += ab[0]
    ab[0] = 0.0
    b = np.zeros((j2, i2))
    return Problem(al, ab, ac, ar, at, b, periodic=True, name=f"idealised{i2}x{j2}")


def prep_assemble(i2, j2, k1, odx, ody, csv, ocs, odyv, odz, iu, iv, nbir, gamma):
    """PREP's coefficient assembly (``P/prep_GLOBAL.f90:170-244``, the 3-D
    branch, without the idealised override of :246-261), in float32 with the
    reference's order of operations.

    Metric arrays are indexed by the Fortran row J = 1..J0 at position J-1;
    ``iu``, ``iv`` are integer masks of shape (K0, J0, I0) (C order of the
    Fortran (I0, J0, K0) arrays).  Returns AL, AB, AC, AR, AT of shape
    (J2, I2).  Row J of AB and AT carries OCS(J+1) ODY(J+1), so the operator
    is symmetric only after each row is divided by that factor.
    """
    f = np.float32
    odx, ody, csv, ocs, odyv, odz = (np.asarray(a, f) for a in (odx, ody, csv, ocs, odyv, odz))
    J = np.arange(1, j2 + 1)  # Fortran rows 1..J2
    al = np.zeros((j2, i2), f)
    ar = np.zeros((j2, i2), f)
    ab = np.zeros((j2, i2), f)
    at = np.zeros((j2, i2), f)
    for k in range(1, k1 + 1):
        tmp = f(1.0) / odz[k - 1]
        dzx = (odx[J] * odx[J]) * tmp
        dzyb = (((csv[J - 1] * ocs[J]) * odyv[J - 1]) * ody[J]) * tmp
        dzyt = (((csv[J] * ocs[J]) * odyv[J]) * ody[J]) * tmp
        if k == 1:  # top layer all water (:184-196)
            al[:] = dzx[:, None]
            ar[:] = dzx[:, None]
            ab[:] = dzyb[:, None]
            at[:] = dzyt[:, None]
            continue
        uk = iu[k - 1].astype(f)
        vk = iv[k - 1].astype(f)
        al += dzx[:, None] * uk[1:j2 + 1, 0:i2]
        ar += dzx[:, None] * uk[1:j2 + 1, 1:i2 + 1]
        ab += dzyb[:, None] * vk[0:j2, 1:i2 + 1]
        at += dzyt[:, None] * vk[1:j2 + 1, 1:i2 + 1]
    if nbir == 1:
        al[:, 0] = 0.0
        ar[:, i2 - 1] = 0.0
    ab[0, :] = 0.0
    at[j2 - 1, :] = 0.0
    if nbir == 1 and j2 >= 2:
        ab[0, i2 // 2 - 1] = ab[1, i2 // 2 - 1]  # pin down pressure (:228-230)
    ac = (((-al - ar) - ab) - at) - f(gamma)
    return al, ab, ac, ar, at


def prep_grid(i2: int = 180, j2: int = 90, k1: int = 6, seed: int = 0, periodic: bool = True,
              dt: float = 900.0, lat_max: float = 78.0) -> Problem:
    """PREP-layout problem in the reference's CGS units: spherical metrics of
    a global grid (R = 6.4e8 cm, lat in [-lat_max, lat_max]), k1 layers with
    seeded land masks below the all-water top layer, FLAG_FS free surface
    (GAMMA = 1 / (0.5 DT^2 G), G = 980), assembled by ``prep_assemble``
    (nonsymmetric, as PREP writes it).  NBIR = 2 keeps the rows periodic in x;
    periodic=False uses NBIR = 1 (closed side walls and the pressure pin).
    The right-hand side is REAL*4 noise of the size of the coefficients."""
    rng = np.random.default_rng(seed)
    i0, j0 = i2 + 2, j2 + 2
    r0 = 6.4e8
    dlat = np.deg2rad(2.0 * lat_max / j2)
    lat_t = np.deg2rad(-lat_max) + (np.arange(j0) - 0.5) * dlat  # T rows, J = 1..J0
    lat_v = lat_t + 0.5 * dlat                                    # V rows
    dlon = 2.0 * np.pi / i2
    cs = np.cos(lat_t)
    csv = np.cos(lat_v)
    odx = 1.0 / (r0 * cs * dlon)
    ody = np.full(j0, 1.0 / (r0 * dlat))
    ocs = 1.0 / cs
    odyv = ody.copy()
    dz = np.sort(rng.uniform(1e3, 5e4, k1))
    odz = 1.0 / dz
    # wet layers per column from a smooth random field; masks of the deeper
    # layers (the top layer is all water in PREP's assembly)
    kb = np.clip(np.rint(k1 * (0.6 + 0.5 * smooth_field(j0, i0, 6.0, rng))), 1, k1)
    if periodic:
        kb[:, 0] = kb[:, i2]
        kb[:, i2 + 1] = kb[:, 1]
    iu = np.zeros((k1 + 1, j0, i0), np.int32)
    iv = np.zeros((k1 + 1, j0, i0), np.int32)
    for k in range(1, k1 + 1):
        wet = kb >= k
        iu[k - 1, :, 1:] = wet[:, 1:] & wet[:, :-1]
        iu[k - 1, :, 0] = wet[:, 0]
        iv[k - 1, 1:, :] = wet[1:, :] & wet[:-1, :]
        iv[k - 1, 0, :] = wet[0, :]
        if periodic:
            iu[k - 1, :, 0] = iu[k - 1, :, i2]
    gamma = 1.0 / (0.5 * dt * dt * 980.0)
    nbir = 2 if periodic else 1
    metrics = dict(odx=odx.astype(np.float32), ody=ody.astype(np.float32),
                   csv=csv.astype(np.float32), ocs=ocs.astype(np.float32),
                   odyv=odyv.astype(np.float32), odz=odz.astype(np.float32))
    al, ab, ac, ar, at = prep_assemble(i2, j2, k1, metrics["odx"], metrics["ody"], metrics["csv"],
                                       metrics["ocs"], metrics["odyv"], metrics["odz"], iu, iv,
                                       nbir, gamma)
    scale = float(np.abs(ac).mean())
    b = (rng.standard_normal((j2, i2)) * scale).astype(np.float32).astype(np.float64)
    return Problem(al, ab, ac, ar, at, b, periodic=periodic, name=f"prep{i2}x{j2}",
                   meta=dict(k1=k1, iu=iu, iv=iv, gamma=np.float32(gamma), nbir=nbir, **metrics))


def apply_operator(p: Problem, x: np.ndarray) -> np.ndarray:
    """y = A x in float64 on the unpadded grid (zero outside, periodic in x)."""
    xs = np.zeros_like(x)
    xs[1:] = x[:-1]
    xn = np.zeros_like(x)
    xn[:-1] = x[1:]
    if p.periodic:
        xw = np.roll(x, 1, axis=1)
        xe = np.roll(x, -1, axis=1)
    else:
        xw = np.zeros_like(x)
        xw[:, 1:] = x[:, :-1]
        xe = np.zeros_like(x)
        xe[:, :-1] = x[:, 1:]
    f64 = np.float64
    return (p.ab.astype(f64) * xs + p.al.astype(f64) * xw + p.ac.astype(f64) * x
            + p.ar.astype(f64) * xe + p.at.astype(f64) * xn)


def sparse_matrix(p: Problem):
    """scipy CSR matrix of the operator (for independent direct solves)."""
    import scipy.sparse as sp

    ny, nx = p.ny, p.nx
    n = nx * ny
    idx = np.arange(n).reshape(ny, nx)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [p.ac.astype(np.float64).ravel()]
    # south / north
    rows.append(idx[1:].ravel()); cols.append(idx[:-1].ravel()); vals.append(p.ab[1:].astype(np.float64).ravel())
    rows.append(idx[:-1].ravel()); cols.append(idx[1:].ravel()); vals.append(p.at[:-1].astype(np.float64).ravel())
    # west / east
    if p.periodic:
        rows.append(idx.ravel()); cols.append(np.roll(idx, 1, axis=1).ravel()); vals.append(p.al.astype(np.float64).ravel())
        rows.append(idx.ravel()); cols.append(np.roll(idx, -1, axis=1).ravel()); vals.append(p.ar.astype(np.float64).ravel())
    else:
        rows.append(idx[:, 1:].ravel()); cols.append(idx[:, :-1].ravel()); vals.append(p.al[:, 1:].astype(np.float64).ravel())
        rows.append(idx[:, :-1].ravel()); cols.append(idx[:, 1:].ravel()); vals.append(p.ar[:, :-1].astype(np.float64).ravel())
    r = np.concatenate(rows); c = np.concatenate(cols); v = np.concatenate(vals)
    return sp.csr_matrix((v, (r, c)), shape=(n, n))
