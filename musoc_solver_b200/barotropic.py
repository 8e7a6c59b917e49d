"""Barotropic pressure correction of FS (the ITMASK loop around the solve,
M/fs_GLOBAL.f90:1154-1283) on the GPU.

Each pass: zero the top-layer velocity on land faces; form the free-surface
right-hand side S from continuity; solve A X = S with the tile-SEVP PCG;
add ODT X to the surface pressure P0 and correct U and V in every layer; stop
when the largest top-layer land velocity is <= tolerance or after mxmask
passes.  The kernels (``sevp_fs_*`` in ``libsevp_b200.so``) follow the
reference's REAL*4 / REAL*8 arithmetic; ``problems.fs_state`` makes a
seeded layered state with a consistent symmetric operator.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .solver import SevpSolver


class BarotropicCorrection:
    """Device copies of a state's masks and metrics, a solver for its
    operator, and the loop's scratch."""

    def __init__(self, state, tile_m=16, tile_h=8, device="cuda", schwarz=False):
        import torch

        self.torch = torch
        self.st = state
        self.i0, self.j0, self.k0 = state.dims
        self.solver = SevpSolver(state.problem, tile_m=tile_m, tile_h=tile_h, device=device,
                                 schwarz=schwarz)
        dev = self.solver.device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.d = {k: t(getattr(state, k)) for k in ("iu0", "iv0", "iu", "iv", "odx", "ody", "ocs",
                                                     "csv", "odyv", "odz", "rscale")}
        n = (self.i0 - 2) * (self.j0 - 2)
        self.b = torch.zeros(n, dtype=torch.float64, device=dev)
        self.x = torch.zeros(n, dtype=torch.float64, device=dev)
        self.vmax = torch.zeros(1, dtype=torch.float32, device=dev)
        self.sp = C.c_void_p(self.solver.stream.cuda_stream)

    def upload(self):
        """Device copies of the state's u, v, p0, scr."""
        t = lambda a: self.torch.from_numpy(np.ascontiguousarray(a)).to(self.solver.device)
        return t(self.st.u), t(self.st.v), t(self.st.p0), t(self.st.scr)

    # single steps (the loop's pieces)
    def mask(self, u, v, periodic=True):
        d = self.d
        N.check(N.lib().sevp_fs_mask(self.i0, self.j0, N.ptr(u), N.ptr(v), N.ptr(d["iu0"]),
                                     N.ptr(d["iv0"]), int(periodic), self.sp), "sevp_fs_mask")

    def rhs(self, u, v, s=None, b=None, scaled=True):
        d = self.d
        N.check(N.lib().sevp_fs_rhs(self.i0, self.j0, self.k0, N.ptr(u), N.ptr(v), N.ptr(d["odx"]),
                                    N.ptr(d["ody"]), N.ptr(d["ocs"]), N.ptr(d["csv"]),
                                    N.ptr(d["odz"]), N.ptr(d["rscale"]) if scaled else None,
                                    N.ptr(s) if s is not None else None,
                                    N.ptr(b) if b is not None else None, self.sp), "sevp_fs_rhs")

    def correct(self, x, u, v, p0, scr, periodic=True):
        d = self.d
        N.check(N.lib().sevp_fs_correct(self.i0, self.j0, self.k0, N.ptr(x), float(self.st.odt),
                                        N.ptr(d["odx"]), N.ptr(d["odyv"]), N.ptr(d["iu"]),
                                        N.ptr(d["iv"]), N.ptr(d["iu0"]), N.ptr(d["iv0"]),
                                        N.ptr(p0), N.ptr(u), N.ptr(v), N.ptr(scr), int(periodic),
                                        N.ptr(self.vmax), self.sp), "sevp_fs_correct")
        return float(self.vmax.item())

    def run(self, u, v, p0, scr, tolerance=1e-3, mxmask=18, precision=1, tol=1e-12,
            periodic=True, inner_tol=1e-5):
        """The whole loop; returns (passes, final land velocity, PCG iterations)."""
        d = self.d
        o = self.solver.opts(precision, tol, inner_tol=inner_tol)
        it, vm, iters = C.c_int(), C.c_float(), C.c_int()
        s = N.lib().sevp_fs_barotropic(
            self.solver.h, self.i0, self.j0, self.k0, N.ptr(u), N.ptr(v), N.ptr(p0), N.ptr(scr),
            N.ptr(d["iu0"]), N.ptr(d["iv0"]), N.ptr(d["iu"]), N.ptr(d["iv"]), N.ptr(d["odx"]),
            N.ptr(d["ody"]), N.ptr(d["ocs"]), N.ptr(d["csv"]), N.ptr(d["odyv"]), N.ptr(d["odz"]),
            N.ptr(d["rscale"]), float(self.st.odt), int(periodic), float(tolerance), int(mxmask),
            C.byref(o), N.ptr(self.b), N.ptr(self.x), N.ptr(self.vmax), C.byref(it), C.byref(vm),
            C.byref(iters))
        if s not in (N.SEVP_OK, N.SEVP_MAXITER):
            raise N.SevpError(s, "sevp_fs_barotropic")
        return it.value, vm.value, iters.value

    def close(self):
        self.solver.close()
