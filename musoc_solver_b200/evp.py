"""EVP influence files: write and read the record that carries the SEVP
operator and its influence matrices from PREP to MAIN (``sevp_evp_write`` /
``sevp_evp_read`` of ``libsevp_b200.so``; the format is described in
``include/sevp_b200.h``).

Arrays are numpy arrays in the reference's memory order: a (I2, J2) Fortran
plane is a C-order (J2, I2) array, RINV (I2, I2, NB0) a C-order
(NB0, I2, I2) array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def write(path, al, ar, ab, at, ac, rinv, rinv1, ie, oac=None, max_subrecord=None):
    """Writes PREP's record (MAIN's, with OAC, when oac is given)."""
    planes = [_f32(a) for a in (al, ar, ab, at, ac)]
    j2, i2 = planes[0].shape
    oac = None if oac is None else _f32(oac)
    rinv = np.ascontiguousarray(rinv, np.float64)
    rinv1 = np.ascontiguousarray(rinv1, np.float64)
    ie = np.ascontiguousarray(ie, np.int32)
    args = [str(path).encode(), i2, j2] + [N.ptr(a) for a in planes] + [
        N.ptr(oac) if oac is not None else None, N.ptr(rinv), rinv.size, N.ptr(rinv1), rinv1.size,
        N.ptr(ie), ie.size]
    if max_subrecord is None:
        s = N.lib().sevp_evp_write(*args)
    else:
        s = N.lib().sevp_evp_write_sub(*args, int(max_subrecord))
    N.check(s, "sevp_evp_write")


def read(path, i2, j2, rinv_shape, rinv1_shape, nb0):
    """Reads a record written by PREP or by ``write``; returns a dict with
    al, ar, ab, at, ac, rinv, rinv1, ie and oac (None when the file has no
    OAC plane)."""
    planes = [np.zeros((j2, i2), np.float32) for _ in range(6)]
    rinv = np.zeros(rinv_shape, np.float64)
    rinv1 = np.zeros(rinv1_shape, np.float64)
    ie = np.zeros(nb0, np.int32)
    has = C.c_int(-1)
    s = N.lib().sevp_evp_read(str(path).encode(), i2, j2, *[N.ptr(a) for a in planes], N.ptr(rinv),
                              rinv.size, N.ptr(rinv1), rinv1.size, N.ptr(ie), nb0, C.byref(has))
    N.check(s, "sevp_evp_read")
    names = ("al", "ar", "ab", "at", "ac")
    out = {k: v for k, v in zip(names, planes[:5])}
    out.update(rinv=rinv, rinv1=rinv1, ie=ie, oac=planes[5] if has.value else None)
    return out
