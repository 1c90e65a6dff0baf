"""Test helper: MDBas's init_ewald / ewald_rec / ewald_free (src/ewald.c) of a
library (MDBas's own in oracle/_ref, or the drop-in) through ctypes."""
from __future__ import annotations

import ctypes as C

import numpy as np

from mdbas_b200 import nb


def _bind(lib):
    lib.init_ewald.argtypes = [C.POINTER(nb.CTRL), C.POINTER(nb.PARAM), C.POINTER(nb.EWALD),
                               C.POINTER(nb.PBC)]
    lib.init_ewald.restype = None
    lib.ewald_free.argtypes = [C.POINTER(nb.EWALD)]
    lib.ewald_free.restype = None
    lib.ewald_rec.argtypes = [C.POINTER(nb.PARAM), C.POINTER(nb.EWALD), C.POINTER(nb.PBC)] + [
        C.c_void_p] * 7 + [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.ewald_rec.restype = C.c_double
    return lib


def init(lib, sysm, prec=1e-6, alpha=None, mmax=None, cutOff=12.0, cell=None,
         box_type=nb.CUBIC):
    """init_ewald of `lib`: the EWALD struct it fills."""
    _bind(lib)
    ctrl = nb.CTRL()
    ctrl.keyAlpha = 0 if alpha is None else 1
    ctrl.keyMmax = 0 if mmax is None else 1
    param = nb.make_param(sysm.n, cutOff=cutOff)
    ew = nb.EWALD()
    ew.prec = prec
    if alpha is not None:
        ew.alpha = alpha
    if mmax is not None:
        ew.m1max, ew.m2max, ew.m3max = mmax
    pbc = nb.make_pbc(sysm.cell() if cell is None else cell, box_type)
    lib.init_ewald(C.byref(ctrl), C.byref(param), C.byref(ew), C.byref(pbc))
    return ew


def rec(lib, sysm, ew, forces=None, cell=None, box_type=nb.CUBIC):
    """ewald_rec of `lib` after its init_ewald: (energy, fx, fy, fz, virial,
    stress); forces start from copies of `forces` (or zeros)."""
    _bind(lib)
    param = nb.make_param(sysm.n)
    pbc = nb.make_pbc(sysm.cell() if cell is None else cell, box_type)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (sysm.x, sysm.y, sysm.z, sysm.q)]
    f = ([np.zeros(sysm.n) for _ in range(3)] if forces is None
         else [np.array(a, dtype=np.float64) for a in forces])
    stress = (C.c_double * 6)()
    vir = C.c_double(0.0)
    e = lib.ewald_rec(C.byref(param), C.byref(ew), C.byref(pbc),
                      *(a.ctypes.data_as(C.c_void_p) for a in arrs[:3]),
                      *(a.ctypes.data_as(C.c_void_p) for a in f),
                      arrs[3].ctypes.data_as(C.c_void_p), stress, C.byref(vir))
    return e, f[0], f[1], f[2], vir.value, list(stress)
