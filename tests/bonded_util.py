"""Test helper: MDBas's own bonded routines (src/internal.c, compiled into
oracle/_ref) called through ctypes with the mirrored MDBas structs."""
from __future__ import annotations

import ctypes as C

import numpy as np

from mdbas_b200 import nb

# MDBas routine per kind (the order of mdbas_b200.nb.BONDED_KINDS)
ROUTINES = ("bond_energy", "angle_energy", "ub_energy", "dihedral_energy", "improper_energy")
# PARAM count field and ENERGY fields (energy, virial) per kind
COUNTS = ("nBond", "nAngle", "nUb", "nDihedral", "nImproper")
FIELDS = (("bond", "virbond"), ("ang", None), ("ub", "virub"), ("dihe", None), ("impr", None))


def _bind(lib):
    for name in ROUTINES:
        fn = getattr(lib, name)
        fn.argtypes = [C.POINTER(nb.PARAM), C.POINTER(nb.ENERGY), C.POINTER(nb.PBC),
                       C.c_void_p] + [C.c_void_p] * 6
        fn.restype = None
    return lib


def call(lib, kind: int, sysm, structs, forces=None, cell=None, box_type=nb.CUBIC):
    """One MDBas bonded routine of `lib` (MDBas's own or the drop-in): returns
    (energy, virial, fx, fy, fz) with the forces added to copies of
    `forces` (or to zeros)."""
    _bind(lib)
    n = sysm.n
    param = nb.make_param(n)
    m, arr = structs[kind]
    setattr(param, COUNTS[kind], m)
    ener = nb.ENERGY()
    pbc = nb.make_pbc(sysm.cell() if cell is None else cell, box_type)
    pos = [np.ascontiguousarray(a, dtype=np.float64) for a in (sysm.x, sysm.y, sysm.z)]
    f = ([np.zeros(n) for _ in range(3)] if forces is None
         else [np.array(a, dtype=np.float64) for a in forces])
    getattr(lib, ROUTINES[kind])(C.byref(param), C.byref(ener), C.byref(pbc),
                                 C.cast(arr, C.c_void_p),
                                 *(a.ctypes.data_as(C.c_void_p) for a in pos),
                                 *(a.ctypes.data_as(C.c_void_p) for a in f))
    e_field, v_field = FIELDS[kind]
    return (getattr(ener, e_field), getattr(ener, v_field) if v_field else 0.0,
            f[0], f[1], f[2])
