"""Test helper: MDBas's own file routines (src/io.c, compiled into oracle/_ref)
through ctypes, for parity with mdbas_b200.mdbas_files."""
from __future__ import annotations

import ctypes as C

import numpy as np

from mdbas_b200 import nb

FINAMELEN = 512  # include/global.h:61


class IO(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("confFile", "forfFile", "propFile", "restFile",
                                          "rconFile", "trajFile", "simuFile")] + [
        (n, C.c_char * FINAMELEN) for n in ("confName", "forfName", "propName", "restName",
                                            "rconName", "trajName", "simuName")]


class ATOM(C.Structure):
    _fields_ = [("label", C.c_char * 5), ("segn", C.c_char * 5), ("resn", C.c_char * 5),
                ("type", C.c_int), ("resi", C.c_int), ("ires", C.c_int)]


class BATH(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("tauT", "chiT", "tauP", "chiP", "compress")]


_dpp = C.POINTER(C.POINTER(C.c_double))


def bind(lib):
    lib.read_SIMU.argtypes = [C.POINTER(IO), C.POINTER(nb.CTRL), C.POINTER(nb.PARAM),
                              C.POINTER(BATH), C.POINTER(nb.NEIGH), C.POINTER(nb.EWALD),
                              C.POINTER(nb.PBC)]
    lib.read_CONF.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(C.POINTER(ATOM)),
                              _dpp, _dpp, _dpp]
    lib.read_FORF.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(ATOM),
                              C.POINTER(C.POINTER(nb.CONSTRAINT)), C.POINTER(C.POINTER(nb.BOND)),
                              C.POINTER(C.POINTER(nb.ANGLE)), C.POINTER(C.POINTER(nb.DIHE)),
                              C.POINTER(C.POINTER(nb.DIHE)), C.POINTER(C.POINTER(nb.BOND))] + [
        C.c_void_p] * 8
    lib.write_CONF.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(ATOM)] + [
        C.c_void_p] * 3
    lib.write_rest.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(nb.ENERGY),
                               C.POINTER(BATH), C.POINTER(ATOM)] + [C.c_void_p] * 9
    lib.read_rest.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(nb.ENERGY),
                              C.POINTER(BATH), C.POINTER(C.POINTER(ATOM))] + [_dpp] * 9
    lib.write_prop.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(nb.ENERGY),
                               C.POINTER(nb.PBC)]
    lib.write_DCD_header.argtypes = [C.POINTER(IO), C.POINTER(nb.CTRL), C.POINTER(nb.PARAM),
                                     C.POINTER(nb.PBC), C.c_void_p]
    lib.write_DCD_traj.argtypes = [C.POINTER(IO), C.POINTER(nb.PARAM), C.POINTER(nb.PBC)] + [
        C.c_void_p] * 4
    for f in ("read_SIMU", "read_CONF", "read_FORF", "write_CONF", "write_rest", "read_rest",
              "write_prop", "write_DCD_header", "write_DCD_traj"):
        getattr(lib, f).restype = None
    return lib


def io_with(**names) -> IO:
    io = IO()
    for k, v in names.items():
        setattr(io, f"{k}Name", str(v).encode())
    return io


def struct_dict(s) -> dict:
    return {name: getattr(s, name) for name, _ in s._fields_}


def arr(p, n) -> np.ndarray:
    return np.ctypeslib.as_array(p, shape=(n,)).copy()
