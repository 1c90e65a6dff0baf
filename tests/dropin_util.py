"""Test helper: one MDBas system driven through the drop-in C ABI (ctypes)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from mdbas_b200 import nb

_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


class DropinSystem:
    """MDBas structs + caller-owned arrays for one generated system."""

    def __init__(self, sysm, linkRatio=1, noLink=0, frozen=None, keyEwald=3, alpha=0.34,
                 cutOff=12.0, cutOn=10.0, delr=2.0, cell=None, box_type=nb.CUBIC):
        self.L = nb.bind_dropin()
        self.s = sysm
        n = sysm.n
        self.n = n
        self.ctrl = nb.CTRL()
        self.ctrl.newjob = 1
        self.ctrl.noLink = noLink
        self.ctrl.keyEwald = keyEwald
        self.ctrl.elecType = nb.FULL
        self.ctrl.vdwType = nb.VSWITCH
        self.param = nb.make_param(n, cutOff, cutOn, delr)
        self.param.nBond = len(sysm.bonds)
        self.param.nAngle = len(sysm.angles)
        self.box = nb.make_pbc(sysm.cell() if cell is None else cell, box_type)
        self.neigh = nb.NEIGH()
        self.neigh.update = 1
        self.neigh.linkRatio = linkRatio
        self.ewald = nb.EWALD()
        self.ewald.alpha = alpha
        self.ener = nb.ENERGY()
        self.bond = (nb.BOND * max(1, len(sysm.bonds)))()
        for k, (a, b) in enumerate(sysm.bonds.tolist()):
            self.bond[k].a, self.bond[k].b = a, b
        self.angle = (nb.ANGLE * max(1, len(sysm.angles)))()
        for k, (a, b, c) in enumerate(sysm.angles.tolist()):
            self.angle[k].a, self.angle[k].b, self.angle[k].c = a, b, c
        self.const = (nb.CONSTRAINT * 1)()
        self.dihe = (nb.DIHE * 1)()
        self.impr = (nb.DIHE * 1)()
        self.x = np.ascontiguousarray(sysm.x, dtype=np.float64).copy()
        self.y = np.ascontiguousarray(sysm.y, dtype=np.float64).copy()
        self.z = np.ascontiguousarray(sysm.z, dtype=np.float64).copy()
        self.q = np.ascontiguousarray(sysm.q, dtype=np.float64)
        self.eps = np.ascontiguousarray(sysm.eps, dtype=np.float64)
        self.sig = np.ascontiguousarray(sysm.sig, dtype=np.float64)
        self.frozen = (np.zeros(n, np.int32) if frozen is None
                       else np.ascontiguousarray(frozen, dtype=np.int32))
        self.param.nFrozen = int((self.frozen != 0).sum())
        self.vx, self.vy, self.vz = np.zeros(n), np.zeros(n), np.zeros(n)
        self.fx, self.fy, self.fz = np.zeros(n), np.zeros(n), np.zeros(n)
        self.neighList = C.POINTER(C.c_int)()
        self.neighPair = C.POINTER(C.c_int)()
        self.neighOrder = C.POINTER(C.c_int)()
        self.neighList14 = C.POINTER(C.c_int)()
        self.exclList = C.POINTER(C.POINTER(C.c_int))()
        self.exclPair = C.POINTER(C.c_int)()
        self.built = False

    def makelist(self):
        L = self.L
        L.makelist(C.byref(self.ctrl), C.byref(self.param), C.byref(self.box),
                   C.byref(self.neigh), self.const, self.bond, self.angle, self.dihe, self.impr,
                   nb.as_dp(self.x), nb.as_dp(self.y), nb.as_dp(self.z), nb.as_ip(self.frozen),
                   C.byref(self.neighList), C.byref(self.neighPair), C.byref(self.neighOrder),
                   C.byref(self.neighList14), C.byref(self.exclList), C.byref(self.exclPair))
        self.built = True
        return self.ctrl.keyLink

    def update(self, x, y, z):
        self.x[:] = x
        self.y[:] = y
        self.z[:] = z
        self.param.step = 0
        self.makelist()

    def get_list(self):
        n = self.n
        pair = np.ctypeslib.as_array(self.neighPair, (n,)).copy()
        order = np.ctypeslib.as_array(self.neighOrder, (n,)).copy()
        tot = int(pair.sum())
        lst = (np.ctypeslib.as_array(self.neighList, (tot,)).copy() if tot
               else np.zeros(0, np.int32))
        return lst, pair, order

    def get_excl(self):
        n = self.n
        pair = np.ctypeslib.as_array(self.exclPair, (n,)).copy()
        rows = []
        for i in range(n):
            rows.extend(self.exclList[i][k] for k in range(pair[i]))
        start = np.zeros(n + 1, np.int32)
        start[1:] = np.cumsum(pair)
        return start, np.array(rows, np.int32)

    def energy(self):
        L = self.L
        L.init_energy_ptrs(C.byref(self.ctrl))
        p = nb.PARAM.from_buffer_copy(self.param)
        p.nBond = 0
        p.nAngle = 0
        L.energy(C.byref(self.ctrl), C.byref(p), C.byref(self.ener), C.byref(self.ewald),
                 C.byref(self.box), C.byref(self.neigh), self.bond, self.bond, self.angle,
                 self.dihe, self.impr, nb.as_dp(self.x), nb.as_dp(self.y), nb.as_dp(self.z),
                 nb.as_dp(self.vx), nb.as_dp(self.vy), nb.as_dp(self.vz), nb.as_dp(self.fx),
                 nb.as_dp(self.fy), nb.as_dp(self.fz), nb.as_dp(self.q), nb.as_dp(self.eps),
                 nb.as_dp(self.sig), nb.as_dp(self.eps), nb.as_dp(self.sig),
                 nb.as_ip(self.frozen), self.neighList, self.neighPair, self.neighOrder,
                 self.neighList14, self.exclList, self.exclPair)
        e = self.ener
        return (self.fx.copy(), self.fy.copy(), self.fz.copy(),
                dict(elec=e.elec, vdw=e.vdw, virelec=e.virelec, virvdw=e.virvdw, pot=e.pot,
                     virpot=e.virpot))

    def free(self):
        if not self.built:
            return
        for p in (self.neighList, self.neighPair, self.neighOrder, self.neighList14):
            _libc.free(C.cast(p, C.c_void_p))
        rows = self.n if self.ctrl.keyLink else self.n - 1
        for i in range(rows):
            _libc.free(C.cast(self.exclList[i], C.c_void_p))
        _libc.free(C.cast(self.exclList, C.c_void_p))
        _libc.free(C.cast(self.exclPair, C.c_void_p))
        self.built = False


def force_rel_rms(f, r):
    fx, fy, fz = f
    rx, ry, rz = r
    num = ((fx - rx) ** 2 + (fy - ry) ** 2 + (fz - rz) ** 2).sum()
    den = (rx ** 2 + ry ** 2 + rz ** 2).sum()
    return float(np.sqrt(num / den))
