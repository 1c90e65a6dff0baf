"""CPU checkers for the nonbonded hot path -- TEST INFRASTRUCTURE ONLY.

Two shared libraries, built by ``make -C oracle``:

* ``_build/liboracle.so``: the repository's own C restatement of MDBas's
  list builders and pair loops (mdbas_oracle.c, bit-exact with MDBas);
* ``_ref/libmdbas_ref.so``: MDBas itself compiled from its own sources, with
  a harness in place of its driver (ref_harness.c).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this package, always as the checker or the CPU baseline; the product
library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmdbas_ref.so")
ORC_BOX_LEN = 23

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(ref: str | None = None) -> None:
    """Compile the restatement and, when the MDBas sources are present, the
    reference library (make -C oracle)."""
    cmd = ["make", "-s", "-C", HERE]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


class OrcParam(C.Structure):
    _fields_ = [("chargeConst", C.c_double), ("alpha", C.c_double), ("cutOff", C.c_double),
                ("cutOn", C.c_double), ("cutOff2", C.c_double), ("cutOn2", C.c_double),
                ("rcutOff", C.c_double), ("rcutOff2", C.c_double), ("switch2", C.c_double),
                ("vdwSwitch", C.c_int), ("elecType", C.c_int)]


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """ctypes front of liboracle.so (the C restatement)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        self.lib = lib
        lib.orc_init_box.argtypes = [C.c_int, _dp, _dp]
        lib.orc_fill_param.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int, C.POINTER(OrcParam)]
        lib.orc_image_update.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        lib.orc_verlet_list.restype = C.c_long
        lib.orc_verlet_list.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double, _dp, _dp,
                                        _dp, C.c_void_p, _ip, _ip, _ip, _ip, C.c_void_p, C.c_long]
        lib.orc_link_cell_list.restype = C.c_long
        lib.orc_link_cell_list.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_int,
                                           _dp, _dp, _dp, C.c_void_p, _ip, _ip, _ip, _ip,
                                           C.c_void_p, C.c_long, C.POINTER(C.c_int)]
        lib.orc_link_cell_counts.restype = C.c_int
        lib.orc_link_cell_counts.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_int, _ip]
        lib.orc_ewald_energy.argtypes = [C.c_int, C.c_int, _dp, C.POINTER(OrcParam), _dp, _dp, _dp,
                                         _dp, _dp, _dp, _ip, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp]
        lib.orc_nonbond_energy.argtypes = [C.c_int, C.c_int, _dp, C.POINTER(OrcParam), _dp, _dp,
                                           _dp, _dp, _dp, _dp, _ip, _ip, _ip, _dp, _dp, _dp, _dp]
        lib.orc_self_energy.restype = C.c_double
        lib.orc_self_energy.argtypes = [C.c_int, _dp, C.c_double, C.c_double]
        lib.orc_pairs_within.restype = C.c_long
        lib.orc_pairs_within.argtypes = [C.c_int, C.c_int, _dp, C.c_double, _dp, _dp, _dp,
                                         C.c_void_p, _ip, _ip, C.c_void_p, C.c_long]
        lib.orc_forces_subset.restype = C.c_int
        lib.orc_forces_subset.argtypes = [C.c_int, C.c_int, _dp, C.POINTER(OrcParam), _dp, _dp,
                                          _dp, _dp, _dp, _dp, _ip, _ip, C.c_int, _ip, _dp, _dp,
                                          _dp]
        lib.orc_nint.restype = C.c_int
        lib.orc_nint.argtypes = [C.c_double]
        lib.orc_dist.restype = C.c_double
        lib.orc_dist.argtypes = [C.c_int, _dp, _dp]

    # -- setup -------------------------------------------------------------
    def box(self, cell, box_type: int = 1) -> np.ndarray:
        out = np.zeros(ORC_BOX_LEN)
        self.lib.orc_init_box(box_type, _d(cell), out)
        return out

    def param(self, cutOff=12.0, cutOn=10.0, alpha=0.34, chargeConst=None, vdwSwitch=1,
              elecType=1) -> OrcParam:
        from mdbas_b200.systems import CHARGE_CONST
        p = OrcParam()
        self.lib.orc_fill_param(cutOff, cutOn, alpha,
                                CHARGE_CONST if chargeConst is None else chargeConst,
                                vdwSwitch, elecType, C.byref(p))
        return p

    # -- lists ---------------------------------------------------------------
    def image_update(self, box, x, y, z, box_type: int = 1):
        x, y, z = _d(x).copy(), _d(y).copy(), _d(z).copy()
        self.lib.orc_image_update(box_type, box, len(x), x, y, z)
        return x, y, z

    def verlet_list(self, box, x, y, z, excl, cutOff=12.0, delr=2.0, frozen=None, box_type=1):
        n = len(x)
        start, flat = excl
        pair, order = np.zeros(n, np.int32), np.zeros(n, np.int32)
        fz = None if frozen is None else _i(frozen)
        fp = None if fz is None else fz.ctypes.data
        cnt = self.lib.orc_verlet_list(n, box_type, box, cutOff, delr, _d(x), _d(y), _d(z), fp,
                                       _i(start), _i(flat), pair, order, None, 0)
        lst = np.zeros(max(cnt, 1), np.int32)
        self.lib.orc_verlet_list(n, box_type, box, cutOff, delr, _d(x), _d(y), _d(z), fp,
                                 _i(start), _i(flat), pair, order, lst.ctypes.data, cnt)
        return lst[:cnt], pair, order

    def link_cell_counts(self, box, cutOff=12.0, delr=2.0, linkRatio=1, box_type=1):
        nlc = np.zeros(3, np.int32)
        ok = self.lib.orc_link_cell_counts(box_type, box, cutOff, delr, linkRatio, nlc)
        return ok, nlc

    def link_cell_list(self, box, x, y, z, excl, cutOff=12.0, delr=2.0, linkRatio=1,
                       frozen=None, box_type=1):
        n = len(x)
        start, flat = excl
        pair, order = np.zeros(n, np.int32), np.zeros(n, np.int32)
        fz = None if frozen is None else _i(frozen)
        fp = None if fz is None else fz.ctypes.data
        nc = C.c_int(0)
        args = (n, box_type, box, cutOff, delr, linkRatio, _d(x), _d(y), _d(z), fp, _i(start),
                _i(flat), pair, order)
        cnt = self.lib.orc_link_cell_list(*args, None, 0, C.byref(nc))
        if cnt < 0:
            raise ValueError("link-cell grid too small")
        lst = np.zeros(max(cnt, 1), np.int32)
        self.lib.orc_link_cell_list(*args, lst.ctypes.data, cnt, C.byref(nc))
        return lst[:cnt], pair, order

    # -- energies ------------------------------------------------------------
    def ewald_energy(self, box, sysm, lst, pair, order, excl, p=None, box_type=1, x=None,
                     y=None, z=None):
        p = p or self.param()
        n = sysm.n
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        out = np.zeros(8)
        xx = sysm.x if x is None else x
        yy = sysm.y if y is None else y
        zz = sysm.z if z is None else z
        self.lib.orc_ewald_energy(n, box_type, box, C.byref(p), _d(xx), _d(yy), _d(zz),
                                  _d(sysm.q), _d(sysm.eps), _d(sysm.sig), _i(lst), _i(pair),
                                  _i(order), _i(excl[0]), _i(excl[1]), fx, fy, fz, out)
        keys = ["e_dir", "e_corr", "e_vdw", "vir_dir", "vir_corr", "vir_vdw", "n_pairs"]
        return fx, fy, fz, dict(zip(keys, out.tolist()))

    def nonbond_energy(self, box, sysm, lst, pair, order, p, box_type=1):
        n = sysm.n
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        out = np.zeros(5)
        self.lib.orc_nonbond_energy(n, box_type, box, C.byref(p), _d(sysm.x), _d(sysm.y),
                                    _d(sysm.z), _d(sysm.q), _d(sysm.eps), _d(sysm.sig), _i(lst),
                                    _i(pair), _i(order), fx, fy, fz, out)
        return fx, fy, fz, dict(zip(["elec", "vdw", "virelec", "virvdw", "n_pairs"], out.tolist()))

    def self_energy(self, q, chargeConst, alpha):
        return self.lib.orc_self_energy(len(q), _d(q), chargeConst, alpha)

    def pairs_within(self, box, x, y, z, excl, r2max, frozen=None, box_type=1):
        n = len(x)
        fz = None if frozen is None else _i(frozen)
        fp = None if fz is None else fz.ctypes.data
        args = (n, box_type, box, r2max, _d(x), _d(y), _d(z), fp, _i(excl[0]), _i(excl[1]))
        cnt = self.lib.orc_pairs_within(*args, None, 0)
        out = np.zeros(2 * max(cnt, 1), np.int32)
        self.lib.orc_pairs_within(*args, out.ctypes.data, cnt)
        return out[:2 * cnt].reshape(-1, 2)

    def forces_subset(self, box, sysm, excl_sym, subset, p=None, box_type=1):
        p = p or self.param()
        subset = _i(subset)
        m = len(subset)
        fx, fy, fz = np.zeros(m), np.zeros(m), np.zeros(m)
        ok = self.lib.orc_forces_subset(sysm.n, box_type, box, C.byref(p), _d(sysm.x),
                                        _d(sysm.y), _d(sysm.z), _d(sysm.q), _d(sysm.eps),
                                        _d(sysm.sig), _i(excl_sym[0]), _i(excl_sym[1]), m, subset,
                                        fx, fy, fz)
        if not ok:
            raise ValueError("box too small for the cell search")
        return fx, fy, fz


class Reference:
    """One MDBas system held by libmdbas_ref.so (MDBas's own code)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(REF_SO)
            lib.ref_create.restype = C.c_void_p
            lib.ref_create.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                       C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp,
                                       C.c_void_p, C.c_int, _ip, C.c_int, _ip]
            lib.ref_box.argtypes = [C.c_void_p, _dp]
            lib.ref_makelist.restype = C.c_int
            lib.ref_makelist.argtypes = [C.c_void_p]
            lib.ref_update_list.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            for f in ("ref_key_link", "ref_n_cells", "ref_size_list"):
                getattr(lib, f).restype = C.c_int
                getattr(lib, f).argtypes = [C.c_void_p]
            for f in ("ref_list_entries", "ref_excl_entries"):
                getattr(lib, f).restype = C.c_long
                getattr(lib, f).argtypes = [C.c_void_p]
            lib.ref_get_list.argtypes = [C.c_void_p, _ip, _ip, _ip]
            lib.ref_list_ptrs.argtypes = [C.c_void_p] + [C.POINTER(C.POINTER(C.c_int))] * 3
            lib.ref_get_excl.argtypes = [C.c_void_p, _ip, _ip]
            lib.ref_get_positions.argtypes = [C.c_void_p, _dp, _dp, _dp]
            lib.ref_set_positions.argtypes = [C.c_void_p, _dp, _dp, _dp]
            lib.ref_energy.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
            lib.ref_self_energy.restype = C.c_double
            lib.ref_self_energy.argtypes = [C.c_void_p]
            lib.ref_set_torsions.argtypes = [C.c_void_p, C.c_int, _ip, C.c_int, _ip]
            lib.ref_n_pair14.restype = C.c_int
            lib.ref_n_pair14.argtypes = [C.c_void_p]
            lib.ref_get_list14.argtypes = [C.c_void_p, _ip]
            lib.ref_layout.restype = C.c_int
            lib.ref_layout.argtypes = [C.c_char_p, C.c_int]
            lib.ref_now.restype = C.c_double
            lib.ref_md_init.restype = C.c_int
            lib.ref_md_init.argtypes = [C.c_void_p, _dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_int, C.c_double, C.c_double]
            lib.ref_md_run.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.ref_get_velocities.argtypes = [C.c_void_p, _dp, _dp, _dp]
            lib.ref_ewald_rec.argtypes = [C.c_void_p, C.c_double, C.c_void_p, _dp, _dp, _dp,
                                          _dp]
            lib.ref_set_bonded.argtypes = [C.c_void_p] + [C.c_int, C.c_void_p] * 5
            lib.ref_set_kspace.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
            lib.ref_set_kspace.restype = C.c_int
            lib.ref_set_nonbond.argtypes = [C.c_void_p, C.c_int, C.c_int]
            lib.ref_set_nonbond.restype = C.c_int
            lib.ref_set_nb14.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_void_p]
            lib.ref_bonded_energies.argtypes = [C.c_void_p, _dp]
            lib.ref_destroy.argtypes = [C.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, sysm, cutOff=12.0, cutOn=10.0, delr=2.0, linkRatio=1, noLink=0,
                 alpha=0.34, frozen=None, box_type=1, cell=None):
        lib = self.lib()
        self.n = sysm.n
        self._keep = []
        cell = sysm.cell() if cell is None else cell
        fz = None if frozen is None else _i(frozen)
        self._keep.append(fz)
        bonds = _i(sysm.bonds.reshape(-1)) if len(sysm.bonds) else np.zeros(1, np.int32)
        angles = _i(sysm.angles.reshape(-1)) if len(sysm.angles) else np.zeros(1, np.int32)
        self.h = lib.ref_create(sysm.n, box_type, _d(cell), cutOff, cutOn, delr, linkRatio,
                                noLink, alpha, _d(sysm.x), _d(sysm.y), _d(sysm.z), _d(sysm.q),
                                _d(sysm.eps), _d(sysm.sig),
                                None if fz is None else fz.ctypes.data,
                                len(sysm.bonds), bonds, len(sysm.angles), angles)

    def set_torsions(self, dihe=None, impr=None):
        d = _i(np.asarray(dihe, dtype=np.int32).reshape(-1)) if dihe is not None and len(dihe) \
            else np.zeros(4, np.int32)
        m = _i(np.asarray(impr, dtype=np.int32).reshape(-1)) if impr is not None and len(impr) \
            else np.zeros(4, np.int32)
        nd = 0 if dihe is None else len(dihe)
        ni = 0 if impr is None else len(impr)
        self.lib().ref_set_torsions(self.h, nd, d, ni, m)

    def set_bonded(self, structs):
        """Bonded terms with parameters: five (count, ctypes array of MDBas
        structs) in the order bonds, angles, Urey-Bradley, dihedrals,
        impropers (ref_set_bonded copies them)."""
        args = []
        for m, arr in structs:
            args += [int(m), C.cast(arr, C.c_void_p)]
        self.lib().ref_set_bonded(self.h, *args)

    def set_kspace(self, mmax, prec=1e-6) -> int:
        """Explicit Ewald k-space (MDBas's init_ewald + ewald_rec) in every
        later energy() call, with the harness alpha and this m-range;
        returns the k-vector count."""
        return self.lib().ref_set_kspace(self.h, prec, *[int(v) for v in mmax])

    def set_nb14(self, scal14: float, dihedrals) -> None:
        """1-4 pairs of these dihedral quadruples (scaled by scal14) in every
        later energy() call; their list is made at the next makelist."""
        from mdbas_b200 import nb
        d = np.asarray(dihedrals, dtype=np.int64).reshape(-1, 4)
        arr = (nb.DIHE * max(1, len(d)))()
        for k, (a, b, c, e) in enumerate(d.tolist()):
            arr[k].a, arr[k].b, arr[k].c, arr[k].d = a, b, c, e
        self._keep.append(arr)
        self.lib().ref_set_nb14(self.h, float(scal14), len(d), C.cast(arr, C.c_void_p))

    def set_nonbond(self, elec_type: int, vdw_type: int) -> None:
        """Cut-off electrostatics: later energy() calls take MDBas's
        nonbond_energy (keyEwald = 0) with these elecType / vdwType."""
        if self.lib().ref_set_nonbond(self.h, int(elec_type), int(vdw_type)) != 0:
            raise ValueError("elecType / vdwType outside MDBas's enums")

    def bonded_energies(self) -> dict:
        """Bonded energies of the last energy() call."""
        out = np.zeros(7)
        self.lib().ref_bonded_energies(self.h, out)
        return dict(zip(["bond", "angle", "ub", "dihedral", "improper", "vir_bond", "vir_ub"],
                        out.tolist()))

    def list14(self):
        n14 = self.lib().ref_n_pair14(self.h)
        out = np.zeros(2 * max(n14, 1), np.int32)
        if n14:
            self.lib().ref_get_list14(self.h, out)
        return out[:2 * n14]

    @classmethod
    def layout(cls) -> str:
        buf = C.create_string_buffer(4096)
        cls.lib().ref_layout(buf, 4096)
        return buf.value.decode()

    def box(self) -> np.ndarray:
        out = np.zeros(30)
        self.lib().ref_box(self.h, out)
        return out

    def makelist(self) -> int:
        return self.lib().ref_makelist(self.h)

    def update_list(self, x=None, y=None, z=None):
        arrs = [None if a is None else _d(a) for a in (x, y, z)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self.lib().ref_update_list(self.h, *ptrs)

    @property
    def key_link(self) -> int:
        return self.lib().ref_key_link(self.h)

    @property
    def n_cells(self) -> int:
        return self.lib().ref_n_cells(self.h)

    @property
    def size_list(self) -> int:
        return self.lib().ref_size_list(self.h)

    def get_list(self):
        lib = self.lib()
        cnt = lib.ref_list_entries(self.h)
        lst = np.zeros(max(cnt, 1), np.int32)
        pair = np.zeros(self.n, np.int32)
        order = np.zeros(self.n, np.int32)
        lib.ref_get_list(self.h, lst, pair, order)
        return lst[:cnt], pair, order

    def list_ptrs(self):
        """MDBas's own neighList, neighPair and neighOrder arrays (pointers
        into the reference's memory, rebuilt in place by update_list)."""
        p = [C.POINTER(C.c_int)() for _ in range(3)]
        self.lib().ref_list_ptrs(self.h, *(C.byref(q) for q in p))
        return tuple(p)

    def get_excl(self):
        lib = self.lib()
        cnt = lib.ref_excl_entries(self.h)
        pair = np.zeros(self.n, np.int32)
        flat = np.zeros(max(cnt, 1), np.int32)
        lib.ref_get_excl(self.h, pair, flat)
        start = np.zeros(self.n + 1, np.int32)
        start[1:] = np.cumsum(pair)
        return start, flat[:cnt]

    def positions(self):
        x, y, z = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.lib().ref_get_positions(self.h, x, y, z)
        return x, y, z

    def set_positions(self, x, y, z):
        self.lib().ref_set_positions(self.h, _d(x), _d(y), _d(z))

    def energy(self):
        fx, fy, fz = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        out = np.zeros(6)
        self.lib().ref_energy(self.h, fx, fy, fz, out)
        return fx, fy, fz, dict(zip(["elec", "vdw", "virelec", "virvdw", "pot", "virpot"],
                                    out.tolist()))

    def self_energy(self) -> float:
        return self.lib().ref_self_energy(self.h)

    def md_init(self, mass, velocities=None, time_step=0.001, list_update=1, constraints=None,
                tol_shake=1e-8, max_cycle=150, temp0=0.0, tau_t=0.0) -> int:
        """Start MDBas's own velocity-Verlet dynamics (after makelist).  Returns
        the degrees of freedom MDBas counts."""
        self._md_keep = [_d(mass)]
        vp = [None, None, None]
        if velocities is not None:
            vs = [_d(a) for a in velocities]
            self._md_keep += vs
            vp = [a.ctypes.data for a in vs]
        nc, cp, cl = 0, None, None
        if constraints is not None and len(constraints[1]):
            pairs = _i(np.asarray(constraints[0]).reshape(-1))
            lens = _d(constraints[1])
            self._md_keep += [pairs, lens]
            nc, cp, cl = len(lens), pairs.ctypes.data, lens.ctypes.data
        r = self.lib().ref_md_init(self.h, self._md_keep[0], *vp, time_step, list_update, nc, cp,
                                   cl, tol_shake, max_cycle, temp0, tau_t)
        if r < 0:
            raise RuntimeError("ref_md_init: list not built or dynamics already started")
        return r

    def md_run(self, n_steps: int) -> np.ndarray:
        """Rows (step, pot, kin, pot + kin) after each step."""
        rows = np.zeros((max(n_steps, 1), 4))
        self.lib().ref_md_run(self.h, n_steps, rows)
        return rows[:n_steps]

    def ewald_rec(self, prec=1e-6, mmax=None):
        """MDBas's explicit Ewald reciprocal sum (init_ewald + ewald_rec) with the
        harness alpha: (energy incl. self and non-neutral terms, fx, fy, fz,
        virial, (m1max, m2max, m3max), k vectors)."""
        fx, fy, fz = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        out = np.zeros(6)
        mm = None
        if mmax is not None:
            self._mm = _i(np.asarray(mmax, dtype=np.int32))
            mm = self._mm.ctypes.data
        self.lib().ref_ewald_rec(self.h, prec, mm, fx, fy, fz, out)
        return (out[0], fx, fy, fz, out[1], tuple(int(v) for v in out[2:5]), int(out[5]))

    def velocities(self):
        vx, vy, vz = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.lib().ref_get_velocities(self.h, vx, vy, vz)
        return vx, vy, vz

    def now(self) -> float:
        return self.lib().ref_now()

    def close(self):
        if self.h:
            self.lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
