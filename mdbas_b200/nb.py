"""Python front of libmdbas_nb.so (ctypes over the C ABI of include/mdbas_nb.h).

* ``lib()`` loads the in-tree library and fails loudly when it is missing:
  there is no CPU fallback.
* ``PBC``, ``PARAM``, ``CTRL``, ``NEIGH``, ``ENERGY``, ``EWALD``, ``BOND``,
  ``ANGLE``, ``DIHE``, ``CONSTRAINT`` mirror MDBas's structs
  (include/global.h:175-316) for calling the drop-in routines.
* ``make_pbc`` fills a PBC the way MDBas's init_box does (src/init.c:840-908),
  with the same FP64 operation order, so the reciprocal vectors are
  bit-identical to MDBas's.
* ``Engine`` drives the device-resident engine (mdbas_nb_engine_*).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdbas_nb.so")

CUBIC, ORBIC, TCLIN = 1, 2, 3
NOELEC, FULL, SHIFT1, SHIFT2, SWITCH = 0, 1, 2, 3, 4
NOVDW, VFULL, VSWITCH = 0, 1, 2
BHARM, BMORSE = 0, 1          # enum BOND_TYPE
DCOS, DHARM = 1, 2            # enum DIHE_TYPE

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NO_DEVICE", 4: "ERR_ALLOC",
          5: "ERR_CAPACITY", 6: "ERR_BOX", 7: "ERR_LINKCELL", 8: "ERR_EXCL",
          9: "ERR_UNSUPPORTED", 10: "ERR_OVERFLOW", 11: "ERR_NONFINITE", 12: "ERR_MISSING",
          13: "ERR_STATE"}


class MdbasNbError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        text = f"{where}: {STATUS.get(status, status)}"
        if msg:
            text += f" ({msg})"
        super().__init__(text)


# ---------------------------------------------------------------------------
# MDBas structs (include/global.h)
# ---------------------------------------------------------------------------
_d = C.c_double
_i = C.c_int


class PBC(C.Structure):
    _fields_ = [("type", _i)] + [(n, _d) for n in (
        "a", "a1", "a2", "a3", "b", "b1", "b2", "b3", "c", "c1", "c2", "c3",
        "u", "u1", "u2", "u3", "v", "v1", "v2", "v3", "w", "w1", "w2", "w3",
        "pa", "pb", "pc", "det", "vol", "vol0",
        "stress1", "stress2", "stress3", "stress4", "stress5", "stress6",
        "stress7", "stress8", "stress9")]


class CTRL(C.Structure):
    _fields_ = [(n, _i) for n in (
        "newjob", "keyRand", "keyTraj", "keyProp", "keyForF", "keyRest", "printOut", "printProp",
        "printTraj", "printRest", "keyMd", "mdType", "seed", "keyMinim", "keyLink", "noLink",
        "keyConstH", "keyNb14", "keyNumForce", "keyEwald", "keyAlpha", "keyMmax", "elecType",
        "vdwType", "integrator", "ens")]


class PARAM(C.Structure):
    _fields_ = [("step", _i), ("nSteps", _i), ("timeStep", _d), ("rTimeStep", _d),
                ("nAtom", _i), ("nDegFree", _i), ("nFrozen", _i), ("nBond", _i),
                ("nAngle", _i), ("nDihedral", _i), ("nImproper", _i), ("nUb", _i),
                ("nConst", _i), ("maxCycle", _i), ("tolShake", _d), ("chargeConst", _d),
                ("delr", _d), ("scal14", _d), ("cutOff", _d), ("rcutOff", _d), ("cutOff2", _d),
                ("rcutOff2", _d), ("cutOn", _d), ("cutOn2", _d), ("switch2", _d),
                ("temp0", _d), ("press0", _d), ("kinTemp0", _d), ("tolMinim", _d),
                ("maxminsiz", _d), ("maxminst", _d)]


class BOND(C.Structure):
    _fields_ = [("type", _i), ("a", _i), ("b", _i), ("k", _d), ("r0", _d), ("beta", _d)]


class ANGLE(C.Structure):
    _fields_ = [("type", _i), ("a", _i), ("b", _i), ("c", _i), ("k", _d), ("theta0", _d)]


class DIHE(C.Structure):
    _fields_ = [("type", _i), ("order", _i), ("a", _i), ("b", _i), ("c", _i), ("d", _i),
                ("k", _d), ("phi0", _d), ("mult", _d)]


class NEIGH(C.Structure):
    _fields_ = [(n, _i) for n in ("update", "linkRatio", "nCells", "sizeList", "nPair14")]


class ENERGY(C.Structure):
    _fields_ = [(n, _d) for n in (
        "tot", "pot", "kin", "elec", "vdw", "bond", "ang", "ub", "dihe", "impr", "conint",
        "consv", "virelec", "virvdw", "virbond", "virub", "virshake", "virpot", "virtot")]


class CONSTRAINT(C.Structure):
    _fields_ = [("a", _i), ("b", _i), ("rc2", _d)]


class EWALD(C.Structure):
    _fields_ = [("nbsp", _i), ("mmax", _i), ("m1max", _i), ("m2max", _i), ("m3max", _i),
                ("prec", _d), ("tol", _d), ("tol1", _d), ("alpha", _d)]


class EngineConfig(C.Structure):
    _fields_ = [("nAtom", _i), ("device", _i), ("cutOff", _d), ("cutOn", _d), ("delr", _d),
                ("alpha", _d), ("chargeConst", _d), ("vdwSwitch", _i), ("precision", _i),
                ("linkRatio", _i), ("noLink", _i)]


class Energies(C.Structure):
    _fields_ = [(n, _d) for n in ("elec_direct", "elec_corr", "elec_self", "vdw", "vir_direct",
                                  "vir_corr", "vir_vdw", "n_pairs")]


def make_pbc(cell, box_type: int = CUBIC) -> PBC:
    """init_box (src/init.c:840-908) with MDBas's FP64 operation order."""
    a1, a2, a3, b1, b2, b3, c1, c2, c3 = (float(v) for v in cell)
    p = PBC()
    p.type = box_type
    p.a1, p.a2, p.a3, p.b1, p.b2, p.b3, p.c1, p.c2, p.c3 = a1, a2, a3, b1, b2, b3, c1, c2, c3
    p.a = math.sqrt(a1 * a1 + a2 * a2 + a3 * a3)
    p.b = math.sqrt(b1 * b1 + b2 * b2 + b3 * b3)
    p.c = math.sqrt(c1 * c1 + c2 * c2 + c3 * c3)
    u1 = b2 * c3 - c2 * b3
    u2 = c1 * b3 - b1 * c3
    u3 = b1 * c2 - c1 * b2
    v1 = c2 * a3 - a2 * c3
    v2 = a1 * c3 - c1 * a3
    v3 = c1 * a2 - a1 * c2
    w1 = a2 * b3 - b2 * a3
    w2 = b1 * a3 - a1 * b3
    w3 = a1 * b2 - b1 * a2
    det = a1 * u1 + a2 * u2 + a3 * u3
    p.det = det
    p.vol = abs(det)
    p.vol0 = p.vol
    p.pa = p.vol / math.sqrt(u1 * u1 + u2 * u2 + u3 * u3)
    p.pb = p.vol / math.sqrt(v1 * v1 + v2 * v2 + v3 * v3)
    p.pc = p.vol / math.sqrt(w1 * w1 + w2 * w2 + w3 * w3)
    p.u, p.v, p.w = 1.0 / p.pa, 1.0 / p.pb, 1.0 / p.pc
    if abs(det) > 0.0:
        u1, u2, u3 = u1 / det, u2 / det, u3 / det
        v1, v2, v3 = v1 / det, v2 / det, v3 / det
        w1, w2, w3 = w1 / det, w2 / det, w3 / det
    else:
        u1 = u2 = u3 = v1 = v2 = v3 = w1 = w2 = w3 = 0.0
    p.u1, p.u2, p.u3, p.v1, p.v2, p.v3, p.w1, p.w2, p.w3 = u1, u2, u3, v1, v2, v3, w1, w2, w3
    return p


def make_param(n_atom: int, cutOff=12.0, cutOn=10.0, delr=2.0, chargeConst=None,
               scal14=1.0) -> PARAM:
    """PARAM with the derived cut-off terms of read_SIMU (src/io.c:714-723)."""
    from .systems import CHARGE_CONST
    p = PARAM()
    p.nAtom = n_atom
    p.cutOff, p.cutOn, p.delr = cutOff, cutOn, delr
    p.chargeConst = CHARGE_CONST if chargeConst is None else chargeConst
    p.scal14 = scal14
    p.rcutOff = 1.0 / cutOff
    p.cutOff2 = cutOff * cutOff
    p.rcutOff2 = 1.0 / p.cutOff2
    p.cutOn2 = cutOn * cutOn
    d = p.cutOff2 - p.cutOn2
    p.switch2 = 1.0 / (d * d * d)
    return p


# ---------------------------------------------------------------------------
# Library loading
# ---------------------------------------------------------------------------
_LIB = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def lib():
    """The CUDA library.  Raises when it is not built: no fallback exists."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing; run mdbas_b200.build.build() first")
    L = C.CDLL(LIB_PATH)
    L.mdbas_nb_status_string.restype = C.c_char_p
    L.mdbas_nb_status_string.argtypes = [C.c_int]
    L.mdbas_nb_last_message.restype = C.c_char_p
    L.mdbas_nb_engine_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(EngineConfig),
                                         C.POINTER(PBC)]
    for name in ("destroy", "build", "refresh", "compute"):
        getattr(L, f"mdbas_nb_engine_{name}").argtypes = [C.c_void_p]
    L.mdbas_nb_engine_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.mdbas_nb_engine_set_box.argtypes = [C.c_void_p, C.POINTER(PBC)]
    L.mdbas_nb_engine_set_topology.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip, _ip, _ip]
    L.mdbas_nb_engine_set_positions.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int]
    L.mdbas_nb_engine_get_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_int]
    L.mdbas_nb_engine_energies.argtypes = [C.c_void_p, C.POINTER(Energies)]
    L.mdbas_nb_engine_evaluate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(Energies)]
    L.mdbas_nb_engine_list_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    L.mdbas_nb_engine_export_pairs.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_longlong,
                                               C.POINTER(C.c_longlong)]
    L.mdbas_nb_engine_launch_count.restype = C.c_longlong
    L.mdbas_nb_engine_launch_count.argtypes = [C.c_void_p]
    L.mdbas_nb_engine_set_timing.argtypes = [C.c_void_p, C.c_int]
    L.mdbas_nb_engine_set_variant.argtypes = [C.c_void_p, C.c_int]
    L.mdbas_nb_engine_build_stages.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.mdbas_nb_engine_kernel_time.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                              C.POINTER(C.c_longlong), C.c_int]
    L.mdbas_nb_engine_md_init.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_double, C.c_int,
                                          C.c_int, _ip, _dp, C.c_double, C.c_int]
    L.mdbas_nb_engine_md_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                         _dp]
    L.mdbas_nb_engine_md_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    L.mdbas_nb_engine_md_set_graph.argtypes = [C.c_void_p, C.c_int]
    L.mdbas_nb_engine_md_set_prune.argtypes = [C.c_void_p, C.c_double]
    L.mdbas_nb_batch_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(EngineConfig), C.c_int,
                                        C.POINTER(PBC), _ip]
    L.mdbas_nb_batch_count.argtypes = [C.c_void_p]
    L.mdbas_nb_engine_autotune.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.mdbas_nb_engine_adjoint.argtypes = [C.c_void_p] + [C.c_void_p] * 12 + [C.c_int]
    L.mdbas_nb_spme.argtypes = [C.c_int, C.POINTER(PBC), C.c_double, C.c_double, C.c_int,
                                C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 7 + [
                                    C.POINTER(C.c_double), C.c_int, C.c_void_p]
    for name in ("get_positions", "get_velocities"):
        getattr(L, f"mdbas_nb_engine_{name}").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p,
                                                          C.c_void_p, C.c_int]
    L.mdbas_nb_ewald_rec.argtypes = [C.c_int, C.POINTER(PBC), C.c_double, C.c_double, C.c_int,
                                     C.c_int, C.c_int] + [C.c_void_p] * 7 + [
                                         C.POINTER(C.c_double), C.c_int, C.c_void_p]
    L.mdbas_nb_engine_set_kspace.argtypes = [C.c_void_p] + [C.c_int] * 5
    L.mdbas_nb_engine_kspace.argtypes = [C.c_void_p] + [C.c_void_p] * 3 + [
        C.POINTER(C.c_double)]
    L.mdbas_nb_bonded.argtypes = [C.c_int, C.c_int, C.POINTER(PBC), C.c_int, C.c_void_p] + [
        C.c_void_p] * 6 + [C.POINTER(C.c_double)]
    L.mdbas_nb_engine_set_bonded.argtypes = [C.c_void_p] + [C.c_int, C.c_void_p] * 5
    L.mdbas_nb_engine_bonded.argtypes = [C.c_void_p] + [C.c_void_p] * 3 + [
        C.c_int, C.POINTER(C.c_double)]
    _LIB = L
    return L


def check(st: int, where: str) -> None:
    if st != 0:
        msg = lib().mdbas_nb_last_message()
        raise MdbasNbError(st, where, msg.decode() if msg else "")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def spme(system, alpha=0.34, grid=(32, 32, 32), nbsp=8, chargeConst=None, cell=None,
         box_type: int = CUBIC):
    """Reciprocal-space Ewald by SPME on the GPU (host arrays): (energy incl.
    self and non-neutral terms, fx, fy, fz, virial)."""
    from .systems import CHARGE_CONST
    pbc = make_pbc(system.cell() if cell is None else cell, box_type)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (system.x, system.y, system.z,
                                                               system.q)]
    f = [np.zeros(system.n) for _ in range(3)]
    out = (C.c_double * 8)()
    check(lib().mdbas_nb_spme(system.n, C.byref(pbc), alpha,
                              CHARGE_CONST if chargeConst is None else chargeConst, *grid, nbsp,
                              *(_ptr(a) for a in arrs), *(_ptr(a) for a in f), out, 0, None),
          "spme")
    return out[0], f[0], f[1], f[2], out[1]


def ewald_rec(system, alpha=0.34, mmax=(8, 8, 8), chargeConst=None, cell=None,
              box_type: int = CUBIC, forces=None):
    """Explicit reciprocal-space Ewald sum on the GPU (host arrays): (energy
    incl. self and non-neutral terms, fx, fy, fz, virial, stress[6]); the
    forces are added to copies of `forces` (or to zeros)."""
    from .systems import CHARGE_CONST
    pbc = make_pbc(system.cell() if cell is None else cell, box_type)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (system.x, system.y, system.z,
                                                               system.q)]
    f = ([np.zeros(system.n) for _ in range(3)] if forces is None
         else [np.array(a, dtype=np.float64) for a in forces])
    out = (C.c_double * 8)()
    check(lib().mdbas_nb_ewald_rec(system.n, C.byref(pbc), alpha,
                                   CHARGE_CONST if chargeConst is None else chargeConst, *mmax,
                                   *(_ptr(a) for a in arrs), *(_ptr(a) for a in f), out, 0,
                                   None), "ewald_rec")
    return out[0], f[0], f[1], f[2], out[1], list(out[2:8])


# Bonded kinds in the order of MDBas's energy() (src/energy.c:167-190).
BONDED_KINDS = ("bonds", "angles", "ub", "dihedrals", "impropers")
BONDED_ENERGIES = ("bond", "angle", "ub", "dihedral", "improper", "vir_bond", "vir_ub")


def bonded_structs(spec: dict | None) -> list:
    """MDBas struct arrays (BOND, ANGLE, BOND, DIHE, DIHE) of a bonded spec:
    spec[kind] = {"atoms": (m, arity) ints, "k": ..., and per kind "type",
    "r0", "beta" (bonds, ub), "theta0" (angles), "phi0", "mult" (torsions)}
    with MDBas's units (k in internal units, angles in radians).  Missing
    kinds give empty arrays."""
    out = []
    for kind, cls in zip(BONDED_KINDS, (BOND, ANGLE, BOND, DIHE, DIHE)):
        t = (spec or {}).get(kind)
        m = 0 if t is None else len(t["atoms"])
        arr = (cls * max(1, m))()
        for i in range(m):
            at = [int(v) for v in t["atoms"][i]]
            e = arr[i]
            e.type = int(t["type"][i]) if "type" in t else (DCOS if cls is DIHE else 0)
            e.k = float(t["k"][i])
            if cls is BOND:
                e.a, e.b = at
                e.r0 = float(t["r0"][i])
                e.beta = float(t["beta"][i]) if "beta" in t else 0.0
            elif cls is ANGLE:
                e.a, e.b, e.c = at
                e.theta0 = float(t["theta0"][i])
            else:
                e.a, e.b, e.c, e.d = at
                e.order = int(t["order"][i]) if "order" in t else 0
                e.phi0 = float(t["phi0"][i])
                e.mult = float(t["mult"][i]) if "mult" in t else 1.0
        out.append((m, arr))
    return out


def bonded(kind: int, system, terms, forces=None, cell=None, box_type: int = CUBIC):
    """One bonded routine on the GPU (mdbas_nb_bonded): kind 0..4 in
    BONDED_KINDS order, terms a ctypes struct array (bonded_structs).
    Returns (energy, virial, fx, fy, fz) with the forces added to `forces`
    (copies) or to zeros."""
    pbc = make_pbc(system.cell() if cell is None else cell, box_type)
    n = system.n
    pos = [np.ascontiguousarray(a, dtype=np.float64) for a in (system.x, system.y, system.z)]
    f = ([np.zeros(n) for _ in range(3)] if forces is None
         else [np.array(a, dtype=np.float64) for a in forces])
    m = len(terms) if terms is not None else 0
    out = (C.c_double * 2)()
    check(lib().mdbas_nb_bonded(kind, n, C.byref(pbc), m, C.cast(terms, C.c_void_p),
                                *(_ptr(a) for a in pos), *(_ptr(a) for a in f), out), "bonded")
    return out[0], out[1], f[0], f[1], f[2]


class Engine:
    """Device-resident nonbonded engine for one system.

    precision 0: plain FP64 form over MDBas's half list (built on the GPU);
    precision 1: FP32 pair arithmetic with 64-bit fixed-point accumulation
    over the cluster-pair list.
    """

    def __init__(self, system, precision: int = 1, device: int = 0, cutOff=12.0, cutOn=10.0,
                 delr=2.0, alpha=0.34, chargeConst=None, vdwSwitch=1, linkRatio=1, noLink=0,
                 frozen=None, box_type: int = CUBIC, cell=None, exclusions=None):
        from .systems import CHARGE_CONST
        L = lib()
        self.n = system.n
        self.precision = precision
        cfg = EngineConfig(self.n, device, cutOff, cutOn, delr, alpha,
                           CHARGE_CONST if chargeConst is None else chargeConst, vdwSwitch,
                           precision, linkRatio, noLink)
        h = C.c_void_p()
        reps = system.meta.get("replicas") if system.meta else None
        if reps:
            # a batch of independent boxes (systems.concat)
            self.pbc = (PBC * len(reps))(*[make_pbc(c, box_type) for c, _ in reps])
            counts = np.array([k for _, k in reps], dtype=np.int32)
            self.offsets = np.concatenate([[0], np.cumsum(counts)])
            check(L.mdbas_nb_batch_create(C.byref(h), C.byref(cfg), len(reps), self.pbc,
                                          counts.ctypes.data_as(_ip)), "batch_create")
        else:
            self.pbc = make_pbc(system.cell() if cell is None else cell, box_type)
            self.offsets = np.array([0, self.n])
            check(L.mdbas_nb_engine_create(C.byref(h), C.byref(cfg), C.byref(self.pbc)),
                  "engine_create")
        self.h = h
        # exclusions: (start[n+1], flat) rows, by default from the system's
        # bonds and angles
        start, flat = system.exclusions(symmetric=True) if exclusions is None else exclusions
        pair = np.diff(start).astype(np.int32)
        self._topo = [np.ascontiguousarray(a, dtype=np.float64)
                      for a in (system.q, system.eps, system.sig)]
        fz = None if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        flat = np.ascontiguousarray(flat if len(flat) else np.zeros(1, np.int32), dtype=np.int32)
        self._frozen, self._excl_pair, self._excl_flat = fz, pair, flat
        check(L.mdbas_nb_engine_set_topology(
            h, *(a.ctypes.data_as(_dp) for a in self._topo),
            None if fz is None else fz.ctypes.data_as(_ip), pair.ctypes.data_as(_ip),
            flat.ctypes.data_as(_ip)), "engine_set_topology")
        self.set_positions(system.x, system.y, system.z)

    def set_parameters(self, q, eps, sig):
        """Replace the per-atom charges and LJ parameters (MDBas per-atom
        values; exclusions and frozen atoms kept)."""
        self._topo = [np.ascontiguousarray(a, dtype=np.float64) for a in (q, eps, sig)]
        check(lib().mdbas_nb_engine_set_topology(
            self.h, *(a.ctypes.data_as(_dp) for a in self._topo),
            None if self._frozen is None else self._frozen.ctypes.data_as(_ip),
            self._excl_pair.ctypes.data_as(_ip), self._excl_flat.ctypes.data_as(_ip)),
            "engine_set_topology")

    def set_positions(self, x, y, z):
        self._pos = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        check(lib().mdbas_nb_engine_set_positions(self.h, *(_ptr(a) for a in self._pos), 0),
              "engine_set_positions")

    def set_positions_device(self, xp: int, yp: int, zp: int):
        check(lib().mdbas_nb_engine_set_positions(self.h, C.c_void_p(xp), C.c_void_p(yp),
                                                  C.c_void_p(zp), 1), "engine_set_positions")

    def build(self):
        check(lib().mdbas_nb_engine_build(self.h), "engine_build")

    def refresh(self):
        check(lib().mdbas_nb_engine_refresh(self.h), "engine_refresh")

    def compute(self):
        check(lib().mdbas_nb_engine_compute(self.h), "engine_compute")

    def forces(self):
        f = [np.zeros(self.n) for _ in range(3)]
        check(lib().mdbas_nb_engine_get_forces(self.h, *(_ptr(a) for a in f), 0),
              "engine_get_forces")
        return f

    def forces_into(self, fx: np.ndarray, fy: np.ndarray, fz: np.ndarray):
        """Copy the forces into caller-owned (e.g. pinned) FP64 arrays."""
        check(lib().mdbas_nb_engine_get_forces(self.h, _ptr(fx), _ptr(fy), _ptr(fz), 0),
              "engine_get_forces")

    def set_stream(self, stream_handle: int):
        check(lib().mdbas_nb_engine_set_stream(self.h, C.c_void_p(stream_handle)),
              "engine_set_stream")

    def forces_device(self, xp: int, yp: int, zp: int):
        check(lib().mdbas_nb_engine_get_forces(self.h, C.c_void_p(xp), C.c_void_p(yp),
                                               C.c_void_p(zp), 1), "engine_get_forces")

    def energies(self) -> dict:
        e = Energies()
        check(lib().mdbas_nb_engine_energies(self.h, C.byref(e)), "engine_energies")
        return {k: getattr(e, k) for k, _ in Energies._fields_}

    def evaluate(self, x, y, z, fx, fy, fz, rebuild: bool = True) -> dict:
        """One evaluation on host arrays in one C-ABI call (positions in,
        forces into the caller's FP64 arrays fx/fy/fz, energies returned):
        set_positions, build (or refresh), compute, get_forces, energies."""
        self._pos = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        for a in (fx, fy, fz):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape[0] != self.n:
                raise ValueError("forces need contiguous float64 arrays of n entries")
        e = Energies()
        check(lib().mdbas_nb_engine_evaluate(self.h, *(_ptr(a) for a in self._pos), int(rebuild),
                                             _ptr(fx), _ptr(fy), _ptr(fz), C.byref(e)),
              "engine_evaluate")
        return {k: getattr(e, k) for k, _ in Energies._fields_}

    def list_stats(self):
        out = (C.c_longlong * 4)()
        check(lib().mdbas_nb_engine_list_stats(self.h, out), "engine_list_stats")
        return list(out)

    def export_pairs(self, r2max: float) -> np.ndarray:
        cnt = C.c_longlong(0)
        check(lib().mdbas_nb_engine_export_pairs(self.h, r2max, None, 0, C.byref(cnt)),
              "engine_export_pairs")
        buf = np.zeros(2 * max(cnt.value, 1), np.int32)
        check(lib().mdbas_nb_engine_export_pairs(self.h, r2max, _ptr(buf), cnt.value,
                                                 C.byref(cnt)), "engine_export_pairs")
        return buf[:2 * cnt.value].reshape(-1, 2)

    def build_stages(self) -> dict:
        """One synchronising list build timed stage by stage (ms)."""
        ms = (C.c_double * 6)()
        check(lib().mdbas_nb_engine_build_stages(self.h, ms), "engine_build_stages")
        return dict(zip(("bin", "grid_scans", "scatter", "column_sort", "cluster_layout",
                         "search"), list(ms)))

    def launches(self) -> int:
        return int(lib().mdbas_nb_engine_launch_count(self.h))

    def set_variant(self, variant: int):
        """Pair kernel: 7 = half clusters (8-atom i x 4-atom j), packed
        f32x2, inner list, lean form (default), 4 = the same in its first
        form, 5 = that at 80 registers, 6 = quad
        (4-atom i x 4-atom j units of the inner list), 2 = packed f32x2 8x8,
        staged, 0 = scalar dense 8x8, 1 = filtered and compacted, 3 = packed
        with bulk-copy staging."""
        check(lib().mdbas_nb_engine_set_variant(self.h, variant), "engine_set_variant")

    def set_timing(self, on: bool):
        check(lib().mdbas_nb_engine_set_timing(self.h, 1 if on else 0), "engine_set_timing")

    def pair_kernel_ms(self, reset: bool = True):
        ms, cnt = C.c_double(0), C.c_longlong(0)
        check(lib().mdbas_nb_engine_kernel_time(self.h, 0, C.byref(ms), C.byref(cnt),
                                                1 if reset else 0), "engine_kernel_time")
        return ms.value, cnt.value

    # -- velocity-Verlet dynamics (mdbas_nb_engine_md_*) ----------------------
    def md_init(self, mass, velocities=None, time_step=0.001, list_update=0, constraints=None,
                tol_shake=1e-8, max_cycle=150):
        """Start dynamics.  constraints = (pairs (k, 2) int, squared lengths (k,))."""
        self._mass = np.ascontiguousarray(mass, dtype=np.float64)
        if velocities is None:
            vp = [None, None, None]
        else:
            self._v0 = [np.ascontiguousarray(a, dtype=np.float64) for a in velocities]
            vp = [a.ctypes.data_as(_dp) for a in self._v0]
        nc, cp, cl = 0, None, None
        if constraints is not None and len(constraints[1]):
            self._cpairs = np.ascontiguousarray(constraints[0], dtype=np.int32).reshape(-1)
            self._clen2 = np.ascontiguousarray(constraints[1], dtype=np.float64)
            nc = len(self._clen2)
            cp, cl = self._cpairs.ctypes.data_as(_ip), self._clen2.ctypes.data_as(_dp)
        check(lib().mdbas_nb_engine_md_init(self.h, self._mass.ctypes.data_as(_dp), *vp,
                                            time_step, list_update, nc, cp, cl, tol_shake,
                                            max_cycle), "engine_md_init")

    def md_run(self, n_steps: int, energy_every: int = 0, target_temp: float = 0.0,
               tau_t: float = 0.0):
        """Advance n_steps; returns rows (step, potential, kinetic, total)."""
        rows = n_steps // energy_every if energy_every > 0 else 0
        buf = np.zeros((max(rows, 1), 4))
        check(lib().mdbas_nb_engine_md_run(self.h, n_steps, energy_every, target_temp, tau_t,
                                           buf.ctypes.data_as(_dp) if rows else None),
              "engine_md_run")
        return buf[:rows]

    def autotune(self) -> dict:
        """Time the pair kernel's variants and launch shapes on the current list
        and keep the fastest (call after build; recompute afterwards)."""
        out = (C.c_int * 4)()
        check(lib().mdbas_nb_engine_autotune(self.h, out), "engine_autotune")
        # the variants differ in their cluster shapes: the quad one (6) pairs
        # 4-atom i-cluster halves with 4-atom j-cluster halves, the half ones
        # (4, 5, 7) 8-atom i clusters with 4-atom j-cluster halves, the others
        # 8-atom i with 8-atom j clusters
        return {"variant": out[0], "block": out[1], "blocks_per_sm": out[2],
                "candidates": out[3], "i_cluster_atoms": 4 if out[0] == 6 else 8,
                "j_cluster_atoms": 4 if out[0] in (4, 5, 6, 7) else 8}

    def split(self, arrays):
        """Per-replica views of concatenated per-atom arrays."""
        o = self.offsets
        return [[a[o[r]:o[r + 1]] for a in arrays] for r in range(len(o) - 1)]

    @staticmethod
    def split_arrays(arrays, batch):
        """Per-replica views of per-atom arrays of a systems.concat batch."""
        o = batch.meta["offsets"]
        return [[a[o[r]:o[r + 1]] for a in arrays] for r in range(len(o) - 1)]

    def set_bonded(self, spec: dict | None):
        """Bonded terms of the dynamics (see bonded_structs; None clears)."""
        self._bonded = bonded_structs(spec)
        args = []
        for m, arr in self._bonded:
            args += [m, C.cast(arr, C.c_void_p)]
        check(lib().mdbas_nb_engine_set_bonded(self.h, *args), "set_bonded")

    def set_kspace(self, kind: int, m=(0, 0, 0), order: int = 0):
        """Reciprocal space of the dynamics: 0 off, 1 explicit Ewald with the
        m-range m, 2 SPME on the grid m with B-spline order `order`."""
        check(lib().mdbas_nb_engine_set_kspace(self.h, int(kind), *[int(v) for v in m],
                                               int(order)), "set_kspace")

    def kspace(self, forces=None):
        """(energy incl. self and non-neutral terms, virial, [fx, fy, fz]) of
        the reciprocal term at the current positions; forces added to copies
        of `forces` (or to zeros)."""
        f = ([np.zeros(self.n) for _ in range(3)] if forces is None
             else [np.array(a, dtype=np.float64) for a in forces])
        out = (C.c_double * 2)()
        check(lib().mdbas_nb_engine_kspace(self.h, *(_ptr(a) for a in f), out), "kspace")
        return out[0], out[1], f

    def bonded(self, forces=None):
        """Bonded energies at the current positions (dict of BONDED_ENERGIES)
        and forces: added to copies of `forces` (3 arrays) or to zeros."""
        f = ([np.zeros(self.n) for _ in range(3)] if forces is None
             else [np.array(a, dtype=np.float64) for a in forces])
        out = (C.c_double * 7)()
        check(lib().mdbas_nb_engine_bonded(self.h, *(_ptr(a) for a in f), 0, out), "bonded")
        return dict(zip(BONDED_ENERGIES, out)), f

    def adjoint(self, v=None) -> dict:
        """dE/d(q, eps, sig) per atom and, with force weights v = (vx, vy, vz),
        d(v.F)/dx and d(v.F)/d(q, eps, sig) (FP64 form engines, after build)."""
        n = self.n
        names = ["gq", "geps", "gsig", "hx", "hy", "hz", "pq", "peps", "psig"]
        out = {k: np.zeros(n) for k in (names if v is not None else names[:3])}
        vv = [None, None, None]
        if v is not None:
            self._adj_v = [np.ascontiguousarray(a, dtype=np.float64) for a in v]
            vv = [_ptr(a) for a in self._adj_v]
        ptrs = [_ptr(out[k]) if k in out else None for k in names]
        check(lib().mdbas_nb_engine_adjoint(self.h, *vv, *ptrs, 0), "engine_adjoint")
        return out

    def md_set_graph(self, steps_per_launch: int):
        """Steps per CUDA-graph launch of the mixed-precision dynamics (0 = off)."""
        check(lib().mdbas_nb_engine_md_set_graph(self.h, steps_per_launch), "engine_md_set_graph")

    def md_set_prune(self, buffer: float):
        """Inner-list buffer (A) of the mixed form's dynamics; 0 disables pruning."""
        check(lib().mdbas_nb_engine_md_set_prune(self.h, buffer), "engine_md_set_prune")

    def md_stats(self):
        out = (C.c_longlong * 6)()
        check(lib().mdbas_nb_engine_md_stats(self.h, out), "engine_md_stats")
        return {"steps": out[0], "rebuilds": out[1], "shake_iter": out[2], "molecules": out[3],
                "prunes": out[4], "pruned_list": bool(out[5])}

    def positions(self):
        p = [np.zeros(self.n) for _ in range(3)]
        check(lib().mdbas_nb_engine_get_positions(self.h, *(_ptr(a) for a in p), 0),
              "engine_get_positions")
        return p

    def velocities(self):
        v = [np.zeros(self.n) for _ in range(3)]
        check(lib().mdbas_nb_engine_get_velocities(self.h, *(_ptr(a) for a in v), 0),
              "engine_get_velocities")
        return v

    def close(self):
        if getattr(self, "h", None):
            lib().mdbas_nb_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Drop-in routines (MDBas prototypes) for Python callers and tests.
# ---------------------------------------------------------------------------
_pp = C.POINTER(C.POINTER(C.c_int))
_ppp = C.POINTER(C.POINTER(C.POINTER(C.c_int)))


def bind_dropin():
    """Declare ctypes prototypes of the drop-in routines on lib()."""
    L = lib()
    if getattr(L, "_dropin_bound", False):
        return L
    P = C.POINTER
    L.init_energy_ptrs.argtypes = [P(CTRL)]
    L.makelist.argtypes = [P(CTRL), P(PARAM), P(PBC), P(NEIGH), P(CONSTRAINT), P(BOND), P(ANGLE),
                           P(DIHE), P(DIHE), _dp, _dp, _dp, _ip, _pp, _pp, _pp, _pp, _ppp, _pp]
    for name in ("exclude_list", "link_cell_exclude_list"):
        getattr(L, name).argtypes = [P(CTRL), P(PARAM), P(NEIGH), P(CONSTRAINT), P(BOND),
                                     P(ANGLE), P(DIHE), P(DIHE), _pp, _ppp, _pp]
    L.mdbas_nb_verlet_list_status.argtypes = [P(PARAM), P(PBC), P(NEIGH), _dp, _dp, _dp, _ip,
                                              _pp, _pp, _pp, P(_ip), _ip, C.c_int]
    L.mdbas_nb_link_cell_list_status.argtypes = L.mdbas_nb_verlet_list_status.argtypes
    L.energy.argtypes = [P(CTRL), P(PARAM), P(ENERGY), P(EWALD), P(PBC), P(NEIGH), P(BOND),
                         P(BOND), P(ANGLE), P(DIHE), P(DIHE), _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                         _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, _ip, P(_ip), _ip]
    L.mdbas_nb_ewald_energy_status.argtypes = [P(CTRL), P(PARAM), P(ENERGY), P(EWALD), P(PBC),
                                               _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip,
                                               _ip, _ip, P(_ip), _ip]
    L.nonbond_energy.argtypes = [P(PARAM), P(ENERGY), P(PBC), _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                 _dp, _dp, _ip, _ip, _ip]
    L.ewald14_energy.argtypes = [P(PARAM), P(ENERGY), P(EWALD), P(PBC), P(NEIGH), _dp, _dp, _dp,
                                 _dp, _dp, _dp, _dp, _dp, _dp, _ip]
    L.nonbond14_energy.argtypes = [P(PARAM), P(ENERGY), P(PBC), P(NEIGH), _dp, _dp, _dp, _dp,
                                   _dp, _dp, _dp, _dp, _dp, _ip]
    L.mdbas_nb_plugin_init.argtypes = [C.c_int, _dp, _dp, _dp, _ip, P(_ip), C.c_double, C.c_int]
    L.mdbas_nb_user_energy.restype = C.c_double
    L.mdbas_nb_user_energy.argtypes = [P(PARAM), P(PBC), _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                       _ip, _ip]
    L.mdbas_nb_plugin_last_energy.argtypes = [_dp]
    L.mdbas_nb_set_mode.argtypes = [C.c_int]
    L._dropin_bound = True
    return L


def as_dp(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def as_ip(a: np.ndarray):
    return a.ctypes.data_as(_ip)
