"""MDBas's input and output files for the GPU engine (src/io.c).

Readers give the values MDBas's own readers leave in its structs, so a run
set up from MDBas's SIMU / CONF / FORF files on the engine starts from the
same numbers as MDBas:

* ``read_simu`` -- the SIMU control file (read_SIMU, src/io.c:29-727):
  keywords, defaults and the derived cut-off terms;
* ``read_conf`` -- the CONF coordinates (read_CONF, src/io.c:728-783), with
  MDBas's fscanf field rules (``%4s`` reads at most four characters);
* ``read_forf`` -- the FORF force field (read_FORF, src/io.c:872-1199): atoms,
  bonds, constraints, Urey-Bradley terms, angles, dihedrals, impropers and
  the per-atom LJ parameters, converted to internal units as MDBas does;
* ``read_rest`` / ``write_rest`` -- the binary restart file (src/io.c:785-870,
  1276-1369), byte for byte MDBas's layout;
* ``write_conf`` -- the RCON coordinates (write_CONF, src/io.c:1201-1228);
* ``write_prop`` -- one 29-double PROP record (write_prop, src/io.c:1230-1274);
* ``write_dcd_header`` / ``write_dcd_frame`` -- the DCD trajectory
  (src/io.c:1371-1520).

``write_simu`` and ``write_forf`` write the inverse (MDBas has no writers for
them), so that generated systems can be handed to MDBas itself; ``load``
turns a SIMU file and the CONF / FORF it names into a ``systems.System``
with its bonded terms, constraints and frozen atoms, ready for
``nb.Engine``.

Errors: where MDBas calls my_error (and exits) these readers raise
``MdbasFileError`` naming MDBas's error; where MDBas would read past a
malformed field silently (a short CONF line, a blank FORF line) they raise
too.

Two deliberate differences: ``write_conf`` keeps a blank between the atom
and residue numbers when MDBas's ``%5d%5d`` would run them together (atom
numbers from 100,000 or residue numbers from 10,000 up), so that large
systems read back; relative file names in SIMU are taken relative to the
SIMU file's directory (MDBas: the working directory) unless ``base_dir`` is
given.
"""
from __future__ import annotations

import math
import os
import re
import struct
import time
from dataclasses import dataclass, field

import numpy as np

KCAL_TO_IU = 418.4        # include/global.h:41 kcaltoiu
BAR_TO_IU = 6.02214129e-3  # include/global.h:44 bartoiu
RBOLTZ_IU = 0.83144621     # include/global.h:47 rboltzui
WATER_COMP = 0.007372      # include/global.h:56 watercomp
PI = 3.141592653589793     # include/global.h:53

# enums of include/global.h:79-153
NOELEC, FULL, SHIFT1, SHIFT2, SWITCH = 0, 1, 2, 3, 4
NOVDW, VFULL, VSWITCH = 0, 1, 2
NOBOX, CUBIC, ORBIC, TCLIN = 0, 1, 2, 3
LEAPFROG, VELOCITY = 0, 1
NVE, NVT_B, NPT_B, NVT_H, NPT_H = 0, 1, 2, 3, 4

ATOM_STRUCT = struct.Struct("<5s5s5sxiii")  # ATOM, include/global.h:165-169 (28 bytes)
ENERGY_FIELDS = ("tot", "pot", "kin", "elec", "vdw", "bond", "ang", "ub", "dihe", "impr",
                 "conint", "consv", "virelec", "virvdw", "virbond", "virub", "virshake",
                 "virpot", "virtot")  # ENERGY, include/global.h:282-290


class MdbasFileError(ValueError):
    """A file MDBas would reject (its error name in the message)."""


# ---------------------------------------------------------------------------
# C conversions with MDBas's semantics
# ---------------------------------------------------------------------------
_INT = re.compile(r"[ \t\n\v\f\r]*([+-]?\d+)")
_FLOAT = re.compile(r"[ \t\n\v\f\r]*([+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))",
                    re.IGNORECASE)


def c_atoi(s: str) -> int:
    """atoi: the leading integer of s, 0 when there is none."""
    m = _INT.match(s)
    return int(m.group(1)) if m else 0


def c_atof(s: str) -> float:
    """atof / strtod: the leading decimal number of s, 0.0 when there is none."""
    m = _FLOAT.match(s)
    return float(m.group(1)) if m else 0.0


def _tokens(line: str) -> list[str]:
    """strtok(line, " \\n\\t") tokens."""
    return [t for t in re.split(r"[ \n\t]+", line) if t]


def _c_int(v: int) -> int:
    """(int) of a C double -> int assignment (truncation toward zero)."""
    return int(math.trunc(v))


# ---------------------------------------------------------------------------
# SIMU
# ---------------------------------------------------------------------------
@dataclass
class Simu:
    """The fields read_SIMU sets, by MDBas struct (CTRL, PARAM, EWALD, NEIGH,
    BATH), the box rows and the file names."""
    ctrl: dict
    param: dict
    ewald: dict
    neigh: dict
    bath: dict
    box_type: int
    cell: np.ndarray
    files: dict


def read_simu(path: str) -> Simu:
    """read_SIMU (src/io.c:29-727)."""
    files = dict(conf="CONF", forf="FORF", prop="PROP", rest="REST", rcon="RCON", traj="TRAJ")
    ctrl = dict(keyMd=1, keyRest=0, keyMinim=0, newjob=1, mdType=1, ens=NVE, keyRand=0,
                seed=12345, keyEwald=0, keyAlpha=0, keyMmax=0, elecType=FULL, vdwType=VFULL,
                keyNb14=0, keyNumForce=0, noLink=0, integrator=VELOCITY, keyConstH=0, keyProp=0,
                keyTraj=0, keyForF=0, printOut=1000, printProp=1000, printTraj=1000,
                printRest=1000)
    param = dict(tolMinim=1.e-3, maxminst=1000, maxminsiz=0.15, step=0, timeStep=0.001,
                 nSteps=0, cutOff=12.0, cutOn=10.0, delr=2.0, temp0=300.0, press0=1.0,
                 scal14=1.0, tolShake=1.e-8, maxCycle=150, nConst=0)
    ewald = dict(nbsp=8, prec=0.0, alpha=0.0, m1max=0, m2max=0, m3max=0)
    neigh = dict(update=20, linkRatio=1)
    bath = dict(tauT=0.1, tauP=0.5, compress=WATER_COMP)
    box_type = 0
    cell = np.zeros(9)
    with open(path, "r", encoding="latin-1") as fh:
        lines = fh.read().split("\n")

    def need(toks, i, what="a value"):
        if len(toks) <= i:
            raise MdbasFileError(f"SIMU_NOTFOUND_ERROR: {what} missing after {toks[0]!r}")
        return toks[i]

    li = 0
    while li < len(lines):
        line = lines[li]
        li += 1
        toks = _tokens(line)
        if not toks:
            continue
        key = toks[0].lower()
        if key == "mdbas":
            ctrl["mdType"] = 0
        elif key == "charmm":
            ctrl["mdType"] = 1
        elif key == "namd":
            ctrl["mdType"] = 2
        elif key == "dlpoly":
            ctrl["mdType"] = 3
        elif key == "nomd":
            ctrl["keyMd"] = 0
        elif key == "restart":
            ctrl["keyRest"] = 1
        elif key == "file":
            kind = need(toks, 1, "type of file").lower()
            if kind not in files:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: file {kind}")
            files[kind] = need(toks, 2, "name of file")
        elif key == "minim":
            ctrl["keyMinim"] = 1
            sub = need(toks, 1).lower()
            if sub == "tol":
                param["tolMinim"] = c_atof(need(toks, 2))
            elif sub == "maxcycle":
                param["maxminst"] = c_atoi(need(toks, 2))
            elif sub == "maxsize":
                param["maxminsiz"] = c_atof(need(toks, 2))
            else:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: minim {sub}")
        elif key in ("timestep", "cutoff", "cuton", "delr", "temperature"):
            name = dict(timestep="timeStep", cutoff="cutOff", cuton="cutOn", delr="delr",
                        temperature="temp0")[key]
            param[name] = c_atof(need(toks, 1))
        elif key == "nsteps":
            param["nSteps"] = c_atoi(need(toks, 1))
        elif key == "ewald":
            sub = need(toks, 1).lower()
            if sub == "prec":
                ewald["prec"] = c_atof(need(toks, 2))
            elif sub == "alpha":
                ctrl["keyAlpha"] = 1
                ewald["alpha"] = c_atof(need(toks, 2))
            elif sub == "nbsp":
                ewald["nbsp"] = c_atoi(need(toks, 2))
            elif sub == "recvec":
                ctrl["keyMmax"] = 1
                ewald["m1max"] = _c_int(c_atof(need(toks, 2)))
                ewald["m2max"] = _c_int(c_atof(need(toks, 3)))
                ewald["m3max"] = _c_int(c_atof(need(toks, 4)))
            else:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: ewald {sub}")
        elif key == "elec":
            sub = need(toks, 1).lower()
            table = dict(noelec=NOELEC, full=FULL, shift1=SHIFT1, shift2=SHIFT2, switch=SWITCH)
            if sub in table:
                ctrl["elecType"] = table[sub]
            elif sub == "ewald":
                ctrl["keyEwald"] = 1
            elif sub == "spme":
                ctrl["keyEwald"] = 2
            else:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: elec {sub}")
        elif key == "vdw":
            sub = need(toks, 1).lower()
            table = dict(novdw=NOVDW, full=VFULL, switch=VSWITCH)
            if sub not in table:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: vdw {sub}")
            ctrl["vdwType"] = table[sub]
        elif key == "nb14":
            ctrl["keyNb14"] = 1
            param["scal14"] = c_atof(need(toks, 1))
        elif key == "numforce":
            ctrl["keyNumForce"] = 1
        elif key == "list":
            neigh["update"] = c_atoi(need(toks, 1))
        elif key == "link":
            neigh["linkRatio"] = c_atoi(need(toks, 1))
        elif key == "nolink":
            ctrl["noLink"] = 1
        elif key == "integrator":
            sub = need(toks, 1).lower()
            if sub not in ("leapfrog", "velocity"):
                raise MdbasFileError(f"SIMU_PARAM_ERROR: integrator {sub}")
            ctrl["integrator"] = LEAPFROG if sub == "leapfrog" else VELOCITY
        elif key == "ensemble":
            sub = need(toks, 1).lower()
            if sub == "nve":
                ctrl["ens"] = NVE
            elif sub in ("nvt", "npt"):
                th = need(toks, 2).lower()
                if th not in ("beren", "hoover"):
                    raise MdbasFileError(f"SIMU_PARAM_ERROR: {sub} {th}")
                ctrl["ens"] = {("nvt", "beren"): NVT_B, ("nvt", "hoover"): NVT_H,
                               ("npt", "beren"): NPT_B, ("npt", "hoover"): NPT_H}[(sub, th)]
            else:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: ensemble {sub}")
        elif key == "taut":
            bath["tauT"] = c_atof(need(toks, 1))
        elif key == "taup":
            bath["tauP"] = c_atof(need(toks, 1))
        elif key == "pressure":
            param["press0"] = c_atof(need(toks, 1)) * BAR_TO_IU
        elif key == "compressibility":
            bath["compress"] = c_atof(need(toks, 1)) / BAR_TO_IU
        elif key == "consth":
            ctrl["keyConstH"] = 1
        elif key == "shake":
            sub = need(toks, 1).lower()
            if sub == "tol":
                param["tolShake"] = c_atof(need(toks, 2))
            elif sub == "maxcycle":
                param["maxCycle"] = c_atoi(need(toks, 2))
            else:
                raise MdbasFileError(f"SIMU_PARAM_ERROR: shake {sub}")
        elif key == "seed":
            ctrl["keyRand"] = 1
            ctrl["seed"] = c_atoi(need(toks, 1))
        elif key == "print":
            ctrl["printOut"] = c_atoi(need(toks, 1))
        elif key == "prop":
            ctrl["keyProp"] = 1
            ctrl["printProp"] = c_atoi(need(toks, 1))
        elif key == "traj":
            ctrl["keyTraj"] = 1
            ctrl["printTraj"] = c_atoi(need(toks, 1))
        elif key == "resconf":
            ctrl["printRest"] = c_atoi(need(toks, 1))
        elif key == "write":
            sub = need(toks, 1).lower()
            if sub != "field":
                raise MdbasFileError(f"SIMU_PARAM_ERROR: write {sub}")
            ctrl["keyForF"] = 1
        elif key == "pbc":
            box_type = c_atoi(need(toks, 1))
            for r in range(3):
                if li >= len(lines):
                    raise MdbasFileError("SIMU_NOTFOUND_ERROR: pbc row missing")
                row = _tokens(lines[li])
                li += 1
                if len(row) < 3:
                    raise MdbasFileError("SIMU_NOTFOUND_ERROR: pbc row needs 3 values")
                for c in range(3):
                    if not row[c][0].isdigit():
                        raise MdbasFileError(f"SIMU_PARAM_ERROR: pbc value {row[c]!r}")
                    cell[3 * r + c] = c_atof(row[c])
        elif key == "end":
            break
        else:
            raise MdbasFileError(f"SIMU_KEYWORD_ERROR: {toks[0]}")
    # derived terms (src/io.c:715-724)
    param["rcutOff"] = 1. / param["cutOff"]
    param["cutOff2"] = param["cutOff"] * param["cutOff"]
    param["rcutOff2"] = 1. / param["cutOff2"]
    param["cutOn2"] = param["cutOn"] * param["cutOn"]
    d = param["cutOff2"] - param["cutOn2"]
    param["switch2"] = 1. / ((d * d) * d) if d != 0 else math.inf
    param["rTimeStep"] = 1. / param["timeStep"]
    return Simu(ctrl, param, ewald, neigh, bath, box_type, cell, files)


def write_simu(path: str, cell, box_type: int = CUBIC, lines: list[str] | None = None) -> None:
    """A SIMU file: the given keyword lines, then the "pbc" block, then
    "end" (values written with 17 significant digits)."""
    with open(path, "w") as fh:
        for ln in lines or []:
            fh.write(ln.rstrip("\n") + "\n")
        c = [float(v) for v in cell]
        fh.write(f"pbc {int(box_type)}\n")
        for r in range(3):
            fh.write(" ".join(f"{v:.17g}" for v in c[3 * r:3 * r + 3]) + "\n")
        fh.write("end\n")


# ---------------------------------------------------------------------------
# CONF / RCON
# ---------------------------------------------------------------------------
@dataclass
class Conf:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    ires: np.ndarray          # residue number within the system
    resi: np.ndarray          # residue number within the segment
    label: list = field(default_factory=list)   # atom names (<= 4 chars)
    resn: list = field(default_factory=list)    # residue names
    segn: list = field(default_factory=list)    # segment names
    weight: np.ndarray | None = None

    @property
    def n(self) -> int:
        return len(self.x)


class _Scan:
    """fscanf conversions over a string (whitespace skipping, %d, %Ns, %lf)."""

    def __init__(self, text: str):
        self.t = text
        self.p = 0

    def _ws(self):
        while self.p < len(self.t) and self.t[self.p] in " \t\n\v\f\r":
            self.p += 1

    def d(self) -> int:
        self._ws()
        m = re.compile(r"[+-]?\d+").match(self.t, self.p)
        if not m:
            raise MdbasFileError(f"CONF: integer expected at offset {self.p}")
        self.p = m.end()
        return int(m.group(0))

    def s(self, width: int) -> str:
        self._ws()
        q = self.p
        while q < len(self.t) and q - self.p < width and self.t[q] not in " \t\n\v\f\r":
            q += 1
        if q == self.p:
            raise MdbasFileError(f"CONF: string expected at offset {self.p}")
        out = self.t[self.p:q]
        self.p = q
        return out

    def lf(self) -> float:
        self._ws()
        m = re.compile(r"[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)",
                       re.IGNORECASE).match(self.t, self.p)
        if not m:
            raise MdbasFileError(f"CONF: number expected at offset {self.p}")
        self.p = m.end()
        return float(m.group(0))


def read_conf(path: str) -> Conf:
    """read_CONF (src/io.c:728-783): '*' title lines, the atom count, then
    per atom "%d %d %4s %4s %lf %lf %lf %4s %d %lf" (number, residue number,
    residue name, atom name, x, y, z, segment name, residue id, weight)."""
    with open(path, "r", encoding="latin-1") as fh:
        text = fh.read()
    pos = 0
    header = None
    while pos < len(text):
        end = text.find("\n", pos)
        end = len(text) if end < 0 else end + 1
        line = text[pos:end]
        pos = end
        if not line.startswith("*"):
            header = line
            break
    if header is None or not _tokens(header):
        raise MdbasFileError("CONF_FILE_ERROR: no atom count")
    n = c_atoi(_tokens(header)[0])
    sc = _Scan(text[pos:])
    x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
    ires, resi, wei = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
    label, resn, segn = [], [], []
    for i in range(n):
        sc.d()
        ires[i] = sc.d()
        resn.append(sc.s(4))
        label.append(sc.s(4))
        x[i], y[i], z[i] = sc.lf(), sc.lf(), sc.lf()
        segn.append(sc.s(4))
        resi[i] = sc.d()
        wei[i] = sc.lf()
    return Conf(x, y, z, ires, resi, label, resn, segn, wei)


def write_conf(path: str, conf: Conf) -> None:
    """write_CONF (src/io.c:1201-1228): three title lines, "%5d" atom count,
    per atom "%5d%5d %-4s %-4s%10.5lf%10.5lf%10.5lf %-4s %-4d%10.5lf" (weight
    0), with a blank between the first two numbers when they would touch."""
    with open(path, "w") as fh:
        fh.write("*Restart Configuration\n* Written by MDBas\n*\n")
        fh.write(f"{conf.n:5d}\n")
        for i in range(conf.n):
            a, r = i + 1, int(conf.ires[i])
            head = f"{a:5d}{r:5d}" if (a < 100000 and -1000 < r < 10000) else f"{a:5d} {r:5d}"
            fh.write(f"{head} {conf.resn[i]:<4s} {conf.label[i]:<4s}{conf.x[i]:10.5f}"
                     f"{conf.y[i]:10.5f}{conf.z[i]:10.5f} {conf.segn[i]:<4s} "
                     f"{int(conf.resi[i]):<4d}{0.0:10.5f}\n")


# ---------------------------------------------------------------------------
# FORF
# ---------------------------------------------------------------------------
@dataclass
class Forf:
    """read_FORF's per-atom arrays (MDBas's units) and topology."""
    type: np.ndarray
    q: np.ndarray
    mass: np.ndarray
    frozen: np.ndarray
    eps: np.ndarray       # sqrt(eps_kcal * 418.4)
    sig: np.ndarray       # as given (MDBas's Rmin/2 convention)
    eps14: np.ndarray
    sig14: np.ndarray
    n_at_const: np.ndarray
    constraints: tuple    # (pairs (m, 2) int32, squared lengths (m,))
    bonded: dict          # mdbas_b200.nb.bonded_structs spec, internal units, radians


def read_forf(path: str, n_atom: int) -> Forf:
    """read_FORF (src/io.c:872-1199).  Section keywords are case-blind
    ("atoms", "bonds", "constraints", "urey-bradley", "angles", "dihedrals",
    "impropers", "vdw", "end"); '#' lines are comments; atom indices are
    1-based in the file; force constants are in kcal/mol and converted with
    418.4, angles in degrees."""
    n = n_atom
    out = dict(type=np.zeros(n, np.int32), q=np.zeros(n), mass=np.zeros(n),
               frozen=np.zeros(n, np.int32), eps=np.zeros(n), sig=np.zeros(n),
               eps14=np.zeros(n), sig14=np.zeros(n), nat=np.zeros(n, np.int32))
    cons_pairs, cons_len2 = [], []
    spec = {}
    with open(path, "r", encoding="latin-1") as fh:
        lines = fh.read().split("\n")
    li = 0

    def body(count, err):
        """the next `count` non-comment lines (fgets, not lower-cased)"""
        nonlocal li
        got = []
        while len(got) < count:
            if li >= len(lines) or (li == len(lines) - 1 and lines[li] == ""):
                raise MdbasFileError(err)
            ln = lines[li]
            li += 1
            if ln.startswith("#"):
                continue
            t = _tokens(ln)
            if not t:
                raise MdbasFileError(f"{err}: blank line in a section")
            got.append(t)
        return got

    def tok(t, i, err):
        if len(t) <= i:
            raise MdbasFileError(f"{err}: field {i + 1} missing in {' '.join(t)!r}")
        return t[i]

    while li < len(lines):
        head = lines[li].lower()
        li += 1
        if head.startswith("#"):
            continue
        toks = _tokens(head)
        if not toks:
            if li >= len(lines):
                break
            raise MdbasFileError("FORF: blank line (MDBas reads no keyword from it)")
        key = toks[0]
        cnt = c_atoi(toks[1]) if len(toks) > 1 else 0
        if key == "atoms":
            if cnt != n:
                raise MdbasFileError(f"CONF_ATNUM_ERROR: FORF has {cnt} atoms, CONF {n}")
            for k, t in enumerate(body(n, "PSF_BADLINE_ERROR")):
                if c_atoi(tok(t, 0, "PSF_FILE_ERROR")) - 1 != k:
                    raise MdbasFileError("PSF_FILE_ERROR: atoms out of order")
                out["type"][k] = c_atoi(tok(t, 2, "PSF_FILE_ERROR"))
                out["q"][k] = c_atof(tok(t, 3, "PSF_FILE_ERROR"))
                out["mass"][k] = c_atof(tok(t, 4, "PSF_FILE_ERROR"))
                fr = c_atoi(tok(t, 5, "PSF_FILE_ERROR"))
                if fr not in (0, 1):
                    raise MdbasFileError("error 21: frozen flag must be 0 or 1")
                out["frozen"][k] = fr
                out["nat"][k] = 0
        elif key == "bonds":
            rows = body(cnt, "PSF_BOND_SEQ_ERROR")
            spec["bonds"] = dict(
                atoms=np.array([[c_atoi(t[0]) - 1, c_atoi(t[1]) - 1] for t in rows],
                               np.int32).reshape(-1, 2),
                type=np.array([c_atoi(tok(t, 2, "PSF_BOND_SEQ_ERROR")) for t in rows], np.int32),
                k=np.array([c_atof(tok(t, 3, "PSF_BOND_SEQ_ERROR")) * KCAL_TO_IU for t in rows]),
                r0=np.array([c_atof(tok(t, 4, "PSF_BOND_SEQ_ERROR")) for t in rows]),
                beta=np.array([c_atof(tok(t, 5, "PSF_BOND_SEQ_ERROR")) for t in rows]))
        elif key == "constraints":
            for t in body(cnt, "error 27"):
                a, b = c_atoi(t[0]) - 1, c_atoi(tok(t, 1, "error 27")) - 1
                r = c_atof(tok(t, 2, "error 27"))
                cons_pairs.append((a, b))
                cons_len2.append(r * r)
                out["nat"][a] += 1
                out["nat"][b] += 1
        elif key == "urey-bradley":
            rows = body(cnt, "error 28")
            spec["ub"] = dict(
                atoms=np.array([[c_atoi(t[0]) - 1, c_atoi(tok(t, 1, "error 28")) - 1]
                                for t in rows], np.int32).reshape(-1, 2),
                type=np.zeros(len(rows), np.int32),
                k=np.array([c_atof(tok(t, 2, "error 28")) * KCAL_TO_IU for t in rows]),
                r0=np.array([c_atof(tok(t, 3, "error 28")) for t in rows]),
                beta=np.array([c_atof(tok(t, 4, "error 28")) for t in rows]))
        elif key == "angles":
            rows = body(cnt, "PSF_ANGL_SEQ_ERROR")
            e = "PSF_ANGL_SEQ_ERROR"
            spec["angles"] = dict(
                atoms=np.array([[c_atoi(t[0]) - 1, c_atoi(tok(t, 1, e)) - 1,
                                 c_atoi(tok(t, 2, e)) - 1] for t in rows], np.int32).reshape(-1, 3),
                type=np.array([c_atoi(tok(t, 3, e)) for t in rows], np.int32),
                k=np.array([c_atof(tok(t, 4, e)) * KCAL_TO_IU for t in rows]),
                theta0=np.array([c_atof(tok(t, 5, e)) * PI / 180. for t in rows]))
        elif key in ("dihedrals", "impropers"):
            e = "PSF_DIHE_SEQ_ERROR" if key == "dihedrals" else "PSF_IMPR_SEQ_ERROR"
            rows = body(cnt, e)
            spec[key] = dict(
                atoms=np.array([[c_atoi(tok(t, c, e)) - 1 for c in range(4)] for t in rows],
                               np.int32).reshape(-1, 4),
                type=np.array([c_atoi(tok(t, 4, e)) for t in rows], np.int32),
                order=np.array([c_atoi(tok(t, 5, e)) for t in rows], np.int32),
                k=np.array([c_atof(tok(t, 6, e)) * KCAL_TO_IU for t in rows]),
                phi0=np.array([c_atof(tok(t, 7, e)) * PI / 180. for t in rows]),
                mult=np.array([c_atof(tok(t, 8, e)) for t in rows]))
        elif key == "vdw":
            if cnt != n:
                raise MdbasFileError(f"CONF_ATNUM_ERROR: FORF vdw has {cnt} atoms, CONF {n}")
            for k, t in enumerate(body(n, "PSF_BADLINE_ERROR")):
                if c_atoi(t[0]) - 1 != k:
                    raise MdbasFileError("PSF_FILE_ERROR: vdw out of order")
                e = "PSF_FILE_ERROR"
                out["eps"][k] = math.sqrt(c_atof(tok(t, 2, e)) * KCAL_TO_IU)
                out["sig"][k] = c_atof(tok(t, 3, e))
                out["eps14"][k] = math.sqrt(c_atof(tok(t, 5, e)) * KCAL_TO_IU)
                out["sig14"][k] = c_atof(tok(t, 6, e))
        elif key == "end":
            break
        else:
            raise MdbasFileError(f"error 29: unknown FORF section {key!r}")
    cons = (np.array(cons_pairs, np.int32).reshape(-1, 2), np.array(cons_len2, np.float64))
    return Forf(out["type"], out["q"], out["mass"], out["frozen"], out["eps"], out["sig"],
                out["eps14"], out["sig14"], out["nat"], cons, spec)


def write_forf(path: str, labels, types, q, mass, frozen, eps_kcal, sig, eps14_kcal=None,
               sig14=None, bonded: dict | None = None, constraints=None) -> None:
    """A FORF file read_FORF reads back to the given values: force constants
    of `bonded` (internal units, radians, as in nb.bonded_structs specs)
    are written in kcal/mol and degrees with 17 significant digits."""
    n = len(q)
    eps14_kcal = eps_kcal if eps14_kcal is None else eps14_kcal
    sig14 = sig if sig14 is None else sig14
    g = lambda v: f"{float(v):.17g}"
    with open(path, "w") as fh:
        fh.write("# force field written by mdbas_b200.mdbas_files\n")
        fh.write(f"atoms {n}\n")
        for i in range(n):
            fh.write(f"{i + 1} {labels[i]} {int(types[i])} {g(q[i])} {g(mass[i])} "
                     f"{int(frozen[i])}\n")
        b = bonded or {}
        if "bonds" in b:
            t = b["bonds"]
            m = len(t["atoms"])
            fh.write(f"bonds {m}\n")
            for k in range(m):
                a = t["atoms"][k]
                fh.write(f"{a[0] + 1} {a[1] + 1} {int(t['type'][k]) if 'type' in t else 0} "
                         f"{g(t['k'][k] / KCAL_TO_IU)} {g(t['r0'][k])} "
                         f"{g(t['beta'][k] if 'beta' in t else 0.0)}\n")
        if constraints is not None and len(constraints[1]):
            pairs, len2 = constraints
            fh.write(f"constraints {len(len2)}\n")
            for k in range(len(len2)):
                fh.write(f"{pairs[k][0] + 1} {pairs[k][1] + 1} {g(math.sqrt(len2[k]))}\n")
        if "ub" in b:
            t = b["ub"]
            m = len(t["atoms"])
            fh.write(f"urey-bradley {m}\n")
            for k in range(m):
                a = t["atoms"][k]
                fh.write(f"{a[0] + 1} {a[1] + 1} {g(t['k'][k] / KCAL_TO_IU)} {g(t['r0'][k])} "
                         f"{g(t['beta'][k] if 'beta' in t else 0.0)}\n")
        if "angles" in b:
            t = b["angles"]
            m = len(t["atoms"])
            fh.write(f"angles {m}\n")
            for k in range(m):
                a = t["atoms"][k]
                fh.write(f"{a[0] + 1} {a[1] + 1} {a[2] + 1} "
                         f"{int(t['type'][k]) if 'type' in t else 0} "
                         f"{g(t['k'][k] / KCAL_TO_IU)} {g(t['theta0'][k] * 180. / PI)}\n")
        for key in ("dihedrals", "impropers"):
            if key in b:
                t = b[key]
                m = len(t["atoms"])
                fh.write(f"{key} {m}\n")
                for k in range(m):
                    a = t["atoms"][k]
                    typ = int(t["type"][k]) if "type" in t else 1
                    order = int(t["order"][k]) if "order" in t else 0
                    mult = t["mult"][k] if "mult" in t else 1.0
                    fh.write(f"{a[0] + 1} {a[1] + 1} {a[2] + 1} {a[3] + 1} {typ} {order} "
                             f"{g(t['k'][k] / KCAL_TO_IU)} {g(t['phi0'][k] * 180. / PI)} "
                             f"{g(mult)}\n")
        fh.write(f"vdw {n}\n")
        for i in range(n):
            fh.write(f"{i + 1} {int(types[i])} {g(eps_kcal[i])} {g(sig[i])} 0 "
                     f"{g(eps14_kcal[i])} {g(sig14[i])} 0\n")
        fh.write("end\n")


# ---------------------------------------------------------------------------
# REST (binary restart), PROP, DCD
# ---------------------------------------------------------------------------
@dataclass
class Rest:
    step: int
    atoms: list            # (label, segn, resn, type, resi, ires) per atom
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    fx: np.ndarray
    fy: np.ndarray
    fz: np.ndarray
    energy: dict
    chiT: float
    chiP: float
    atom_bytes: bytes | None = None  # the ATOM records as read (padding included)


def _cstr(b: bytes) -> str:
    return b.split(b"\0", 1)[0].decode("latin-1")


def read_rest(path: str) -> Rest:
    """read_rest (src/io.c:785-870): native-endian int step and atom count,
    ATOM records, nine double arrays, the ENERGY struct, chiT, chiP."""
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < 8:
        raise MdbasFileError("error 502: truncated restart file")
    step, n = struct.unpack_from("<ii", data, 0)
    p = 8
    need = p + n * ATOM_STRUCT.size + 9 * 8 * n + 8 * len(ENERGY_FIELDS) + 16
    if n < 0 or len(data) < need:
        raise MdbasFileError("error 502: truncated restart file")
    atoms = []
    raw = data[p:p + n * ATOM_STRUCT.size]
    for i in range(n):
        lab, seg, res, typ, resi, ires = ATOM_STRUCT.unpack_from(data, p)
        atoms.append((_cstr(lab), _cstr(seg), _cstr(res), typ, resi, ires))
        p += ATOM_STRUCT.size
    arrs = []
    for _ in range(9):
        arrs.append(np.frombuffer(data, dtype="<f8", count=n, offset=p).copy())
        p += 8 * n
    en = struct.unpack_from("<" + "d" * len(ENERGY_FIELDS), data, p)
    p += 8 * len(ENERGY_FIELDS)
    chiT, chiP = struct.unpack_from("<dd", data, p)
    return Rest(step, atoms, *arrs, dict(zip(ENERGY_FIELDS, en)), chiT, chiP, raw)


def write_rest(path: str, rest: Rest) -> None:
    """write_rest (src/io.c:1276-1369), byte for byte: the ATOM records as
    read when `atom_bytes` holds them (MDBas writes its structs' padding
    byte as it finds it), else packed from `atoms` with zero padding."""
    n = len(rest.x)
    with open(path, "wb") as fh:
        fh.write(struct.pack("<ii", int(rest.step), n))
        if rest.atom_bytes is not None and len(rest.atom_bytes) == n * ATOM_STRUCT.size:
            fh.write(rest.atom_bytes)
        for lab, seg, res, typ, resi, ires in (rest.atoms if rest.atom_bytes is None or
                                               len(rest.atom_bytes) != n * ATOM_STRUCT.size
                                               else []):
            fh.write(ATOM_STRUCT.pack(lab.encode("latin-1")[:4], seg.encode("latin-1")[:4],
                                      res.encode("latin-1")[:4], int(typ), int(resi),
                                      int(ires)))
        for a in (rest.x, rest.y, rest.z, rest.vx, rest.vy, rest.vz, rest.fx, rest.fy, rest.fz):
            fh.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        fh.write(struct.pack("<" + "d" * len(ENERGY_FIELDS),
                             *[float(rest.energy.get(k, 0.0)) for k in ENERGY_FIELDS]))
        fh.write(struct.pack("<dd", float(rest.chiT), float(rest.chiP)))


def _lattice(pbc) -> list[float]:
    """box_to_lattice (src/utils.c:456-473): a, b, c and the angles (deg)."""
    def ang(u1, u2, u3, v1, v2, v3, lu, lv):
        return math.acos(((u1 * v1) + (u2 * v2) + (u3 * v3)) / (lu * lv)) * 180. / PI
    return [pbc.a, pbc.b, pbc.c,
            ang(pbc.b1, pbc.b2, pbc.b3, pbc.c1, pbc.c2, pbc.c3, pbc.b, pbc.c),
            ang(pbc.a1, pbc.a2, pbc.a3, pbc.c1, pbc.c2, pbc.c3, pbc.a, pbc.c),
            ang(pbc.a1, pbc.a2, pbc.a3, pbc.b1, pbc.b2, pbc.b3, pbc.a, pbc.b)]


def prop_record(step: int, time_step: float, n_deg_free: int, energy: dict, pbc) -> np.ndarray:
    """The 29 doubles write_prop appends (src/io.c:1230-1274): step, time,
    temperature, pressure, volume, energies and virials in kcal/mol,
    conserved quantity, lattice a b c alpha beta gamma."""
    e = {k: float(energy.get(k, 0.0)) for k in ENERGY_FIELDS}
    buf = np.zeros(29)
    temp = 2. * e["kin"] / (float(n_deg_free) * RBOLTZ_IU)
    press = (2. * e["kin"] - e["virtot"]) / (3. * pbc.vol * BAR_TO_IU) if pbc.type > 0 else 0.
    buf[0] = float(step)
    buf[1] = float(step) * time_step
    buf[2] = temp
    buf[3] = press
    buf[4] = pbc.vol
    for i, k in enumerate(("tot", "kin", "pot", "elec", "vdw", "bond", "ang", "ub", "dihe",
                           "impr", "virtot", "virpot", "virelec", "virvdw", "virbond", "virub",
                           "virshake", "consv")):
        buf[5 + i] = e[k] / KCAL_TO_IU
    buf[23:29] = _lattice(pbc)
    return buf


def write_prop(path: str, step: int, time_step: float, n_deg_free: int, energy: dict,
               pbc) -> None:
    """Append one PROP record (write_prop, src/io.c:1230-1274)."""
    with open(path, "ab") as fh:
        fh.write(prop_record(step, time_step, n_deg_free, energy, pbc).astype("<f8").tobytes())


def _record(fh, payload: bytes) -> None:
    fh.write(struct.pack("<I", len(payload)))
    fh.write(payload)
    fh.write(struct.pack("<I", len(payload)))


def write_dcd_header(path: str, n_steps: int, print_traj: int, n_deg_free: int, frozen,
                     box_type: int, titles: list[str] | None = None) -> None:
    """write_DCD_header (src/io.c:1371-1460): CORD + ICNTRL[20], three
    80-character titles (by default MDBas's: creation date, user and host,
    working directory), NATOM and, with frozen atoms, the free atoms' list."""
    frozen = np.asarray(frozen, dtype=np.int32)
    natom = len(frozen)
    nfrozen = int((frozen != 0).sum())
    icntrl = [0] * 20
    icntrl[0] = int(n_steps / print_traj) if print_traj else 0
    icntrl[1] = print_traj
    icntrl[2] = print_traj
    icntrl[3] = n_steps
    icntrl[7] = n_deg_free
    icntrl[8] = nfrozen
    icntrl[10] = 0 if box_type == NOBOX else 1
    icntrl[19] = 37
    if titles is None:
        titles = [f"* CREATION DATE : {time.asctime()}\n",
                  f"* USER : {os.environ.get('USER', 'UNKNOWN')} HOSTNAME : "
                  f"{os.environ.get('HOSTNAME', 'UNKNOWN')}",
                  f"* PWD : {os.environ.get('PWD', 'UNKNOWN')}"]
    tb = [t.encode("latin-1")[:79].ljust(80, b"\0") for t in titles]
    with open(path, "wb") as fh:
        _record(fh, b"CORD" + struct.pack("<20i", *icntrl))
        _record(fh, struct.pack("<i", 3) + b"".join(tb))
        _record(fh, struct.pack("<i", natom))
        if nfrozen:
            free = np.nonzero(frozen == 0)[0].astype("<i4")
            _record(fh, free.tobytes())


def write_dcd_frame(path: str, pbc, x, y, z, frozen, first: bool) -> None:
    """write_DCD_traj (src/io.c:1462-1520): the box (a1 a2 b2 a3 b3 c3) when
    periodic, then x, y, z in FP32 -- every atom in the first frame, the free
    atoms after it."""
    frozen = np.asarray(frozen, dtype=np.int32)
    sel = np.ones(len(frozen), bool) if first else (frozen == 0)
    with open(path, "ab") as fh:
        if pbc.type != NOBOX:
            _record(fh, struct.pack("<6d", pbc.a1, pbc.a2, pbc.b2, pbc.a3, pbc.b3, pbc.c3))
        for a in (x, y, z):
            _record(fh, np.asarray(a, dtype=np.float64)[sel].astype("<f4").tobytes())


# ---------------------------------------------------------------------------
# A run's system from MDBas's files
# ---------------------------------------------------------------------------
def load(simu_path: str, base_dir: str | None = None):
    """(System, Simu, Conf, Forf) of a MDBas run: the SIMU file, and the CONF
    and FORF files it names.  The System carries MDBas's per-atom q, eps,
    sig, masses, bonds and angles, and in meta the box rows and type
    ("cell", "box_type"), the bonded spec ("bonded"), constraints
    ("constraints"), frozen atoms ("frozen") and the dihedral quadruples."""
    from .systems import System
    simu = read_simu(simu_path)
    base = os.path.dirname(os.path.abspath(simu_path)) if base_dir is None else base_dir

    def where(name):
        return name if os.path.isabs(name) else os.path.join(base, name)

    conf = read_conf(where(simu.files["conf"]))
    forf = read_forf(where(simu.files["forf"]), conf.n)
    bonds = forf.bonded.get("bonds", {}).get("atoms", np.zeros((0, 2), np.int32))
    angles = forf.bonded.get("angles", {}).get("atoms", np.zeros((0, 3), np.int32))
    edge = float(simu.cell[0]) if simu.box_type in (CUBIC, ORBIC, TCLIN) else 0.0
    meta = {"cell": simu.cell.copy(), "box_type": simu.box_type, "bonded": forf.bonded,
            "constraints": forf.constraints, "frozen": forf.frozen.copy(),
            "dihedrals": forf.bonded.get("dihedrals", {}).get("atoms",
                                                              np.zeros((0, 4), np.int32)),
            "impropers": forf.bonded.get("impropers", {}).get("atoms",
                                                              np.zeros((0, 4), np.int32)),
            "source": os.path.abspath(simu_path)}
    s = System(os.path.basename(simu_path), edge, conf.x.copy(), conf.y.copy(), conf.z.copy(),
               forf.q.copy(), forf.eps.copy(), forf.sig.copy(), forf.mass.copy(),
               np.ascontiguousarray(bonds, np.int32), np.ascontiguousarray(angles, np.int32),
               types=forf.type.copy(), meta=meta)
    return s, simu, conf, forf
