"""TEST INFRASTRUCTURE ONLY: numpy restatement of MDBas's bonded terms
(src/internal.c), a checker of the GPU bonded kernels
(mdbas_b200/csrc/bonded.cu) beside MDBas's own compiled routines
(oracle/_ref).

Per kind, vectorised over terms, with MDBas's formulas:

* bond_energy (src/internal.c:21-105): harmonic E = k/2 (r - r0)^2 or Morse
  E = k (e^{-2b(r-r0)} - 2 e^{-b(r-r0)}) + k; virial sum dE/dr * r;
* ub_energy (src/internal.c:107-171): harmonic in the 1-3 distance;
* angle_energy (src/internal.c:173-256): E = k/2 (theta - theta0)^2 with
  sin(theta) floored at 1e-8 in the force;
* dihedral_energy / improper_energy (src/internal.c:258-620): the angle phi
  between the normals of (i,j,k) and (j,k,l) by atan2; cosine E = k (1 +
  cos(m phi - phi0)) or harmonic E = k/2 (phi - phi0)^2 (wrapped to
  [-pi, pi]); sin(phi) floored at DBL_EPSILON in the force.

Minimum image as MDBas's dist() for cubic and orthorhombic boxes.  Forces
are summed with np.add.at, so they agree with MDBas to rounding (not bit
for bit).  Pinned against MDBas itself by tests/test_bonded_oracle.py.
"""
from __future__ import annotations

import math

import numpy as np

DBL_EPSILON = np.finfo(np.float64).eps


def _nint(x):
    """MDBas nint (src/utils.c:606-609): round half away from zero."""
    return np.where(x >= 0, np.trunc(x + 0.5), np.trunc(x - 0.5))


def _image(d, lengths):
    """dist() of src/utils.c for cubic/orthorhombic boxes; d is (m, 3)."""
    L = np.asarray(lengths, dtype=np.float64)
    return d - L * _nint(d / L)


def _pos(x, y, z):
    return np.stack([np.asarray(x, np.float64), np.asarray(y, np.float64),
                     np.asarray(z, np.float64)], 1)


def _scatter(n, atoms, forces):
    f = np.zeros((n, 3))
    for p in range(atoms.shape[1]):
        np.add.at(f, atoms[:, p], forces[p])
    return f


def bonds(t: dict, x, y, z, lengths, ub: bool = False):
    """(energy, virial, forces (n, 3)) of bond_energy (or ub_energy)."""
    r_ = _pos(x, y, z)
    a = np.asarray(t["atoms"], dtype=np.int64)
    if len(a) == 0:
        return 0.0, 0.0, np.zeros_like(r_)
    d = _image(r_[a[:, 1]] - r_[a[:, 0]], lengths)
    r = np.sqrt((d * d).sum(1))
    k = np.asarray(t["k"], np.float64)
    dr = r - np.asarray(t["r0"], np.float64)
    typ = np.zeros(len(a), np.int64) if ub or "type" not in t else np.asarray(t["type"])
    morse = typ == 1
    beta = np.asarray(t.get("beta", np.zeros(len(a))), np.float64)
    ma = np.exp(-beta * dr)
    mb = ma * ma
    e = np.where(morse, k * (mb - 2.0 * ma) + k, 0.5 * k * dr * dr)
    db = np.where(morse, 2.0 * k * beta * (ma - mb), k * dr)
    tf = (db / r)[:, None] * d
    f = _scatter(len(r_), a, [tf, -tf])
    return float(e.sum()), float((db * r).sum()), f


def angles(t: dict, x, y, z, lengths):
    """(energy, forces (n, 3)) of angle_energy."""
    r_ = _pos(x, y, z)
    a = np.asarray(t["atoms"], dtype=np.int64)
    if len(a) == 0:
        return 0.0, np.zeros_like(r_)
    dab = _image(r_[a[:, 0]] - r_[a[:, 1]], lengths)
    dbc = _image(r_[a[:, 2]] - r_[a[:, 1]], lengths)
    rab = np.sqrt((dab * dab).sum(1))
    rbc = np.sqrt((dbc * dbc).sum(1))
    cost = (dab * dbc).sum(1) / (rab * rbc)
    sint = np.maximum(1e-8, np.sqrt(1.0 - cost * cost))
    theta = np.arccos(cost)
    k = np.asarray(t["k"], np.float64)
    dt = theta - np.asarray(t["theta0"], np.float64)
    e = 0.5 * k * dt * dt
    da = (k * dt / sint)[:, None]
    fa = da * (dbc / rbc[:, None] - dab * (cost / rab)[:, None]) / rab[:, None]
    fc = da * (dab / rab[:, None] - dbc * (cost / rbc)[:, None]) / rbc[:, None]
    f = _scatter(len(r_), a, [fa, -fa - fc, fc])
    return float(e.sum()), f


def torsions(t: dict, x, y, z, lengths):
    """(energy, forces (n, 3)) of dihedral_energy / improper_energy."""
    r_ = _pos(x, y, z)
    a = np.asarray(t["atoms"], dtype=np.int64)
    if len(a) == 0:
        return 0.0, np.zeros_like(r_)
    dab = _image(r_[a[:, 0]] - r_[a[:, 1]], lengths)
    dbc = _image(r_[a[:, 1]] - r_[a[:, 2]], lengths)
    dcd = _image(r_[a[:, 2]] - r_[a[:, 3]], lengths)
    rbc = np.sqrt((dbc * dbc).sum(1))
    pb = np.cross(dab, dbc)
    pc = np.cross(dbc, dcd)
    r2pb = (pb * pb).sum(1)
    r2pc = (pc * pc).sum(1)
    rpb, rpc = np.sqrt(r2pb), np.sqrt(r2pc)
    pbpc = (pb * pc).sum(1)
    cosp = pbpc / (rpb * rpc)
    sinp = (dbc * np.cross(pc, pb)).sum(1) / (rpb * rpc * rbc)
    phi = np.arctan2(sinp, cosp)
    sinp = np.where(sinp >= 0, 1.0, -1.0) * np.maximum(DBL_EPSILON, np.abs(sinp))
    k = np.asarray(t["k"], np.float64)
    phi0 = np.asarray(t["phi0"], np.float64)
    mult = np.asarray(t.get("mult", np.ones(len(a))), np.float64)
    typ = np.asarray(t.get("type", np.ones(len(a))), np.int64)
    harm = typ == 2
    ph = phi - phi0
    ph = ph - _nint(ph / (2.0 * math.pi)) * (2.0 * math.pi)
    arg = mult * phi - phi0
    e = np.where(harm, 0.5 * k * ph * ph, k * (1.0 + np.cos(arg)))
    den = rpb * rpc * sinp
    dd = np.where(harm, k * ph / den, -k * mult * np.sin(arg) / den)[:, None]
    # d(pb)/d(r_a) and friends through the cross products, as MDBas writes them
    fa = dd * (np.cross(dbc, pc) - (pbpc / r2pb)[:, None] * np.cross(dbc, pb))
    fc = dd * (np.cross(dab, pc) - (pbpc / r2pb)[:, None] * np.cross(dab, pb))
    fb = dd * (np.cross(dcd, pb) - (pbpc / r2pc)[:, None] * np.cross(dcd, pc))
    fd = dd * (np.cross(dbc, pb) - (pbpc / r2pc)[:, None] * np.cross(dbc, pc))
    f = _scatter(len(r_), a, [fa, -fa - fc + fb, fc - fb - fd, fd])
    return float(e.sum()), f


def all_terms(spec: dict, x, y, z, lengths):
    """Energies (bond, angle, ub, dihedral, improper, vir_bond, vir_ub) and
    total forces (n, 3) of a bonded spec (mdbas_b200.nb.bonded_structs)."""
    n = len(x)
    f = np.zeros((n, 3))
    out = dict(bond=0.0, angle=0.0, ub=0.0, dihedral=0.0, improper=0.0, vir_bond=0.0,
               vir_ub=0.0)
    if "bonds" in spec:
        out["bond"], out["vir_bond"], fb = bonds(spec["bonds"], x, y, z, lengths)
        f += fb
    if "angles" in spec:
        out["angle"], fa = angles(spec["angles"], x, y, z, lengths)
        f += fa
    if "ub" in spec:
        out["ub"], out["vir_ub"], fu = bonds(spec["ub"], x, y, z, lengths, ub=True)
        f += fu
    for kind, key in (("dihedrals", "dihedral"), ("impropers", "improper")):
        if kind in spec:
            out[key], ft = torsions(spec[kind], x, y, z, lengths)
            f += ft
    return out, f
