"""Seeded synthetic systems for the nonbonded hot path.

There is no public benchmark suite for this path; every workload is
generated here from a seed, in MDBas's conventions:

* positions in Angstrom, box centred on the origin (MDBas's image_update
  wraps into [-L/2, L/2), src/utils.c:162-218);
* per-atom LJ parameters as read_FORF leaves them: ``eps_i = sqrt(eps *
  418.4)`` (src/io.c:1174) and ``sig_i`` = half the LJ sigma (the CHARMM
  Rmin/2 convention of tools/prepare.c:1999-2000), so that MDBas's
  ``veps = eps_i*eps_j`` and ``vsig = sig_i+sig_j`` (src/energy.c:505-506)
  are Lorentz-Berthelot combinations;
* topology as FORF bonds and angles, from which MDBas's exclusion builders
  (src/list.c:108, :1125) derive the excluded pairs.

Water model (all water workloads): rigid 3-site water, O -0.834 e / H
+0.417 e, LJ on O only (eps 0.1521 kcal/mol, sigma 3.1507 A), O-H 0.9572 A,
H-O-H 104.52 deg.  Molecules: oxygen on the sites of an n^3 lattice
(n = ceil(cbrt(M)), spacing L/n, first M sites in i, j, k order), each
jittered by a seeded uniform +-0.5 A per axis, with a seeded uniform random
orientation.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

KCAL_TO_IU = 418.4                 # include/global.h:41
CHARGE_CONST = 332.0716 * KCAL_TO_IU  # CHARMM, src/init.c:102-103
RBOLTZ_IU = 0.83144621             # include/global.h:49

WATER_Q = (-0.834, 0.417, 0.417)
WATER_EPS_KCAL = 0.1521
WATER_SIGMA = 3.1507
WATER_ROH = 0.9572
WATER_THETA = math.radians(104.52)
WATER_MASS = (15.9994, 1.008, 1.008)
WATER_DENSITY = 0.0334             # molecules / A^3


@dataclass
class System:
    """One periodic system in MDBas's per-atom layout (FP64, original order)."""

    name: str
    box: float                      # cubic edge (A)
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    q: np.ndarray
    eps: np.ndarray                 # sqrt(eps_kcal * 418.4)
    sig: np.ndarray                 # sigma / 2
    mass: np.ndarray
    bonds: np.ndarray               # (nb, 2) int32
    angles: np.ndarray              # (na, 3) int32
    vx: np.ndarray | None = None
    vy: np.ndarray | None = None
    vz: np.ndarray | None = None
    types: np.ndarray | None = None
    type_eps_kcal: np.ndarray | None = None
    type_sigma: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def cell(self) -> np.ndarray:
        """The three box rows a, b, c as MDBas's SIMU "pbc" block holds them
        (meta["cell"] when the box is not a cube of edge `box`)."""
        if self.meta and "cell" in self.meta:
            return np.asarray(self.meta["cell"], dtype=np.float64)
        return np.array([self.box, 0, 0, 0, self.box, 0, 0, 0, self.box], dtype=np.float64)

    def water_constraints(self):
        """Rigid-water constraints (O-H1, O-H2, H1-H2) of every molecule:
        (pairs (3M, 2) int32, squared lengths (3M,))."""
        m = self.n // 3
        base = 3 * np.arange(m, dtype=np.int32)
        pairs = np.stack([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1),
                          np.stack([base + 1, base + 2], 1)], 1).reshape(-1, 2)
        rhh = 2.0 * WATER_ROH * math.sin(0.5 * WATER_THETA)
        lens = np.tile(np.array([WATER_ROH ** 2, WATER_ROH ** 2, rhh ** 2]), m)
        return pairs.astype(np.int32), lens

    def exclusions(self, symmetric: bool = True):
        """Excluded pairs from bonds + angles as CSR (start[n+1], flat).

        Symmetric rows are what link_cell_exclude_list builds; half rows (j>i)
        what exclude_list builds.  Entries keep bond-then-angle order."""
        n = self.n
        rows = [[] for _ in range(n)]

        def add(a, b):
            if b not in rows[a]:
                rows[a].append(b)

        pairs = [tuple(b) for b in self.bonds.tolist()]
        for a, b, c in self.angles.tolist():
            pairs += [(a, b), (a, c), (b, c)]
        for a, b in pairs:
            if symmetric:
                add(a, b)
                add(b, a)
            else:
                add(min(a, b), max(a, b))
        start = np.zeros(n + 1, dtype=np.int32)
        start[1:] = np.cumsum([len(r) for r in rows])
        flat = np.array([v for r in rows for v in r], dtype=np.int32)
        return start, flat


def _random_rotations(rng: np.random.Generator, m: int) -> np.ndarray:
    """m uniform random rotation matrices from uniform unit quaternions."""
    u1, u2, u3 = rng.random((3, m))
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    qw = a * np.sin(2 * np.pi * u2)
    qx = a * np.cos(2 * np.pi * u2)
    qy = b * np.sin(2 * np.pi * u3)
    qz = b * np.cos(2 * np.pi * u3)
    r = np.empty((m, 3, 3))
    r[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    r[:, 0, 1] = 2 * (qx * qy - qz * qw)
    r[:, 0, 2] = 2 * (qx * qz + qy * qw)
    r[:, 1, 0] = 2 * (qx * qy + qz * qw)
    r[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    r[:, 1, 2] = 2 * (qy * qz - qx * qw)
    r[:, 2, 0] = 2 * (qx * qz - qy * qw)
    r[:, 2, 1] = 2 * (qy * qz + qx * qw)
    r[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    return r


def _wrap(v: np.ndarray, box: float) -> np.ndarray:
    return v - box * np.floor(v / box + 0.5)


def water_box(n_molecules: int, box: float, seed: int = 1, jitter: float = 0.5,
              temperature: float | None = None, name: str | None = None) -> System:
    """Lattice-plus-jitter rigid water box (atoms O, H1, H2 per molecule)."""
    rng = np.random.default_rng(seed)
    m = int(n_molecules)
    nl = int(math.ceil(round(m ** (1.0 / 3.0), 9)))
    while nl ** 3 < m:
        nl += 1
    spacing = box / nl
    idx = np.arange(m)
    i = idx % nl
    j = (idx // nl) % nl
    k = idx // (nl * nl)
    centres = np.stack([(i + 0.5) * spacing, (j + 0.5) * spacing, (k + 0.5) * spacing], 1)
    centres -= 0.5 * box
    centres += rng.uniform(-jitter, jitter, size=(m, 3))
    # Body frame: O at origin, H in the xy plane symmetric about x.
    half = 0.5 * WATER_THETA
    body = np.array([[0.0, 0.0, 0.0],
                     [WATER_ROH * math.cos(half), WATER_ROH * math.sin(half), 0.0],
                     [WATER_ROH * math.cos(half), -WATER_ROH * math.sin(half), 0.0]])
    rot = _random_rotations(rng, m)
    pos = centres[:, None, :] + np.einsum('mij,aj->mai', rot, body)
    pos = _wrap(pos.reshape(-1, 3), box)
    n = 3 * m
    q = np.tile(np.array(WATER_Q), m)
    eps = np.tile(np.array([math.sqrt(WATER_EPS_KCAL * KCAL_TO_IU), 0.0, 0.0]), m)
    sig = np.tile(np.array([0.5 * WATER_SIGMA, 0.0, 0.0]), m)
    mass = np.tile(np.array(WATER_MASS), m)
    base = 3 * np.arange(m, dtype=np.int32)
    bonds = np.concatenate([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1)])
    bonds = bonds.reshape(2, m, 2).transpose(1, 0, 2).reshape(-1, 2).astype(np.int32)
    angles = np.stack([base + 1, base, base + 2], 1).astype(np.int32)
    sysm = System(name or f"water{n}", float(box), pos[:, 0].copy(), pos[:, 1].copy(),
                  pos[:, 2].copy(), q, eps, sig, mass, bonds, angles,
                  meta={"molecules": m, "seed": seed})
    if temperature is not None:
        sd = np.sqrt(RBOLTZ_IU * temperature / mass)
        v = rng.normal(size=(n, 3)) * sd[:, None]
        sysm.vx, sysm.vy, sysm.vz = v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy()
    return sysm


def water_box_ortho(lengths, seed: int = 1, jitter: float = 0.5,
                    density: float = WATER_DENSITY, name: str | None = None) -> System:
    """Rigid water filling an orthorhombic box (edges Lx, Ly, Lz): molecule
    centres on a full nx x ny x nz lattice (n_a = round(L_a * density^(1/3)),
    spacing L_a / n_a) with seeded jitter and random orientations, the same
    molecule as water_box.  The box rows are in meta["cell"]."""
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths, dtype=np.float64)
    nl = np.maximum(1, np.rint(L * density ** (1.0 / 3.0)).astype(int))
    spacing = L / nl
    i, j, k = np.meshgrid(np.arange(nl[0]), np.arange(nl[1]), np.arange(nl[2]), indexing="ij")
    centres = (np.stack([i.ravel(), j.ravel(), k.ravel()], 1) + 0.5) * spacing - 0.5 * L
    m = centres.shape[0]
    centres += rng.uniform(-jitter, jitter, size=(m, 3))
    half = 0.5 * WATER_THETA
    body = np.array([[0.0, 0.0, 0.0],
                     [WATER_ROH * math.cos(half), WATER_ROH * math.sin(half), 0.0],
                     [WATER_ROH * math.cos(half), -WATER_ROH * math.sin(half), 0.0]])
    rot = _random_rotations(rng, m)
    pos = (centres[:, None, :] + np.einsum('mij,aj->mai', rot, body)).reshape(-1, 3)
    pos = pos - L * np.floor(pos / L + 0.5)
    q = np.tile(np.array(WATER_Q), m)
    eps = np.tile(np.array([math.sqrt(WATER_EPS_KCAL * KCAL_TO_IU), 0.0, 0.0]), m)
    sig = np.tile(np.array([0.5 * WATER_SIGMA, 0.0, 0.0]), m)
    mass = np.tile(np.array(WATER_MASS), m)
    base = 3 * np.arange(m, dtype=np.int32)
    bonds = np.stack([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1)],
                     1).reshape(-1, 2).astype(np.int32)
    angles = np.stack([base + 1, base, base + 2], 1).astype(np.int32)
    cell = [L[0], 0.0, 0.0, 0.0, L[1], 0.0, 0.0, 0.0, L[2]]
    return System(name or f"water{3 * m}_ortho", float(L[0]), pos[:, 0].copy(),
                  pos[:, 1].copy(), pos[:, 2].copy(), q, eps, sig, mass, bonds, angles,
                  meta={"molecules": m, "seed": seed, "cell": cell})


def water_box_for_atoms(n_atoms: int, seed: int = 1, density: float = WATER_DENSITY,
                        **kw) -> System:
    """Water box holding n_atoms (a multiple of 3) at the given density."""
    m = n_atoms // 3
    box = (m / density) ** (1.0 / 3.0)
    return water_box(m, box, seed=seed, **kw)


def lj_fluid(n: int = 12000, box: float = 50.0, seed: int = 1, n_types: int = 4,
             min_sep: float = 2.0, qmax: float = 0.8, max_iter: int = 2000) -> System:
    """Charged LJ fluid: seeded uniform positions relaxed to a minimum
    separation, per-atom charges U[-qmax, qmax] shifted to net zero, per-type
    eps U[0.05, 0.3] kcal/mol and sigma U[2.8, 3.8] A, no exclusions.

    12,000 spheres of diameter 2 A in a 50 A cube fill 40% of the volume,
    above the ~38% jamming limit of random sequential addition, so rejection
    sampling cannot reach that density.  Positions are therefore drawn
    uniformly and then every pair closer than 1.04 * ``min_sep`` is pushed
    apart along its axis (each atom by half the shortfall) until no pair is
    closer than ``min_sep``."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, box, size=(n, 3))
    target = 1.04 * min_sep
    for _ in range(max_iter):
        tree = cKDTree(pos, boxsize=box)
        pairs = tree.query_pairs(target, output_type='ndarray')
        d = pos[pairs[:, 1]] - pos[pairs[:, 0]]
        d -= box * np.round(d / box)
        r = np.sqrt((d * d).sum(1))
        if len(r) == 0 or r.min() >= min_sep:
            break
        r = np.maximum(r, 1e-6)
        push = (0.5 * (target - r) / r)[:, None] * d
        delta = np.zeros_like(pos)
        np.add.at(delta, pairs[:, 0], -push)
        np.add.at(delta, pairs[:, 1], push)
        pos = np.mod(pos + delta, box)
    else:
        raise RuntimeError("lj_fluid: overlap removal did not converge")
    pos -= 0.5 * box
    types = rng.integers(0, n_types, size=n).astype(np.int32)
    t_eps = rng.uniform(0.05, 0.3, size=n_types)
    t_sig = rng.uniform(2.8, 3.8, size=n_types)
    q = rng.uniform(-qmax, qmax, size=n)
    q -= q.mean()
    eps = np.sqrt(t_eps[types] * KCAL_TO_IU)
    sig = 0.5 * t_sig[types]
    empty2 = np.zeros((0, 2), dtype=np.int32)
    empty3 = np.zeros((0, 3), dtype=np.int32)
    return System(f"ljfluid{n}", float(box), pos[:, 0].copy(), pos[:, 1].copy(),
                  pos[:, 2].copy(), q, eps, sig, np.full(n, 39.948), empty2, empty3,
                  types=types, type_eps_kcal=t_eps, type_sigma=t_sig,
                  meta={"seed": seed})


def thermal_velocities(mass: np.ndarray, temperature: float, seed: int = 1):
    """Seeded Maxwell-Boltzmann velocities (A/ps) for masses in amu."""
    rng = np.random.default_rng(seed)
    sd = np.sqrt(RBOLTZ_IU * temperature / np.asarray(mass, dtype=np.float64))
    v = rng.normal(size=(len(sd), 3)) * sd[:, None]
    return v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy()


def replica_sizes(count: int = 64, lo: int = 1500, hi: int = 30000, seed: int = 1) -> list[int]:
    """Atom counts drawn log-uniform in [lo, hi], rounded to multiples of 3."""
    rng = np.random.default_rng(seed)
    v = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))
    return [int(max(lo, min(hi, 3 * round(x / 3)))) for x in v]


def concat(parts: list[System], name: str = "batch") -> System:
    """Independent boxes as one batch: atoms concatenated in order, bonds and
    angles renumbered, meta["replicas"] = [(cell rows, atom count), ...]."""
    offs = np.cumsum([0] + [p.n for p in parts])
    cat = lambda attr: np.concatenate([getattr(p, attr) for p in parts])
    bonds = np.concatenate([p.bonds + o for p, o in zip(parts, offs)]).astype(np.int32)
    angles = np.concatenate([p.angles + o for p, o in zip(parts, offs)]).astype(np.int32)
    out = System(name, parts[0].box, cat("x"), cat("y"), cat("z"), cat("q"), cat("eps"),
                 cat("sig"), cat("mass"), bonds.reshape(-1, 2), angles.reshape(-1, 3),
                 meta={"replicas": [(p.cell(), p.n) for p in parts],
                       "offsets": offs.tolist()})
    if all(p.vx is not None for p in parts):
        out.vx, out.vy, out.vz = cat("vx"), cat("vy"), cat("vz")
    return out


def replica(batch: System, r: int) -> System:
    """Replica r of a systems.concat batch as a System of its own."""
    o = batch.meta["offsets"]
    lo, hi = o[r], o[r + 1]
    cell = batch.meta["replicas"][r][0]
    sel = slice(lo, hi)
    bsel = (batch.bonds[:, 0] >= lo) & (batch.bonds[:, 0] < hi)
    asel = (batch.angles[:, 0] >= lo) & (batch.angles[:, 0] < hi)
    out = System(f"{batch.name}[{r}]", float(cell[0]), batch.x[sel], batch.y[sel], batch.z[sel],
                 batch.q[sel], batch.eps[sel], batch.sig[sel], batch.mass[sel],
                 batch.bonds[bsel] - lo, batch.angles[asel] - lo)
    if batch.vx is not None:
        out.vx, out.vy, out.vz = batch.vx[sel], batch.vy[sel], batch.vz[sel]
    return out


def config_replicas(count: int = 64, seed: int = 1, temperature: float | None = None,
                    subset=None) -> System:
    """Batched replicas: `count` water boxes with seeded log-uniform atom
    counts in [1,500, 30,000] (multiples of 3), each at 0.0334 molecules/A^3
    from the lattice-plus-jitter generator (replica i uses seed + i).
    `subset`: only these replica indices (one rank's share of the batch)."""
    sizes = replica_sizes(count, seed=seed)
    idx = range(count) if subset is None else subset
    parts = [water_box_for_atoms(sizes[i], seed=seed + i, temperature=temperature) for i in idx]
    return concat(parts, name=f"replicas{count}" if subset is None else
                  f"replicas{count}_part{len(parts)}")


def flexible_chains(n_side: int = 4, box: float = 26.0, seed: int = 3, jitter: float = 0.05,
                    temperature: float | None = None) -> System:
    """n_side^3 flexible six-atom chains with every bonded kind of MDBas.

    Chains are zig-zags (bond 1.53 A, angle 109.5 deg, planar trans) along
    the box diagonal, centred on the sites of an n_side^3 lattice, each atom
    jittered by a seeded uniform +-jitter A; charges alternate +-0.2 e, LJ
    eps 0.1 kcal/mol, sigma 3.2 A, mass 14 amu.  meta["bonded"] holds the
    bonded spec (mdbas_b200.nb.bonded_structs), in MDBas units (energies in
    10 J/mol, angles in radians):

    * bonds (k, k+1): harmonic k = 250 kcal/mol/A^2 (E = k/2 dr^2), r0 1.53,
      except the middle bond (2, 3): Morse, depth 80 kcal/mol, beta 2 /A;
    * angles (k, k+1, k+2): k = 60 kcal/mol/rad^2, theta0 109.5 deg;
    * Urey-Bradley (k, k+2): k = 20 kcal/mol/A^2, r0 2.5 A;
    * dihedrals (k..k+3): cosine, k = 1.5 kcal/mol, mult 3, phi0 0, except
      the last (2..5): harmonic, k = 4 kcal/mol/rad^2, phi0 pi;
    * impropers (k+1, k, k+2, k+3), k = 0..2 (planar, phi = 0, in the
      unjittered chain): harmonic, k = 5 kcal/mol/rad^2, phi0 0.1 rad, except
      the first: cosine, k = 2 kcal/mol, mult 2, phi0 0.5 rad.

    meta["dihedrals"] lists the dihedral quadruples (for exclusion builders
    that need them)."""
    rng = np.random.default_rng(seed)
    m = n_side ** 3
    sp = box / n_side
    idx = np.arange(m)
    centres = np.stack([(idx % n_side + 0.5) * sp, (idx // n_side % n_side + 0.5) * sp,
                        (idx // n_side ** 2 + 0.5) * sp], 1) - 0.5 * box
    u = np.ones(3) / math.sqrt(3.0)
    w = np.array([1.0, -1.0, 0.0]) / math.sqrt(2.0)
    half = math.radians(109.5) / 2
    step_u, step_w = 1.53 * math.sin(half), 1.53 * math.cos(half)
    local = np.array([(k - 2.5) * step_u * u + (0.5 * step_w if k % 2 else -0.5 * step_w) * w
                      for k in range(6)])
    pos = centres[:, None, :] + local[None] + rng.uniform(-jitter, jitter, (m, 6, 3))
    pos = _wrap(pos.reshape(-1, 3), box)
    n = 6 * m
    base = 6 * np.arange(m)

    def terms(offsets):
        return np.stack([np.stack([base + o for o in offs], 1) for offs in offsets],
                        1).reshape(-1, len(offsets[0])).astype(np.int32)

    kc = KCAL_TO_IU
    bonds = terms([(k, k + 1) for k in range(5)])
    btype = np.tile([0, 0, 1, 0, 0], m)
    bk = np.where(btype == 1, 80.0 * kc, 250.0 * kc)
    angles = terms([(k, k + 1, k + 2) for k in range(4)])
    ub = terms([(k, k + 2) for k in range(4)])
    dihe = terms([(k, k + 1, k + 2, k + 3) for k in range(3)])
    dtype = np.tile([1, 1, 2], m)
    impr = terms([(k + 1, k, k + 2, k + 3) for k in range(3)])
    itype = np.tile([1, 2, 2], m)
    spec = {
        "bonds": dict(atoms=bonds, type=btype, k=bk, r0=np.full(len(bonds), 1.53),
                      beta=np.where(btype == 1, 2.0, 0.0)),
        "angles": dict(atoms=angles, k=np.full(len(angles), 60.0 * kc),
                       theta0=np.full(len(angles), math.radians(109.5))),
        "ub": dict(atoms=ub, k=np.full(len(ub), 20.0 * kc), r0=np.full(len(ub), 2.5)),
        "dihedrals": dict(atoms=dihe, type=dtype, k=np.where(dtype == 1, 1.5 * kc, 4.0 * kc),
                          phi0=np.where(dtype == 1, 0.0, math.pi),
                          mult=np.where(dtype == 1, 3.0, 1.0)),
        "impropers": dict(atoms=impr, type=itype, k=np.where(itype == 1, 2.0 * kc, 5.0 * kc),
                          phi0=np.where(itype == 1, 0.5, 0.1),
                          mult=np.where(itype == 1, 2.0, 1.0)),
    }
    q = np.tile([0.2, -0.2, 0.2, -0.2, 0.2, -0.2], m)
    s = System("chains", box, pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), q,
               np.full(n, math.sqrt(0.1 * KCAL_TO_IU)), np.full(n, 1.6), np.full(n, 14.0),
               bonds, angles, meta={"bonded": spec, "dihedrals": dihe})
    if temperature is not None:
        s.vx, s.vy, s.vz = thermal_velocities(s.mass, temperature, seed=seed)
    return s


# Named workloads (sizes of the reference's headline configurations).
def config_small(seed: int = 1) -> System:
    """3,000-atom water (1,000 molecules) in a 31.0 A box."""
    return water_box(1000, 31.0, seed=seed, name="water3000")


def config_96k(seed: int = 1, temperature: float | None = 300.0) -> System:
    """96,000-atom water (32,000 molecules) in a 98.6 A box, MB velocities."""
    return water_box(32000, 98.6, seed=seed, temperature=temperature, name="water96000")


def config_1m(seed: int = 1) -> System:
    """999,999-atom water (333,333 molecules) in a 215 A box."""
    return water_box(333333, 215.0, seed=seed, name="water999999")


POTENTIAL = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34, chargeConst=CHARGE_CONST)
