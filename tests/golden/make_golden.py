"""Regenerate the golden fixtures of tests/golden/ from MDBas itself.

MDBas has no tests or golden vectors of its own, so the pins of this
repository are outputs of MDBas's own code (oracle/_ref/libmdbas_ref.so,
built from MDBas's sources by oracle/Makefile) on seeded inputs from
mdbas_b200.systems.  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

Fixtures:
  water3000_seed1.npz   all-pairs list path (31 A box): positions, list
                        checksum, forces of every atom, energies and virials
  water18558_seed3.npz  link-cell path (57.3 A box): wrapped-position and list
                        checksums, forces of the first 512 atoms, energies
  chains_torsions.json  exclusion rows and 1-4 list of a topology with bonds,
                        angles, dihedrals and impropers (both builders)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def chains_topology(n_chains: int = 40, length: int = 6):
    """Linear 6-atom chains: bonds, angles, dihedrals, one improper each."""
    bonds, angles, dihe, impr = [], [], [], []
    for c in range(n_chains):
        b = c * length
        for k in range(length - 1):
            bonds.append((b + k, b + k + 1))
        for k in range(length - 2):
            angles.append((b + k, b + k + 1, b + k + 2))
        for k in range(length - 3):
            dihe.append((b + k, b + k + 1, b + k + 2, b + k + 3))
        impr.append((b + 1, b, b + 2, b + 3))
    return (np.array(bonds, np.int32), np.array(angles, np.int32), np.array(dihe, np.int32),
            np.array(impr, np.int32))


def main():
    import oracle
    from mdbas_b200 import systems
    if not oracle.Reference.available():
        raise SystemExit("build oracle/_ref first (make -C oracle)")

    # all-pairs path
    s = systems.config_small(seed=1)
    r = oracle.Reference(s)
    assert r.makelist() == 0
    lst, pair, order = r.get_list()
    fx, fy, fz, e = r.energy()
    np.savez_compressed(os.path.join(HERE, "water3000_seed1.npz"), x=s.x, y=s.y, z=s.z,
                        list_sha=digest(lst, pair, order), list_len=len(lst),
                        size_list=r.size_list, fx=fx, fy=fy, fz=fz,
                        energies=np.array([e["elec"], e["vdw"], e["virelec"], e["virvdw"]]),
                        self_energy=r.self_energy())
    r.close()

    # link-cell path
    s = systems.water_box_for_atoms(18558, seed=3)
    r = oracle.Reference(s)
    assert r.makelist() == 1
    xw, yw, zw = r.positions()
    lst, pair, order = r.get_list()
    fx, fy, fz, e = r.energy()
    np.savez_compressed(os.path.join(HERE, "water18558_seed3.npz"),
                        pos_sha=digest(xw, yw, zw), list_sha=digest(lst, pair, order),
                        list_len=len(lst), n_cells=r.n_cells, fx=fx[:512], fy=fy[:512],
                        fz=fz[:512],
                        energies=np.array([e["elec"], e["vdw"], e["virelec"], e["virvdw"]]))
    r.close()

    # exclusion builders on a topology with torsions
    s = systems.config_small(seed=1)
    bonds, angles, dihe, impr = chains_topology()
    s.bonds, s.angles = bonds, angles
    out = {"bonds": bonds.tolist(), "angles": angles.tolist(), "dihedrals": dihe.tolist(),
           "impropers": impr.tolist(), "n_atoms": s.n}
    for name, nolink in (("half", 1), ("symmetric", 0)):
        cell = None if nolink else [60.0, 0, 0, 0, 60.0, 0, 0, 0, 60.0]
        r = oracle.Reference(s, noLink=nolink, cell=cell)
        r.set_torsions(dihe, impr)
        r.makelist()
        start, flat = r.get_excl()
        out[name] = {"excl_pair": np.diff(start).tolist(), "excl_flat": flat.tolist(),
                     "list14": r.list14().tolist()}
        r.close()
    with open(os.path.join(HERE, "chains_torsions.json"), "w") as f:
        json.dump(out, f)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
