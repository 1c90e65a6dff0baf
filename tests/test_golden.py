"""The restatement and the host-side code against the committed golden
fixtures (made from MDBas itself by tests/golden/make_golden.py).  These run
without MDBas's sources, e.g. on a machine that only has this repository."""
import hashlib
import json
import os

import numpy as np
import pytest

from mdbas_b200 import systems

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_generator_reproduces_fixture_positions():
    g = np.load(os.path.join(GOLD, "water3000_seed1.npz"))
    s = systems.config_small(seed=1)
    assert np.array_equal(s.x, g["x"]) and np.array_equal(s.y, g["y"])
    assert np.array_equal(s.z, g["z"])


def test_all_pairs_golden(oracle_lib):
    g = np.load(os.path.join(GOLD, "water3000_seed1.npz"))
    s = systems.config_small(seed=1)
    box = oracle_lib.box(s.cell())
    excl = s.exclusions(symmetric=False)
    lst, pair, order = oracle_lib.verlet_list(box, s.x, s.y, s.z, excl)
    assert len(lst) == int(g["list_len"])
    assert digest(lst, pair, order) == str(g["list_sha"])
    fx, fy, fz, e = oracle_lib.ewald_energy(box, s, lst, pair, order, excl)
    assert np.array_equal(fx, g["fx"]) and np.array_equal(fy, g["fy"])
    assert np.array_equal(fz, g["fz"])
    en = g["energies"]
    assert (e["e_dir"] + 0.0) + e["e_corr"] == en[0] and e["e_vdw"] == en[1]
    assert (e["vir_dir"] + 0.0) + e["vir_corr"] == en[2] and e["vir_vdw"] == en[3]
    assert oracle_lib.self_energy(s.q, systems.CHARGE_CONST, 0.34) == float(g["self_energy"])


def test_link_cell_golden(oracle_lib):
    g = np.load(os.path.join(GOLD, "water18558_seed3.npz"))
    s = systems.water_box_for_atoms(18558, seed=3)
    box = oracle_lib.box(s.cell())
    xw, yw, zw = oracle_lib.image_update(box, s.x, s.y, s.z)
    assert digest(xw, yw, zw) == str(g["pos_sha"])
    excl = s.exclusions(symmetric=True)
    lst, pair, order = oracle_lib.link_cell_list(box, xw, yw, zw, excl)
    assert digest(lst, pair, order) == str(g["list_sha"])
    fx, fy, fz, e = oracle_lib.ewald_energy(box, s, lst, pair, order, excl, x=xw, y=yw, z=zw)
    assert np.array_equal(fx[:512], g["fx"]) and np.array_equal(fz[:512], g["fz"])
    en = g["energies"]
    assert (e["e_dir"] + 0.0) + e["e_corr"] == en[0] and e["e_vdw"] == en[1]


@pytest.mark.parametrize("form", ["half", "symmetric"])
def test_exclusion_builders_golden(nb_lib, form):
    """The library's host exclusion builders (exclude_list and
    link_cell_exclude_list drop-ins) reproduce MDBas's rows and 1-4 list."""
    import ctypes as C

    from mdbas_b200 import nb
    from dropin_util import DropinSystem
    g = json.load(open(os.path.join(GOLD, "chains_torsions.json")))
    s = systems.config_small(seed=1)
    s.bonds = np.array(g["bonds"], np.int32)
    s.angles = np.array(g["angles"], np.int32)
    d = DropinSystem(s)
    L = nb.bind_dropin()
    dihe = (nb.DIHE * len(g["dihedrals"]))()
    for k, (a, b, c, dd) in enumerate(g["dihedrals"]):
        dihe[k].a, dihe[k].b, dihe[k].c, dihe[k].d = a, b, c, dd
    impr = (nb.DIHE * len(g["impropers"]))()
    for k, (a, b, c, dd) in enumerate(g["impropers"]):
        impr[k].a, impr[k].b, impr[k].c, impr[k].d = a, b, c, dd
    d.param.nDihedral = len(g["dihedrals"])
    d.param.nImproper = len(g["impropers"])
    l14 = C.POINTER(C.c_int)()
    excl = C.POINTER(C.POINTER(C.c_int))()
    ep = C.POINTER(C.c_int)()
    fn = L.exclude_list if form == "half" else L.link_cell_exclude_list
    fn(C.byref(d.ctrl), C.byref(d.param), C.byref(d.neigh), d.const, d.bond, d.angle, dihe, impr,
       C.byref(l14), C.byref(excl), C.byref(ep))
    want = g[form]
    pair = np.ctypeslib.as_array(ep, (s.n,)).tolist()
    assert pair == want["excl_pair"]
    flat = [excl[i][k] for i in range(s.n) for k in range(pair[i])]
    assert flat == want["excl_flat"]
    n14 = d.neigh.nPair14
    assert [l14[k] for k in range(2 * n14)] == want["list14"]
