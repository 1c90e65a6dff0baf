"""The C restatement (oracle/mdbas_oracle.c) against MDBas itself, bit for bit.

Every case builds the same system in MDBas (oracle/_ref, MDBas's own list.c,
energy.c, ewald.c, vdw.c, utils.c) and in the restatement and requires
identical lists (entries and order), forces, energies and virials.
"""
import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems

pytestmark = pytest.mark.skipif(not oracle.Reference.available(),
                                reason="MDBas reference library not built")


def _check_case(o, s, linkRatio=1, frozen=None, noLink=0):
    r = oracle.Reference(s, linkRatio=linkRatio, frozen=frozen, noLink=noLink)
    kl = r.makelist()
    rl, rp, ro = r.get_list()
    excl = r.get_excl()
    xw, yw, zw = r.positions()
    box = o.box(s.cell())
    if kl:
        ol, op, oo = o.link_cell_list(box, xw, yw, zw, excl, linkRatio=linkRatio, frozen=frozen)
    else:
        ol, op, oo = o.verlet_list(box, xw, yw, zw, excl, frozen=frozen)
    assert np.array_equal(op, rp) and np.array_equal(oo, ro) and np.array_equal(ol, rl)
    fx, fy, fz, e = r.energy()
    ofx, ofy, ofz, oe = o.ewald_energy(box, s, rl, rp, ro, excl, x=xw, y=yw, z=zw)
    assert np.array_equal(ofx, fx) and np.array_equal(ofy, fy) and np.array_equal(ofz, fz)
    assert (oe["e_dir"] + 0.0) + oe["e_corr"] == e["elec"]
    assert oe["e_vdw"] == e["vdw"]
    assert (oe["vir_dir"] + 0.0) + oe["vir_corr"] == e["virelec"]
    assert oe["vir_vdw"] == e["virvdw"]
    assert o.self_energy(s.q, systems.CHARGE_CONST, 0.34) == r.self_energy()
    r.close()
    return kl, len(rl)


def test_all_pairs_path_small_box(oracle_lib):
    kl, n = _check_case(oracle_lib, systems.config_small(1))
    assert kl == 0 and n == 1745777


def test_link_cell_path(oracle_lib):
    kl, n = _check_case(oracle_lib, systems.water_box_for_atoms(18558, 3))
    assert kl == 1


@pytest.mark.parametrize("ratio", [2, 3])
def test_link_cell_finer_stencils(oracle_lib, ratio):
    kl, _ = _check_case(oracle_lib, systems.water_box_for_atoms(18558, 4), linkRatio=ratio)
    assert kl == 1


def test_frozen_pairs_dropped(oracle_lib):
    s = systems.config_small(2)
    fz = (np.random.default_rng(5).random(s.n) < 0.15).astype(np.int32)
    _check_case(oracle_lib, s, frozen=fz)


def test_nolink_forces_all_pairs(oracle_lib):
    kl, _ = _check_case(oracle_lib, systems.water_box_for_atoms(18558, 3), noLink=1)
    assert kl == 0


def test_lj_fluid_no_exclusions(oracle_lib):
    s = systems.lj_fluid(3000, 31.0, seed=2)
    _check_case(oracle_lib, s)


def test_init_box_restatements_match(oracle_lib):
    cells = [[31.0, 0, 0, 0, 31.0, 0, 0, 0, 31.0],
             [40.0, 0, 0, 0, 35.5, 0, 0, 0, 33.25],
             [40.0, 0.0, 0.0, 3.0, 38.0, 0.0, 1.5, 2.5, 36.0]]
    for k, cell in enumerate(cells):
        btype = [nb.CUBIC, nb.ORBIC, nb.TCLIN][k]
        s = systems.config_small(1)
        r = oracle.Reference(s, cell=np.array(cell), box_type=btype)
        rb = r.box()  # a a1 a2 a3 b ... pa pb pc det vol vol0
        p = nb.make_pbc(cell, btype)
        mine = [p.a, p.a1, p.a2, p.a3, p.b, p.b1, p.b2, p.b3, p.c, p.c1, p.c2, p.c3, p.u, p.u1,
                p.u2, p.u3, p.v, p.v1, p.v2, p.v3, p.w, p.w1, p.w2, p.w3, p.pa, p.pb, p.pc,
                p.det, p.vol, p.vol0]
        assert np.array_equal(np.array(mine), rb), cell
        ob = oracle_lib.box(cell, btype)
        assert ob[oracle.ORC_BOX_LEN - 1] == p.det
        assert np.array_equal(ob[9:18], np.array([p.u1, p.u2, p.u3, p.v1, p.v2, p.v3, p.w1,
                                                  p.w2, p.w3]))
        r.close()


def test_triclinic_all_pairs(oracle_lib):
    s = systems.config_small(3)
    cell = np.array([31.0, 0.0, 0.0, 1.5, 31.0, 0.0, 1.0, 2.0, 31.0])
    r = oracle.Reference(s, cell=cell, box_type=nb.TCLIN)
    assert r.makelist() == 0
    rl, rp, ro = r.get_list()
    excl = r.get_excl()
    box = oracle_lib.box(cell, nb.TCLIN)
    ol, op, oo = oracle_lib.verlet_list(box, s.x, s.y, s.z, excl, box_type=nb.TCLIN)
    assert np.array_equal(ol, rl) and np.array_equal(op, rp)
    r.close()
