"""Orthorhombic and triclinic boxes (MDBas's pbc 2 and 3) on the GPU against
MDBas itself: the drop-in list builders entry for entry, energy() in the FP64
form to 1e-12, the mixed form (orthorhombic boxes take the cluster-pair path,
triclinic ones the FP64 form over MDBas's list) and the engine.  The water
boxes sit inside larger cells, so the images across a tilted face keep their
distance."""
import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems
from dropin_util import DropinSystem, force_rel_rms

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


def _system(which):
    # small: 3,000 atoms, O(N^2) list (fewer than 3 link cells per edge);
    # link: 18,558 atoms, link cells
    return systems.config_small(2) if which == "small" else systems.water_box_for_atoms(18558, 5)


def _cell(kind, edge):
    if kind == "orbic":
        return nb.ORBIC, np.array([edge + 2.0, 0, 0, 0, edge + 3.5, 0, 0, 0, edge + 5.0])
    return nb.TCLIN, np.array([edge + 4.0, 0, 0, 1.5, edge + 4.0, 0, 1.0, 2.0, edge + 4.0])


def _reference(s, cell, btype):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    return oracle.Reference(s, cell=cell, box_type=btype)


@pytest.mark.parametrize("which", ["small", "link"])
@pytest.mark.parametrize("kind", ["orbic", "tclin"])
def test_list_and_fp64_energy(gpu, kind, which):
    s = _system(which)
    btype, cell = _cell(kind, s.box)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    d = DropinSystem(s, cell=cell, box_type=btype)
    r = _reference(s, cell, btype)
    link = d.makelist()
    assert link == r.makelist() == (0 if which == "small" else 1)
    lst, pair, order = d.get_list()
    rl, rp, ro = r.get_list()
    assert np.array_equal(pair, rp) and np.array_equal(order, ro)
    assert np.array_equal(lst, rl)
    rx, ry, rz = r.positions()   # both wrapped the coordinates the same way
    assert np.array_equal(d.x, rx) and np.array_equal(d.y, ry) and np.array_equal(d.z, rz)
    fx, fy, fz, e = d.energy()
    rfx, rfy, rfz, re = r.energy()
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < FP64_TOL
    for k in ("elec", "vdw", "virelec", "virvdw"):
        assert abs(e[k] - re[k]) <= FP64_TOL * abs(re[k]), k
    d.free()
    r.close()


@pytest.mark.parametrize("kind", ["orbic", "tclin"])
def test_mixed_dropin(gpu, kind):
    s = _system("link")
    btype, cell = _cell(kind, s.box)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(1)
    try:
        d = DropinSystem(s, cell=cell, box_type=btype)
        d.makelist()
        fx, fy, fz, e = d.energy()
    finally:
        L.mdbas_nb_set_mode(0)
    r = _reference(s, cell, btype)
    r.makelist()
    rfx, rfy, rfz, re = r.energy()
    # triclinic cells take the FP64 form over MDBas's list
    tol = MIXED_TOL if kind == "orbic" else FP64_TOL
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < tol
    for k in ("elec", "vdw"):
        assert abs(e[k] - re[k]) <= tol * abs(re[k]), k
    d.free()
    r.close()


@pytest.mark.parametrize("kind", ["orbic", "tclin"])
def test_engine(gpu, kind):
    s = _system("link")
    btype, cell = _cell(kind, s.box)
    r = _reference(s, cell, btype)
    r.makelist()
    rx, ry, rz = r.positions()
    rfx, rfy, rfz, re = r.energy()
    s.x, s.y, s.z = rx, ry, rz
    for precision, tol in ((0, FP64_TOL), (1, MIXED_TOL)):
        if precision == 1 and kind == "tclin":
            # the cluster-pair path needs an orthorhombic cell; it says so
            with pytest.raises(nb.MdbasNbError):
                nb.Engine(s, precision=1, box_type=btype, cell=cell).build()
            continue
        eng = nb.Engine(s, precision=precision, box_type=btype, cell=cell)
        eng.build()
        eng.compute()
        f = eng.forces()
        e = eng.energies()
        assert force_rel_rms(f, (rfx, rfy, rfz)) < tol
        elec = e["elec_direct"] + e["elec_corr"]
        assert abs(elec - re["elec"]) <= tol * abs(re["elec"])
        assert abs(e["vdw"] - re["vdw"]) <= tol * abs(re["vdw"])
    r.close()
