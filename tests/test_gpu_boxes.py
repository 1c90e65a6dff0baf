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


@pytest.mark.parametrize("kind", ["orbic", "tclin"])
def test_md_fp64_matches_mdbas(gpu, kind):
    """10 velocity-Verlet steps of an LJ fluid in a non-cubic cell (list
    rebuilt every 5 steps, positions wrapped by image_update): the engine's
    FP64 dynamics against MDBas's integrator.  (This fluid, sampled with a
    2 A minimum separation, blows up a few steps later: MDBas's kinetic
    energy passes 1e22 at step 15.)"""
    s = systems.lj_fluid(3000, 33.0, seed=4)
    btype, cell = _cell(kind, 33.0)
    vel = systems.thermal_velocities(s.mass, 150.0, seed=4)
    pot = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
    r = _reference(s, cell, btype)
    r.makelist()
    r.md_init(s.mass, vel, time_step=0.002, list_update=5)
    rrows = r.md_run(10)
    rp = r.positions()
    rself = r.self_energy()
    r.close()
    e = nb.Engine(s, precision=0, box_type=btype, cell=cell, **pot)
    e.md_init(s.mass, vel, time_step=0.002, list_update=5)
    grows = e.md_run(10, energy_every=1)
    gp = e.positions()
    e.close()
    # positions up to a lattice vector of the cell (rows a, b, c)
    h = cell.reshape(3, 3)
    d = np.stack([np.asarray(gp[k]) - np.asarray(rp[k]) for k in range(3)], 1)
    frac = d @ np.linalg.inv(h)
    d = (frac - np.round(frac)) @ h
    perr = np.max(np.abs(d))
    tot_err = np.max(np.abs(grows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    print(f"{kind}: pos {perr:.3e} A, total energy {tot_err:.3e}")
    assert tot_err < 1e-10
    assert perr < 1e-9


@pytest.mark.parametrize("precision", [0, 1])
def test_md_kinetic_overflow_is_reported(gpu, precision):
    """A kinetic energy beyond the 64-bit fixed-point range (one atom at
    1e8 A/ps) stops the run with MDBAS_NB_ERR_OVERFLOW instead of reporting
    a wrapped sum."""
    s = systems.lj_fluid(3000, 33.0, seed=4)
    vel = [np.array(v) for v in systems.thermal_velocities(s.mass, 150.0, seed=4)]
    vel[0][7] = 1.0e8
    e = nb.Engine(s, precision=precision, cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
    e.md_init(s.mass, vel, time_step=0.002, list_update=5)
    with pytest.raises(nb.MdbasNbError) as err:
        e.md_run(2, energy_every=1)
    assert err.value.status == 10 and "overflow" in str(err.value)   # MDBAS_NB_ERR_OVERFLOW
    e.close()
