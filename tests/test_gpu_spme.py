"""GPU SPME (csrc/spme.cu: MDBas's spme_energy with cuFFT) against the numpy
restatement of src/spme.c (oracle/spme_oracle.py, itself pinned to MDBas's
explicit Ewald sum), and the drop-in energy() with keyEwald = 2."""
import ctypes as C

import numpy as np
import pytest

from mdbas_b200 import nb, systems

from dropin_util import DropinSystem, force_rel_rms

pytestmark = pytest.mark.gpu


# grids that are multiples of 8 take the binned (deterministic) spreading,
# the others the atomic one; order 12 reaches three 8^3 tiles per dimension
@pytest.mark.parametrize("grid,nbsp", [((32, 32, 32), 8), ((64, 64, 64), 8),
                                       ((32, 32, 32), 4), ((16, 32, 64), 6),
                                       ((20, 24, 36), 8), ((32, 32, 32), 12),
                                       ((8, 16, 8), 6)])
def test_spme_matches_restatement(gpu, oracle_lib, grid, nbsp):
    from oracle import spme_oracle as so
    s = systems.water_box(1000, 31.0, seed=3)
    e, fx, fy, fz, vir = nb.spme(s, alpha=0.34, grid=grid, nbsp=nbsp)
    box = oracle_lib.box(s.cell())
    er, rx, ry, rz, rvir = so.spme_energy(box, s.x, s.y, s.z, s.q, 0.34, systems.CHARGE_CONST,
                                          grid, nbsp)
    rel = force_rel_rms((fx, fy, fz), (rx, ry, rz))
    print(f"grid {grid} order {nbsp}: E {e:.10e} vs {er:.10e}; force {rel:.2e}")
    assert abs(e - er) <= 1e-11 * abs(er)
    assert abs(vir - rvir) <= 1e-10 * abs(rvir)
    assert rel < 1e-10


def test_spme_deterministic(gpu):
    """Binned spreading: two calls give the same bits."""
    s = systems.water_box(1000, 31.0, seed=5)
    a = nb.spme(s, alpha=0.34, grid=(32, 32, 32), nbsp=8)
    b = nb.spme(s, alpha=0.34, grid=(32, 32, 32), nbsp=8)
    assert a[0] == b[0] and a[4] == b[4]
    for k in (1, 2, 3):
        assert np.array_equal(a[k], b[k])


def test_spme_atoms_outside_the_box(gpu, oracle_lib):
    """Atoms whole box lengths beyond the upper faces spread like their
    images, and every grid access stays in bounds.  (MDBas only sees atoms in
    the box -- image_update wraps them before each energy call -- and would
    fold such stencils onto plane 0.)"""
    s = systems.water_box(1000, 31.0, seed=6)
    rng = np.random.default_rng(2)
    shift = 31.0 * rng.integers(0, 3, size=(s.n, 3))
    moved = systems.System(**{**s.__dict__})
    moved.x, moved.y, moved.z = s.x + shift[:, 0], s.y + shift[:, 1], s.z + shift[:, 2]
    for grid in ((32, 32, 32), (20, 24, 36)):   # binned and atomic spreading
        e0, *f0, v0 = nb.spme(s, alpha=0.34, grid=grid, nbsp=8)
        e1, *f1, v1 = nb.spme(moved, alpha=0.34, grid=grid, nbsp=8)
        assert abs(e1 - e0) <= 1e-10 * abs(e0)
        assert abs(v1 - v0) <= 1e-10 * abs(v0)
        assert force_rel_rms(f1, f0) < 1e-10


def test_spme_orthorhombic_charged(gpu, oracle_lib):
    """Orthorhombic box and a net charge (non-neutral term)."""
    from oracle import spme_oracle as so
    s = systems.lj_fluid(1500, 30.0, seed=8)
    s.q = s.q + 0.01
    cell = np.array([30.0, 0, 0, 0, 33.0, 0, 0, 0, 36.0])
    e, fx, fy, fz, vir = nb.spme(s, alpha=0.3, grid=(32, 32, 64), nbsp=8, cell=cell,
                                 box_type=nb.ORBIC)
    box = oracle_lib.box(cell, box_type=2)
    er, rx, ry, rz, rvir = so.spme_energy(box, s.x, s.y, s.z, s.q, 0.3, systems.CHARGE_CONST,
                                          (32, 32, 64), 8)
    assert abs(e - er) <= 1e-11 * abs(er)
    assert force_rel_rms((fx, fy, fz), (rx, ry, rz)) < 1e-10


def test_dropin_energy_keyewald2(gpu, oracle_lib):
    """energy() with keyEwald = 2: real space on the GPU (FP64 form) plus the
    GPU SPME, against the oracle's real-space terms plus the restatement."""
    from oracle import spme_oracle as so
    s = systems.water_box(1000, 31.0, seed=4)
    d = DropinSystem(s, keyEwald=2, alpha=0.34)
    L = nb.lib()
    L.init_spme.argtypes = [C.c_void_p] * 4
    d.ewald.prec = 1e-6
    d.ewald.nbsp = 8
    d.ctrl.keyAlpha = 1
    L.init_spme(C.byref(d.ctrl), C.byref(d.param), C.byref(d.ewald), C.byref(d.box))
    grid = (d.ewald.m1max, d.ewald.m2max, d.ewald.m3max)
    assert grid == (32, 32, 32)
    d.makelist()
    fx, fy, fz, e = d.energy()
    lst, pair, order = d.get_list()
    excl = d.get_excl()
    box = oracle_lib.box(s.cell())
    rfx, rfy, rfz, re = oracle_lib.ewald_energy(box, s, lst, pair, order, excl)
    er, sx, sy, sz, _ = so.spme_energy(box, d.x, d.y, d.z, s.q, 0.34, systems.CHARGE_CONST,
                                       grid, 8)
    d.free()
    elec_ref = re["e_dir"] + re["e_corr"] + er
    # the total is a small difference of large terms: scale by the terms
    scale = abs(re["e_dir"]) + abs(re["e_corr"]) + abs(er)
    print(f"elec {e['elec']:.10e} vs {elec_ref:.10e} (terms {scale:.3e})")
    assert abs(e["elec"] - elec_ref) <= 1e-12 * scale
    assert force_rel_rms((fx, fy, fz), (rfx + sx, rfy + sy, rfz + sz)) < 1e-10
