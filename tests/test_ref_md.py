"""MDBas's own velocity-Verlet dynamics through the harness (CPU).

These pin the reference side of the GPU dynamics tests: the harness drives
vv_integrate / vv_shake_r / vv_shake_v (src/integrate.c:1479-1750,
src/shake.c:209-456) the way src/mdbas.c:244-300 does, and the results must
look like MDBas's: bonds held to tolShake, NVE total energy steady, the
Berendsen bath pulling the kinetic energy toward its target, and the degrees
of freedom of get_degfree (src/utils.c:569-581).
"""
import numpy as np
import pytest

from mdbas_b200 import systems

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)


@pytest.fixture(scope="module")
def ref_md_run(ref_available):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s = systems.water_box(1000, 31.0, seed=5, temperature=300.0)
    cons = s.water_constraints()
    r = oracle.Reference(s, **POT)
    r.makelist()
    ndf = r.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.0005, list_update=10,
                    constraints=cons)
    rows = r.md_run(12)
    pos = r.positions()
    r.close()
    return s, cons, ndf, rows, pos


def test_ref_md_degrees_of_freedom(ref_md_run):
    s, cons, ndf, _, _ = ref_md_run
    assert ndf == 3 * s.n - 3 - len(cons[1])


def test_ref_md_constraints_hold(ref_md_run):
    s, (pairs, len2), _, _, pos = ref_md_run
    d = [pos[k][pairs[:, 1]] - pos[k][pairs[:, 0]] for k in range(3)]
    d = [v - s.box * np.round(v / s.box) for v in d]
    r2 = d[0] ** 2 + d[1] ** 2 + d[2] ** 2
    # vv_shake_r stops when max |r^2 - d^2| / d / 2 < tolShake (1e-8)
    assert np.max(np.abs(r2 - len2) / np.sqrt(len2)) < 2 * 1e-8


def test_ref_md_nve_energy_steady(ref_md_run):
    _, _, _, rows, _ = ref_md_run
    tot, kin = rows[:, 3], rows[:, 2]
    assert np.all(np.diff(rows[:, 0]) == 1)
    assert np.max(np.abs(tot - tot[0])) / np.mean(kin) < 5e-3


def test_ref_md_berendsen_moves_toward_target(ref_available):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s = systems.lj_fluid(1500, 26.0, seed=2)
    v = systems.thermal_velocities(s.mass, 100.0, seed=2)
    r = oracle.Reference(s, **POT)
    r.makelist()
    ndf = r.md_init(s.mass, v, time_step=0.001, list_update=5, temp0=400.0, tau_t=0.01)
    rows = r.md_run(6)
    r.close()
    temps = 2.0 * rows[:, 2] / (ndf * systems.RBOLTZ_IU)
    assert temps[-1] > temps[0]
