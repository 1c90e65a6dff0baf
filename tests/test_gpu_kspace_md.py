"""Reciprocal space inside the engine's dynamics (mdbas_nb_engine_set_kspace):
the engine's k-space term equals the standalone GPU sums, and dynamics with
explicit Ewald follow MDBas's own integrator with energy()'s keyEwald = 1
(ewald_rec, src/ewald.c:131-354) step by step."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
M = (8, 8, 8)


@pytest.fixture(scope="module")
def water():
    return systems.water_box(500, 25.0, seed=4, temperature=300.0)


def test_engine_kspace_equals_standalone(gpu, water):
    e = nb.Engine(water, precision=1, **POT)
    e.set_kspace(1, M)
    ee, ev, ef = e.kspace()
    se, sfx, sfy, sfz, sv, _ = nb.ewald_rec(water, 0.34, M)
    assert ee == se and ev == sv
    for a, b in zip(ef, (sfx, sfy, sfz)):
        assert np.array_equal(a, b)
    e.set_kspace(2, (32, 32, 32), 6)
    pe, pv, pf = e.kspace()
    qe, qx, qy, qz, qv = nb.spme(water, 0.34, (32, 32, 32), 6)
    scale = max(np.max(np.abs(b)) for b in (qx, qy, qz))
    assert abs(pe - qe) <= 1e-12 * abs(qe)
    assert max(np.max(np.abs(a - b)) for a, b in zip(pf, (qx, qy, qz))) <= 1e-12 * scale
    e.close()


def test_md_explicit_ewald_matches_mdbas(gpu, ref_available, water):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    r = oracle.Reference(water, **POT)
    nk = r.set_kspace(M)
    r.makelist()
    r.md_init(water.mass, vel, time_step=0.001, list_update=10, constraints=cons)
    rrows = r.md_run(20)
    rp = r.positions()
    r.close()
    e = nb.Engine(water, precision=0, **POT)
    e.set_kspace(1, M)
    e.md_init(water.mass, vel, time_step=0.001, list_update=10, constraints=cons)
    grows = e.md_run(20, energy_every=1)
    gp = e.positions()
    e.close()
    d = max(np.max(np.abs((gp[k] - rp[k]) - water.box * np.round((gp[k] - rp[k]) / water.box)))
            for k in range(3))
    pot = np.max(np.abs(grows[:, 1] - rrows[:, 1])) / np.max(np.abs(rrows[:, 1]))
    tot = np.max(np.abs(grows[:, 3] - rrows[:, 3])) / np.max(np.abs(rrows[:, 3]))
    print(f"explicit Ewald dynamics ({nk} k-vectors): pos {d:.3e} A, pot {pot:.3e}, "
          f"total {tot:.3e}")
    assert nk > 1000
    assert d < 1e-6
    # SHAKE stops each molecule at its own convergence (MDBas: all at the
    # worst one's), a 1e-8 A-scale difference in positions
    assert pot < 1e-6 and tot < 1e-6


@pytest.mark.parametrize("kind,m,order", [(1, M, 0), (2, (32, 32, 32), 6)])
def test_md_kspace_graph_equals_host_driven(gpu, water, kind, m, order):
    """Explicit Ewald or SPME (both deterministic) inside the mixed form's
    20-step graphs: the trajectory equals the host-driven one bit for bit."""
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    out = []
    for graph in (20, 0):
        e = nb.Engine(water, precision=1, **POT)
        e.set_kspace(kind, m, order)
        e.md_set_graph(graph)
        e.md_init(water.mass, vel, time_step=0.001, list_update=0, constraints=cons)
        rows = e.md_run(40, energy_every=1)
        out.append((e.positions(), rows))
        e.close()
    for k in range(3):
        assert np.array_equal(out[0][0][k], out[1][0][k])
    assert np.array_equal(out[0][1], out[1][1])


def test_md_spme_nve_conserves_energy(gpu, water):
    """SPME (32^3, order 6) in every step of 20-step graphs: after 400
    Berendsen steps, 1,000 NVE steps of 0.5 fs keep the total energy within
    0.5% of the kinetic scale."""
    e = nb.Engine(water, precision=1, **POT)
    e.set_kspace(2, (32, 32, 32), 6)
    e.md_init(water.mass, (water.vx, water.vy, water.vz), time_step=0.0005, list_update=0,
              constraints=water.water_constraints())
    e.md_run(400, target_temp=300.0, tau_t=0.05)
    rows = e.md_run(1000, energy_every=50)
    e.close()
    spread = np.max(rows[:, 3]) - np.min(rows[:, 3])
    print(f"SPME NVE: total spread {spread:.3e}, mean kin {np.mean(rows[:, 2]):.3e}")
    assert np.all(np.isfinite(rows))
    assert spread < 5e-3 * np.mean(rows[:, 2])
