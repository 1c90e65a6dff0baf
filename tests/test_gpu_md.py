"""Device-resident velocity-Verlet dynamics against MDBas's own integrator.

The reference side runs MDBas's vv_integrate / vv_shake_r / vv_shake_v /
makelist / energy (src/integrate.c:1479-1750, src/shake.c:209-456,
src/mdbas.c:244-300) through oracle/_ref; the GPU side runs
mdbas_nb_engine_md_run.  Both start from the same positions, velocities and
list, so short trajectories agree to the accumulated round-off:

* FP64 form: positions within 1e-6 A after 20 steps (force sums differ in
  order at 1e-15 relative; SHAKE stops each molecule at its own convergence,
  MDBas iterates all molecules until the worst converges, a difference below
  tolShake * bond length per step);
* mixed precision: positions within 1e-3 A after 20 steps (force RMS error
  ~1e-6 relative).
"""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)


def _min_image(d, box):
    return d - box * np.round(d / box)


def _pos_err(a, b, box):
    return max(np.max(np.abs(_min_image(np.asarray(a[k]) - np.asarray(b[k]), box)))
               for k in range(3))


def _ref_md(sysm, vel, dt, steps, list_update, constraints=None, temp0=0.0, tau_t=0.0,
            dihedrals=None):
    import oracle
    r = oracle.Reference(sysm, **POT)
    if dihedrals is not None:
        r.set_torsions(dihedrals, None)
    r.makelist()
    r.md_init(sysm.mass, vel, time_step=dt, list_update=list_update, constraints=constraints,
              temp0=temp0, tau_t=tau_t)
    rows = r.md_run(steps)
    out = r.positions(), r.velocities(), rows, r.self_energy()
    r.close()
    return out


def _gpu_md(sysm, vel, dt, steps, list_update, precision, constraints=None, temp0=0.0,
            tau_t=0.0, frozen=None, graph=None, exclusions=None, prune=None):
    e = nb.Engine(sysm, precision=precision, frozen=frozen, exclusions=exclusions, **POT)
    if graph is not None:
        e.md_set_graph(graph)
    if prune is not None:
        e.md_set_prune(prune)
    e.md_init(sysm.mass, vel, time_step=dt, list_update=list_update, constraints=constraints)
    rows = e.md_run(steps, energy_every=1, target_temp=temp0, tau_t=tau_t)
    out = e.positions(), e.velocities(), rows, e.md_stats(), e.launches()
    e.close()
    return out


@pytest.fixture(scope="module")
def water():
    s = systems.water_box(1000, 31.0, seed=5, temperature=300.0)
    return s


def test_md_fp64_matches_mdbas_rigid_water(gpu, ref_available, water):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    rp, rv, rrows, rself = _ref_md(water, vel, 0.001, 20, 10, cons)
    gp, gv, grows, st, launches = _gpu_md(water, vel, 0.001, 20, 10, 0, cons)
    perr = _pos_err(gp, rp, water.box)
    verr = max(np.max(np.abs(gv[k] - rv[k])) for k in range(3))
    # energies: MDBas's pot has no self term; pot + self passes through zero
    # here, so the difference is scaled by MDBas's real-space pot itself
    pot_err = np.max(np.abs(grows[:, 1] - (rrows[:, 1] + rself))) / np.max(np.abs(rrows[:, 1]))
    kin_err = np.max(np.abs(grows[:, 2] - rrows[:, 2]) / rrows[:, 2])
    print(f"fp64 water: pos {perr:.3e} A, vel {verr:.3e} A/ps, pot {pot_err:.3e}, "
          f"kin {kin_err:.3e}, shake iter {st['shake_iter']}")
    assert st["steps"] == 20 and st["rebuilds"] == 3 and st["molecules"] == 1000
    assert launches > 20 * 5
    assert perr < 1e-6
    assert verr < 1e-3
    assert pot_err < 1e-8
    assert kin_err < 1e-6


def test_md_fp64_matches_mdbas_lj_fluid_nve(gpu, ref_available):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.lj_fluid(3000, 33.0, seed=4)
    vel = systems.thermal_velocities(s.mass, 150.0, seed=4)
    rp, rv, rrows, rself = _ref_md(s, vel, 0.002, 20, 5)
    gp, gv, grows, st, _ = _gpu_md(s, vel, 0.002, 20, 5, 0)
    perr = _pos_err(gp, rp, s.box)
    verr = max(np.max(np.abs(gv[k] - rv[k])) for k in range(3))
    tot_err = np.max(np.abs(grows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    print(f"fp64 lj: pos {perr:.3e} A, vel {verr:.3e}, total {tot_err:.3e}")
    assert perr < 1e-9
    assert verr < 1e-7
    assert tot_err < 1e-10


def test_md_mixed_tracks_mdbas(gpu, ref_available, water):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    rp, rv, rrows, rself = _ref_md(water, vel, 0.001, 20, 10, cons)
    gp, gv, grows, st, _ = _gpu_md(water, vel, 0.001, 20, 10, 1, cons)
    perr = _pos_err(gp, rp, water.box)
    tot_err = np.max(np.abs(grows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    print(f"mixed water: pos {perr:.3e} A, total {tot_err:.3e}")
    assert perr < 1e-3
    assert tot_err < 1e-5


def test_md_berendsen_matches_mdbas(gpu, ref_available, water):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    rp, rv, rrows, rself = _ref_md(water, vel, 0.001, 20, 10, cons, temp0=250.0, tau_t=0.05)
    gp, gv, grows, st, _ = _gpu_md(water, vel, 0.001, 20, 10, 0, cons, temp0=250.0, tau_t=0.05)
    perr = _pos_err(gp, rp, water.box)
    kin_err = np.max(np.abs(grows[:, 2] - rrows[:, 2]) / rrows[:, 2])
    print(f"berendsen: pos {perr:.3e} A, kin {kin_err:.3e}")
    assert perr < 1e-6
    assert kin_err < 1e-6


def test_md_displacement_rebuild_matches_every_step(gpu, water):
    """listUpdate = 0 (rebuild on half-skin displacement) gives the trajectory
    of a rebuild at every step: no pair inside the cut-off is ever missing."""
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    ap, av, arows, ast, _ = _gpu_md(water, vel, 0.002, 60, 0, 0, cons)
    bp, bv, brows, bst, _ = _gpu_md(water, vel, 0.002, 60, 1, 0, cons)
    perr = _pos_err(ap, bp, water.box)
    print(f"displacement rebuilds {ast['rebuilds']} vs {bst['rebuilds']}; pos {perr:.3e}")
    assert bst["rebuilds"] == 61
    assert 1 < ast["rebuilds"] < 61
    assert perr < 1e-8


def test_md_constraints_hold_and_frozen_atoms_stay(gpu, water):
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    frozen = np.zeros(water.n, np.int32)
    frozen[:30] = 1          # the first ten molecules
    gp, gv, grows, st, _ = _gpu_md(water, vel, 0.001, 30, 10, 1, cons, frozen=frozen)
    pairs, len2 = cons
    d = [_min_image(gp[k][pairs[:, 1]] - gp[k][pairs[:, 0]], water.box) for k in range(3)]
    r2 = d[0] ** 2 + d[1] ** 2 + d[2] ** 2
    rel = np.max(np.abs(r2 - len2) / len2)
    moved = max(np.max(np.abs(_min_image(gp[k][:30] - (water.x, water.y, water.z)[k][:30],
                                         water.box))) for k in range(3))
    print(f"constraint rel err {rel:.3e}; frozen moved {moved:.3e}")
    assert rel < 4e-8
    assert moved == 0.0
    assert all(np.all(gv[k][:30] == 0.0) for k in range(3))


def test_md_mixed_nve_conserves_energy(gpu):
    """Rigid water, mixed precision: after a Berendsen warm-up, 2 fs NVE keeps
    the total energy within 1% of the kinetic energy over 1000 steps."""
    s = systems.water_box(1000, 31.0, seed=7, temperature=300.0, jitter=0.2)
    eq = nb.Engine(s, precision=1, **POT)
    eq.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.0005, list_update=0,
               constraints=s.water_constraints())
    eq.md_run(2000, target_temp=300.0, tau_t=0.05)
    pos, vel = eq.positions(), eq.velocities()
    eq.close()
    s2 = systems.System(s.name, s.box, *pos, s.q, s.eps, s.sig, s.mass, s.bonds, s.angles)
    md = nb.Engine(s2, precision=1, **POT)
    md.md_init(s2.mass, vel, time_step=0.002, list_update=0, constraints=s2.water_constraints())
    rows = md.md_run(1000, energy_every=10)
    st = md.md_stats()
    md.close()
    tot, kin = rows[:, 3], rows[:, 2]
    drift = (tot[-1] - tot[0]) / np.mean(kin)
    spread = (tot.max() - tot.min()) / np.mean(kin)
    print(f"NVE 2 fs x 1000: drift {drift:.3e}, spread {spread:.3e} of <K>; "
          f"rebuilds {st['rebuilds']}")
    assert abs(drift) < 0.01
    assert spread < 0.02


@pytest.mark.parametrize("list_update", [0, 7])
def test_md_graph_matches_stepwise_bitwise(gpu, water, list_update):
    """Whole steps captured as CUDA graphs (device-side rebuild decision,
    conditional list build) give the trajectory of the host-driven loop bit
    for bit, energies included; 70 steps = three 20-step launches + 10 more."""
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    ap, av, arows, ast, al = _gpu_md(water, vel, 0.002, 70, list_update, 1, cons, graph=20)
    bp, bv, brows, bst, bl = _gpu_md(water, vel, 0.002, 70, list_update, 1, cons, graph=0)
    print(f"graph rebuilds {ast['rebuilds']} launches {al}; stepwise {bst['rebuilds']} {bl}")
    assert ast["rebuilds"] == bst["rebuilds"] > 1
    for k in range(3):
        assert np.array_equal(ap[k], bp[k])
        assert np.array_equal(av[k], bv[k])
    assert np.array_equal(arows, brows)
    assert al > 70 * 10


def test_md_graph_berendsen_and_frozen(gpu, water):
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    frozen = np.zeros(water.n, np.int32)
    frozen[3:9] = 1
    a = _gpu_md(water, vel, 0.001, 40, 0, 1, cons, temp0=250.0, tau_t=0.05, frozen=frozen,
                graph=20)
    b = _gpu_md(water, vel, 0.001, 40, 0, 1, cons, temp0=250.0, tau_t=0.05, frozen=frozen,
                graph=0)
    for k in range(3):
        assert np.array_equal(a[0][k], b[0][k])
    assert np.array_equal(a[2], b[2])
    assert all(np.all(a[1][k][3:9] == 0.0) for k in range(3))


def _chain_system(n_side=4, box=26.0, seed=3):
    """n_side^3 six-atom zig-zag chains (bond 1.53 A, angle 109.5 deg) along
    the box diagonal on a cubic lattice, alternating charges +-0.2 e; every
    bond is a constraint, so each molecule has 6 atoms and 5 constraints
    (the large class of the SHAKE kernels)."""
    rng = np.random.default_rng(seed)
    m = n_side ** 3
    sp = box / n_side
    idx = np.arange(m)
    centres = np.stack([(idx % n_side + 0.5) * sp, (idx // n_side % n_side + 0.5) * sp,
                        (idx // n_side ** 2 + 0.5) * sp], 1) - 0.5 * box
    u = np.ones(3) / np.sqrt(3.0)
    w = np.array([1.0, -1.0, 0.0]) / np.sqrt(2.0)
    half = np.radians(109.5) / 2
    step_u, step_w = 1.53 * np.sin(half), 1.53 * np.cos(half)
    local = np.array([(k - 2.5) * step_u * u + (0.5 * step_w if k % 2 else -0.5 * step_w) * w
                      for k in range(6)])
    pos = (centres[:, None, :] + local[None] + rng.uniform(-0.05, 0.05, (m, 6, 3)))
    pos = pos.reshape(-1, 3)
    pos -= box * np.floor(pos / box + 0.5)
    n = 6 * m
    q = np.tile([0.2, -0.2, 0.2, -0.2, 0.2, -0.2], m)
    eps = np.full(n, np.sqrt(0.1 * systems.KCAL_TO_IU))
    sig = np.full(n, 1.6)
    mass = np.full(n, 14.0)
    base = 6 * np.arange(m)
    bonds = np.concatenate([np.stack([base + k, base + k + 1], 1) for k in range(5)])
    bonds = bonds.reshape(5, m, 2).transpose(1, 0, 2).reshape(-1, 2).astype(np.int32)
    angles = np.concatenate([np.stack([base + k, base + k + 1, base + k + 2], 1)
                             for k in range(4)]).astype(np.int32)
    dihedrals = np.concatenate([np.stack([base + k, base + k + 1, base + k + 2, base + k + 3], 1)
                                for k in range(3)]).astype(np.int32)
    d = pos[bonds[:, 1]] - pos[bonds[:, 0]]
    d -= box * np.round(d / box)
    sysm = systems.System("chains", box, pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(),
                          q, eps, sig, mass, bonds, angles)
    return sysm, (bonds, (d * d).sum(1)), dihedrals


def test_md_large_molecule_shake_matches_mdbas(gpu, ref_available):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s, cons, dihe = _chain_system()
    vel = systems.thermal_velocities(s.mass, 200.0, seed=3)
    # MDBas's own exclusions (bonds, angles and dihedrals; 1-4 pairs excluded)
    r = oracle.Reference(s, **POT)
    r.set_torsions(dihe, None)
    r.makelist()
    excl = r.get_excl()
    r.close()
    rp, rv, rrows, rself = _ref_md(s, vel, 0.001, 20, 10, cons, dihedrals=dihe)
    gp, gv, grows, st, _ = _gpu_md(s, vel, 0.001, 20, 10, 0, cons, exclusions=excl)
    perr = _pos_err(gp, rp, s.box)
    kin_err = np.max(np.abs(grows[:, 2] - rrows[:, 2]) / rrows[:, 2])
    print(f"chains: pos {perr:.3e} A, kin {kin_err:.3e}, shake iter {st['shake_iter']}")
    assert st["molecules"] == 64
    assert perr < 1e-6
    assert kin_err < 1e-6


@pytest.mark.parametrize("graph", [0, 20])
def test_md_pruned_list_matches_unpruned(gpu, water, graph):
    """Dynamic pruning (inner list at rc + 0.5 A, re-pruned after half that
    displacement) drops only pairs beyond the cut-off, whose contributions
    are exact zeros.  The half-cluster kernel then walks a different sequence
    of j-cluster halves than over the full list, so its FP32 sums of the i
    forces run in another order: the trajectories agree to FP32 rounding,
    and each is bit-for-bit reproducible."""
    vel = (water.vx, water.vy, water.vz)
    cons = water.water_constraints()
    ap, av, arows, ast, _ = _gpu_md(water, vel, 0.002, 60, 0, 1, cons, graph=graph, prune=0.5)
    cp, cv, crows, cst, _ = _gpu_md(water, vel, 0.002, 60, 0, 1, cons, graph=graph, prune=0.5)
    bp, bv, brows, bst, _ = _gpu_md(water, vel, 0.002, 60, 0, 1, cons, graph=graph, prune=0.0)
    print(f"pruned: {ast['prunes']} prunes, {ast['rebuilds']} rebuilds")
    assert ast["pruned_list"] and not bst["pruned_list"]
    assert ast["prunes"] > ast["rebuilds"]
    for k in range(3):
        assert np.array_equal(ap[k], cp[k]) and np.array_equal(av[k], cv[k])
    assert np.array_equal(arows, crows)
    # FP32 rounding differences of the forces (~1e-7 relative) grow over the
    # 120 fs of chaotic dynamics to ~5e-5 A
    perr = _pos_err(ap, bp, water.box)
    print(f"pruned vs unpruned: pos {perr:.3e} A")
    assert perr < 5e-4
    assert np.allclose(arows[:, 1:], brows[:, 1:], rtol=1e-6, atol=0.0)
