"""GPU bonded terms (mdbas_b200/csrc/bonded.cu) against MDBas's own
bond_energy / angle_energy / ub_energy / dihedral_energy / improper_energy
(src/internal.c, compiled into oracle/_ref).

Each force component receives the terms' contributions in MDBas's order and
the kernels are compiled without FMA contraction, so harmonic bonds and
Urey-Bradley terms (no library function) give MDBas's forces bit for bit;
Morse bonds, angles and torsions (exp, acos, atan2, cos, sin) agree to 1e-12
of the largest force.  Energies are block sums (order differs): 1e-12
relative.  Dynamics with bonded terms (no constraints) then follow MDBas's
vv_integrate + energy() trajectory."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

import bonded_util

pytestmark = pytest.mark.gpu

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
KINDS = list(enumerate(nb.BONDED_KINDS))


@pytest.fixture(scope="module")
def chains():
    return systems.flexible_chains(4, 26.0, seed=3, jitter=0.08)


@pytest.fixture(scope="module")
def start_forces(chains):
    rng = np.random.default_rng(11)
    return [rng.normal(scale=300.0, size=chains.n) for _ in range(3)]


def _ref_lib():
    import oracle
    return oracle.Reference.lib()


@pytest.mark.parametrize("kind,name", KINDS)
def test_bonded_routine_matches_mdbas(gpu, ref_available, chains, start_forces, kind, name):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    structs = nb.bonded_structs(chains.meta["bonded"])
    e_ref, v_ref, *fref = bonded_util.call(_ref_lib(), kind, chains, structs, start_forces)
    e, v, *f = nb.bonded(kind, chains, structs[kind][1] if structs[kind][0] else None,
                         start_forces)
    scale = max(np.max(np.abs(a - b)) for a, b in zip(fref, start_forces))
    err = max(np.max(np.abs(a - b)) for a, b in zip(f, fref))
    print(f"{name}: E {e:.10e} vs {e_ref:.10e}, max|dF| {err / scale:.2e} of the largest")
    assert scale > 0
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    assert abs(v - v_ref) <= 1e-12 * max(abs(v_ref), 1.0)
    assert err <= 1e-12 * scale
    if name == "ub":
        for a, b in zip(f, fref):
            assert np.array_equal(a, b)


def test_harmonic_bonds_bit_identical(gpu, ref_available, chains, start_forces):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    spec = dict(chains.meta["bonded"]["bonds"])
    spec["type"] = np.zeros_like(spec["type"])
    structs = nb.bonded_structs({"bonds": spec})
    e_ref, v_ref, *fref = bonded_util.call(_ref_lib(), 0, chains, structs, start_forces)
    e, v, *f = nb.bonded(0, chains, structs[0][1], start_forces)
    for a, b in zip(f, fref):
        assert np.array_equal(a, b)
    assert abs(e - e_ref) <= 1e-13 * abs(e_ref)


@pytest.mark.parametrize("kind,name", KINDS)
def test_dropin_prototypes_match_mdbas(gpu, ref_available, chains, start_forces, kind, name):
    """libmdbas_nb's bond_energy ... improper_energy (MDBas's prototypes)
    fill ENERGY like MDBas's routines."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    structs = nb.bonded_structs(chains.meta["bonded"])
    ref = bonded_util.call(_ref_lib(), kind, chains, structs, start_forces)
    got = bonded_util.call(nb.bind_dropin(), kind, chains, structs, start_forces)
    assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
    assert abs(got[1] - ref[1]) <= 1e-12 * max(abs(ref[1]), 1.0)
    scale = max(np.max(np.abs(a)) for a in ref[2:])
    for a, b in zip(got[2:], ref[2:]):
        assert np.max(np.abs(a - b)) <= 1e-12 * scale


def test_bonded_edge_cases(gpu, chains):
    structs = nb.bonded_structs(chains.meta["bonded"])
    # no terms: nothing added
    e, v, fx, fy, fz = nb.bonded(0, chains, None)
    assert e == 0.0 and v == 0.0 and not (fx.any() or fy.any() or fz.any())
    # an atom index outside the system is refused before any launch
    bad = nb.bonded_structs({"bonds": dict(atoms=np.array([[0, chains.n]]), k=[1.0], r0=[1.0])})
    with pytest.raises(nb.MdbasNbError) as ei:
        nb.bonded(0, chains, bad[0][1])
    assert ei.value.status == 1
    # the terms cache follows changed parameters
    spec = {k: dict(v) for k, v in chains.meta["bonded"].items()}
    e1 = nb.bonded(1, chains, structs[1][1])[0]
    spec["angles"]["k"] = 2.0 * spec["angles"]["k"]
    e2 = nb.bonded(1, chains, nb.bonded_structs(spec)[1][1])[0]
    assert e2 == pytest.approx(2.0 * e1, rel=1e-14)


@pytest.mark.parametrize("precision", [0, 1])
def test_engine_bonded_matches_mdbas(gpu, ref_available, chains, start_forces, precision):
    """Engine-held terms: all five kinds in one launch, forces added in
    energy()'s order (bonds, angles, Urey-Bradley, dihedrals, impropers)."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    structs = nb.bonded_structs(chains.meta["bonded"])
    f = [a.copy() for a in start_forces]
    ref_e = {}
    for kind, name in KINDS:
        e, v, *f = bonded_util.call(_ref_lib(), kind, chains, structs, f)
        ref_e[name] = (e, v)
    eng = nb.Engine(chains, precision=precision, **POT)
    eng.set_bonded(chains.meta["bonded"])
    got, fg = eng.bonded(start_forces)
    eng.close()
    scale = max(np.max(np.abs(a - b)) for a, b in zip(f, start_forces))
    assert max(np.max(np.abs(a - b)) for a, b in zip(fg, f)) <= 1e-12 * scale
    for (kind, name), key in zip(KINDS, nb.BONDED_ENERGIES):
        assert abs(got[key] - ref_e[name][0]) <= 1e-12 * abs(ref_e[name][0])
    assert abs(got["vir_bond"] - ref_e["bonds"][1]) <= 1e-12 * abs(ref_e["bonds"][1])
    assert abs(got["vir_ub"] - ref_e["ub"][1]) <= 1e-12 * abs(ref_e["ub"][1])


def _ref_md_bonded(s, vel, dt, steps, list_update):
    import oracle
    r = oracle.Reference(s, **POT)
    r.set_bonded(nb.bonded_structs(s.meta["bonded"]))
    r.makelist()
    excl = r.get_excl()
    r.md_init(s.mass, vel, time_step=dt, list_update=list_update)
    rows = r.md_run(steps)
    out = r.positions(), r.velocities(), rows, r.self_energy(), excl
    r.close()
    return out


def _gpu_md_bonded(s, vel, dt, steps, list_update, precision, excl, graph=None):
    e = nb.Engine(s, precision=precision, exclusions=excl, **POT)
    e.set_bonded(s.meta["bonded"])
    if graph is not None:
        e.md_set_graph(graph)
    e.md_init(s.mass, vel, time_step=dt, list_update=list_update)
    rows = e.md_run(steps, energy_every=1)
    out = e.positions(), e.velocities(), rows
    e.close()
    return out


def _pos_err(a, b, box):
    return max(np.max(np.abs((np.asarray(a[k]) - np.asarray(b[k]))
                             - box * np.round((np.asarray(a[k]) - np.asarray(b[k])) / box)))
               for k in range(3))


def test_md_flexible_chains_fp64_matches_mdbas(gpu, ref_available):
    """Flexible chains (no constraints) for 20 steps of 0.5 fs: the FP64 form
    follows MDBas's trajectory to round-off."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.flexible_chains(4, 26.0, seed=5, temperature=300.0)
    vel = (s.vx, s.vy, s.vz)
    rp, rv, rrows, rself, excl = _ref_md_bonded(s, vel, 0.0005, 20, 10)
    gp, gv, grows = _gpu_md_bonded(s, vel, 0.0005, 20, 10, 0, excl)
    perr = _pos_err(gp, rp, s.box)
    verr = max(np.max(np.abs(gv[k] - rv[k])) for k in range(3))
    tot_err = np.max(np.abs(grows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    pot_err = np.max(np.abs(grows[:, 1] - (rrows[:, 1] + rself))) / np.max(np.abs(rrows[:, 1]))
    print(f"flexible chains fp64: pos {perr:.3e} A, vel {verr:.3e}, pot {pot_err:.3e}, "
          f"total {tot_err:.3e}")
    assert perr < 1e-9
    assert verr < 1e-6
    assert pot_err < 1e-10
    assert tot_err < 1e-10


def test_md_flexible_chains_mixed_graph(gpu, ref_available):
    """Mixed precision with bonded terms: the graph form equals the
    host-driven form bit for bit and both track MDBas."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.flexible_chains(4, 26.0, seed=5, temperature=300.0)
    vel = (s.vx, s.vy, s.vz)
    rp, rv, rrows, rself, excl = _ref_md_bonded(s, vel, 0.0005, 20, 10)
    ap, av, arows = _gpu_md_bonded(s, vel, 0.0005, 20, 10, 1, excl, graph=20)
    bp, bv, brows = _gpu_md_bonded(s, vel, 0.0005, 20, 10, 1, excl, graph=0)
    for k in range(3):
        assert np.array_equal(ap[k], bp[k])
        assert np.array_equal(av[k], bv[k])
    assert np.array_equal(arows, brows)
    perr = _pos_err(ap, rp, s.box)
    tot_err = np.max(np.abs(arows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    print(f"flexible chains mixed: pos {perr:.3e} A, total {tot_err:.3e}")
    assert perr < 1e-4
    assert tot_err < 1e-5


def test_md_flexible_chains_nve_conserves_energy(gpu):
    """2,000 steps of 0.5 fs NVE with every bonded kind: the total energy
    stays within 0.5% of the kinetic energy scale (no drift from the
    bonded forces or their order of accumulation)."""
    s = systems.flexible_chains(4, 26.0, seed=7, temperature=300.0)
    e = nb.Engine(s, precision=1, **POT)
    e.set_bonded(s.meta["bonded"])
    e.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.0005, list_update=0)
    rows = e.md_run(2000, energy_every=100)
    e.close()
    tot, kin = rows[:, 3], rows[:, 2]
    spread = np.max(tot) - np.min(tot)
    print(f"NVE chains: total spread {spread:.3e}, mean kin {np.mean(kin):.3e}")
    assert np.all(np.isfinite(rows))
    assert spread < 5e-3 * np.mean(kin)
