"""GPU force/energy parity.

* plain FP64 form: against MDBas's own energy() (relative 1e-12: only CUDA's
  erfc/exp and the FP64 atomic order differ from the CPU build);
* FP32 pair arithmetic + fixed-point accumulation: against the FP64
  restatement, per-atom force RMS relative error <= 1e-5 and energy
  relative error <= 1e-5; the evaluated pair set equals MDBas's.
"""
import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems
from dropin_util import force_rel_rms

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_FORCE_TOL = 1e-5
MIXED_ENERGY_TOL = 1e-5


def _oracle_fp64(s, link=None):
    o = oracle.Oracle()
    box = o.box(s.cell())
    ok, _ = o.link_cell_counts(box)
    if link is None:
        link = ok
    if link:
        excl = s.exclusions(symmetric=True)
        lst, pair, order = o.link_cell_list(box, s.x, s.y, s.z, excl)
    else:
        excl = s.exclusions(symmetric=False)
        lst, pair, order = o.verlet_list(box, s.x, s.y, s.z, excl)
    fx, fy, fz, e = o.ewald_energy(box, s, lst, pair, order, excl)
    return (fx, fy, fz), e


@pytest.mark.parametrize("which", ["small", "link"])
def test_fp64_form_matches_reference(gpu, which):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    s = systems.config_small(1) if which == "small" else systems.water_box_for_atoms(18558, 3)
    r = oracle.Reference(s)
    r.makelist()
    rx, ry, rz = r.positions()
    rf = r.energy()
    s.x, s.y, s.z = rx, ry, rz
    eng = nb.Engine(s, precision=0)
    eng.build()
    eng.compute()
    f = eng.forces()
    e = eng.energies()
    assert force_rel_rms(f, rf[:3]) < FP64_TOL
    elec = e["elec_direct"] + e["elec_corr"]
    assert abs(elec - rf[3]["elec"]) <= FP64_TOL * abs(rf[3]["elec"])
    assert abs(e["vdw"] - rf[3]["vdw"]) <= FP64_TOL * abs(rf[3]["vdw"])
    vir = e["vir_direct"] + e["vir_corr"]
    assert abs(vir - rf[3]["virelec"]) <= FP64_TOL * abs(rf[3]["virelec"])
    # MDBas sums q^2 sequentially in FP64 (its own rounding is ~1e-13 here)
    assert abs(e["elec_self"] - r.self_energy()) <= 1e-12 * abs(r.self_energy())
    eng.close()


@pytest.mark.parametrize("which", ["small", "link", "ljfluid"])
def test_mixed_form_accuracy(gpu, which):
    if which == "small":
        s = systems.config_small(1)
    elif which == "link":
        s = systems.water_box_for_atoms(18558, 3)
    else:
        s = systems.lj_fluid(12000, 50.0, seed=1)
    rf, re = _oracle_fp64(s)
    eng = nb.Engine(s, precision=1)
    eng.build()
    eng.compute()
    f = eng.forces()
    e = eng.energies()
    err = force_rel_rms(f, rf)
    assert err < MIXED_FORCE_TOL, err
    relec = re["e_dir"] + re["e_corr"]
    elec = e["elec_direct"] + e["elec_corr"]
    assert abs(elec - relec) <= MIXED_ENERGY_TOL * abs(relec)
    assert abs(e["vdw"] - re["e_vdw"]) <= MIXED_ENERGY_TOL * max(abs(re["e_vdw"]), 1.0)
    vir = e["vir_direct"] + e["vir_corr"] + e["vir_vdw"]
    rvir = re["vir_dir"] + re["vir_corr"] + re["vir_vdw"]
    assert abs(vir - rvir) <= MIXED_ENERGY_TOL * abs(rvir)
    assert abs(e["n_pairs"] - re["n_pairs"]) <= 2
    eng.close()


def test_mixed_pair_set_equals_reference(gpu):
    s = systems.water_box_for_atoms(18558, 3)
    o = oracle.Oracle()
    box = o.box(s.cell())
    excl = s.exclusions(symmetric=True)
    ref = o.pairs_within(box, s.x, s.y, s.z, excl, 144.0)
    eng = nb.Engine(s, precision=1)
    eng.build()
    got = eng.export_pairs(144.0)
    a = set(map(tuple, ref.tolist()))
    b = set(map(tuple, got.tolist()))
    assert len(got) == len(b), "a pair was evaluated twice"
    diff = a ^ b
    # only pairs within FP32 rounding of the cut-off may differ
    pos = np.stack([s.x, s.y, s.z], 1)
    for i, j in diff:
        d = pos[j] - pos[i]
        d -= s.box * np.round(d / s.box)
        assert abs(np.sqrt(d @ d) - 12.0) < 1e-4, (i, j)
    eng.close()


def test_mixed_deterministic_and_permutation_invariant(gpu):
    s = systems.water_box_for_atoms(18558, 6)
    eng = nb.Engine(s, precision=1)
    eng.build()
    eng.compute()
    f1 = eng.forces()
    e1 = eng.energies()
    eng.compute()
    f2 = eng.forces()
    eng.build()
    eng.compute()
    f3 = eng.forces()
    e3 = eng.energies()
    for a, b, c in zip(f1, f2, f3):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    assert e1 == e3
    eng.close()
    # permute the atoms (exclusions follow): same forces bit for bit
    perm = np.random.default_rng(11).permutation(s.n)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(s.n)
    sp = systems.System(s.name, s.box, s.x[perm], s.y[perm], s.z[perm], s.q[perm], s.eps[perm],
                        s.sig[perm], s.mass[perm], inv[s.bonds].astype(np.int32),
                        inv[s.angles].astype(np.int32))
    engp = nb.Engine(sp, precision=1)
    engp.build()
    engp.compute()
    fp = engp.forces()
    ep = engp.energies()
    for a, b in zip(f1, fp):
        assert np.array_equal(a[perm], b)
    assert ep == e1
    engp.close()


def test_refresh_between_builds(gpu):
    # moving atoms by less than half the skin and refreshing must give the
    # same forces as a full rebuild at the new positions
    s = systems.water_box_for_atoms(18558, 8)
    eng = nb.Engine(s, precision=1)
    eng.build()
    rng = np.random.default_rng(2)
    x = s.x + rng.uniform(-0.4, 0.4, s.n)
    y = s.y + rng.uniform(-0.4, 0.4, s.n)
    z = s.z + rng.uniform(-0.4, 0.4, s.n)
    eng.set_positions(x, y, z)
    eng.refresh()
    eng.compute()
    f_ref = eng.forces()
    e_ref = eng.energies()
    eng.build()
    eng.compute()
    f_new = eng.forces()
    e_new = eng.energies()
    assert force_rel_rms(f_ref, f_new) < 2 * MIXED_FORCE_TOL
    assert e_ref["n_pairs"] == e_new["n_pairs"]
    eng.close()


def test_pair_kernel_variants_agree(gpu):
    s = systems.water_box_for_atoms(18558, 3)
    eng = nb.Engine(s, precision=1)
    eng.build()
    out = {}
    for v in (0, 1, 2, 3):
        eng.set_variant(v)
        eng.compute()
        out[v] = (eng.forces(), eng.energies())
    # packed f32x2 with per-lane loads (2) and with bulk-copy staging (3): the
    # same arithmetic, bit for bit
    for k in range(3):
        assert np.array_equal(out[2][0][k], out[3][0][k])
    assert out[2][1] == out[3][1]
    assert force_rel_rms(out[2][0], out[0][0]) < 2e-6
    assert force_rel_rms(out[1][0], out[0][0]) < 2e-6
    assert out[1][1]["n_pairs"] == out[0][1]["n_pairs"]
    e0, e1 = out[0][1], out[1][1]
    # the direct sum cancels heavily; compare on the scale of the total
    scale = abs(e0["elec_direct"] + e0["elec_corr"])
    assert abs(e1["elec_direct"] - e0["elec_direct"]) <= 1e-6 * scale
    eng.close()


def test_quad_kernel_variants(gpu):
    """The 4 x 4 kernel (i-cluster halves against j-cluster halves of the
    inner list) gives the same pair count as the 8 x 4 half kernel and its
    forces within FP32 rounding; repeated evaluations are bitwise
    identical."""
    s = systems.water_box_for_atoms(18558, 3)
    eng = nb.Engine(s, precision=1)
    eng.build()
    out = {}
    for v in (4, 6):
        eng.set_variant(v)
        eng.compute()
        out[v] = (eng.forces(), eng.energies())
    eng.compute()
    again = (eng.forces(), eng.energies())
    for k in range(3):
        assert np.array_equal(out[6][0][k], again[0][k])
    assert out[6][1] == again[1]
    assert out[6][1]["n_pairs"] == out[4][1]["n_pairs"]
    assert force_rel_rms(out[6][0], out[4][0]) < 2e-6
    e4, e6 = out[4][1], out[6][1]
    scale = abs(e4["elec_direct"] + e4["elec_corr"])
    assert abs(e6["elec_direct"] - e4["elec_direct"]) <= 1e-6 * scale
    assert abs(e6["vdw"] - e4["vdw"]) <= 1e-6 * abs(e4["vdw"])
    assert abs(e6["vir_direct"] - e4["vir_direct"]) <= 1e-6 * abs(e4["vir_direct"])
    eng.close()


def test_quad_kernel_in_pruned_dynamics(gpu):
    """Dynamics with a pruned inner list (rc + 0.5 A, so the kernel tests
    the cut-off itself) on the 4 x 4 kernel follow the 8 x 4 kernel's
    trajectory to FP32 rounding."""
    s = systems.water_box(1000, 31.0, seed=5, temperature=300.0)
    rows = {}
    pos = {}
    for v in (4, 6):
        e = nb.Engine(s, precision=1)
        e.set_variant(v)
        e.md_set_graph(0)
        e.md_set_prune(0.5)
        e.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.002, list_update=0,
                  constraints=s.water_constraints())
        rows[v] = e.md_run(40, energy_every=1)
        pos[v] = e.positions()
        assert e.md_stats()["pruned_list"]
        e.close()
    err = max(np.max(np.abs(pos[4][k] - pos[6][k])) for k in range(3))
    assert err < 5e-4, err
    assert np.allclose(rows[4][:, 1:], rows[6][:, 1:], rtol=1e-6, atol=0.0)


def test_evaluate_equals_separate_calls(gpu):
    """mdbas_nb_engine_evaluate (positions in, forces and energies out, one
    call) gives the results of set_positions + build/refresh + compute +
    get_forces + energies made one by one, bit for bit, with a rebuild and
    with a refresh after motion within the skin."""
    s = systems.water_box_for_atoms(18558, seed=6)
    a = nb.Engine(s, precision=1)
    b = nb.Engine(s, precision=1)
    rng = np.random.default_rng(11)
    x, y, z = s.x.copy(), s.y.copy(), s.z.copy()
    for rebuild in (True, False, True):
        fx, fy, fz = (np.zeros(s.n) for _ in range(3))
        ea = a.evaluate(x, y, z, fx, fy, fz, rebuild=rebuild)
        b.set_positions(x, y, z)
        if rebuild:
            b.build()
        else:
            b.refresh()
        b.compute()
        gx, gy, gz = b.forces()
        eb = b.energies()
        for u, v in ((fx, gx), (fy, gy), (fz, gz)):
            assert np.array_equal(u, v)
        assert ea == eb
        # move every atom by at most 0.3 A (within half the 2 A skin)
        x, y, z = (v + rng.uniform(-0.3, 0.3, s.n) for v in (x, y, z))
    with pytest.raises(ValueError):
        a.evaluate(x, y, z, np.zeros(s.n, np.float32), fy, fz)

    def separate(px, py, pz):
        b.set_positions(px, py, pz)
        b.build()
        b.compute()
        return b.forces(), b.energies()

    # the same array objects again with their contents changed in place (the
    # kept pointer arguments read the new values), and float32 positions,
    # converted on every call
    fx, fy, fz = (np.zeros(s.n) for _ in range(3))
    x, y, z = s.x.copy(), s.y.copy(), s.z.copy()
    a.evaluate(x, y, z, fx, fy, fz)
    for shift in (0.05, 0.1):
        x += shift
        ea = a.evaluate(x, y, z, fx, fy, fz)
        g, eb = separate(x, y, z)
        assert all(np.array_equal(u, v) for u, v in zip((fx, fy, fz), g)) and ea == eb
    x32, y32, z32 = (v.astype(np.float32) for v in (s.x, s.y, s.z))
    for shift in (0.0, 0.125):
        x32 += np.float32(shift)
        ea = a.evaluate(x32, y32, z32, fx, fy, fz)
        g, eb = separate(*(v.astype(np.float64) for v in (x32, y32, z32)))
        assert all(np.array_equal(u, v) for u, v in zip((fx, fy, fz), g)) and ea == eb
    a.close()
    b.close()


def test_lean_half_kernel_matches_half(gpu):
    """The lean form of the half-cluster kernel (variant 7: masked pairs at
    r^2 = 1e30 instead of zeroed products, items from a counter) gives the
    first form's forces and energies bit for bit, over the exact inner list
    and over the full list once the atoms have moved."""
    s = systems.water_box_for_atoms(18558, 3)
    eng = nb.Engine(s, precision=1)
    eng.build()
    out = {}
    for v in (4, 7):
        eng.set_variant(v)
        eng.compute()
        out[v] = (eng.forces(), eng.energies())
    for k in range(3):
        assert np.array_equal(out[4][0][k], out[7][0][k])
    assert out[4][1] == out[7][1]
    # moved atoms, layout refreshed: the inner list is stale and both forms
    # walk the full list
    rng = np.random.default_rng(5)
    eng.set_positions(*(v + rng.uniform(-0.3, 0.3, s.n) for v in (s.x, s.y, s.z)))
    eng.refresh()
    for v in (4, 7):
        eng.set_variant(v)
        eng.compute()
        out[v] = (eng.forces(), eng.energies())
    for k in range(3):
        assert np.array_equal(out[4][0][k], out[7][0][k])
    assert out[4][1] == out[7][1]
    eng.close()

