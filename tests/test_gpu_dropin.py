"""The drop-in C ABI (MDBas prototypes) end to end on the GPU."""
import ctypes as C

import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems
from dropin_util import DropinSystem, force_rel_rms

pytestmark = pytest.mark.gpu


def _ref_energy(s, **kw):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    r = oracle.Reference(s, **kw)
    r.makelist()
    return r, r.energy()


@pytest.mark.parametrize("which", ["small", "link"])
def test_energy_dropin_fp64(gpu, which):
    s = systems.config_small(1) if which == "small" else systems.water_box_for_atoms(18558, 3)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    d = DropinSystem(s)
    d.makelist()
    fx, fy, fz, e = d.energy()
    r, (rfx, rfy, rfz, re) = _ref_energy(s)
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < 1e-12
    for k in ("elec", "vdw", "virelec", "virvdw", "pot", "virpot"):
        assert abs(e[k] - re[k]) <= 1e-12 * abs(re[k]), k
    d.free()


def test_energy_dropin_mixed(gpu):
    s = systems.water_box_for_atoms(18558, 3)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(1)
    try:
        d = DropinSystem(s)
        d.makelist()
        fx, fy, fz, e = d.energy()
        # a second call reuses the cluster list (nothing moved)
        fx2, fy2, fz2, e2 = d.energy()
    finally:
        L.mdbas_nb_set_mode(0)
    r, (rfx, rfy, rfz, re) = _ref_energy(s)
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < 1e-5
    assert abs(e["elec"] - re["elec"]) <= 1e-5 * abs(re["elec"])
    assert np.array_equal(fx, fx2) and e == e2
    d.free()


def test_plugin_matches_ewald_energy(gpu):
    s = systems.config_small(2)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    d = DropinSystem(s)
    d.makelist()
    fx, fy, fz, e = d.energy()
    pair = np.ctypeslib.as_array(d.exclPair, (s.n,)).copy()
    assert L.mdbas_nb_plugin_init(s.n, nb.as_dp(d.q), nb.as_dp(d.eps), nb.as_dp(d.sig),
                                  nb.as_ip(pair), d.exclList, 0.34, 1) == 0
    px, py, pz = np.zeros(s.n), np.zeros(s.n), np.zeros(s.n)
    etot = L.mdbas_nb_user_energy(C.byref(d.param), C.byref(d.box), nb.as_dp(d.x),
                                  nb.as_dp(d.y), nb.as_dp(d.z), nb.as_dp(px), nb.as_dp(py),
                                  nb.as_dp(pz), d.neighList, d.neighPair, d.neighOrder,
                                  d.neighList14)
    assert force_rel_rms((px, py, pz), (fx, fy, fz)) < 1e-13
    assert abs(etot - (e["elec"] + e["vdw"])) <= 1e-12 * abs(e["elec"])
    out = np.zeros(4)
    assert L.mdbas_nb_plugin_last_energy(nb.as_dp(out)) == 0
    assert abs(out[2] - e["virelec"]) <= 1e-12 * abs(e["virelec"])
    d.free()


def test_status_forms_report_instead_of_exit(gpu):
    # a 31 A box has 2 link cells per side: the link-cell builder must refuse
    s = systems.config_small(1)
    L = nb.bind_dropin()
    d = DropinSystem(s)
    lst = C.POINTER(C.c_int)()
    pair = C.POINTER(C.c_int)()
    order = C.POINTER(C.c_int)()
    excl = (C.POINTER(C.c_int) * s.n)()
    ep = np.zeros(s.n, np.int32)
    st = L.mdbas_nb_link_cell_list_status(C.byref(d.param), C.byref(d.box), C.byref(d.neigh),
                                          nb.as_dp(d.x), nb.as_dp(d.y), nb.as_dp(d.z),
                                          nb.as_ip(d.frozen), C.byref(lst), C.byref(pair),
                                          C.byref(order), excl, nb.as_ip(ep), 0)
    assert st == 7  # MDBAS_NB_ERR_LINKCELL (MDBas LNKCELL_NCELLS_ERROR)
    # non-finite coordinates are rejected by the engine, not computed
    s2 = systems.config_small(1)
    s2.x = s2.x.copy()
    s2.x[5] = np.nan
    eng = nb.Engine(s2, precision=1)
    with pytest.raises(nb.MdbasNbError) as ei:
        eng.build()
    assert ei.value.status == 11
    eng.close()


@pytest.mark.parametrize("elec,vdw", [(nb.SHIFT1, nb.VSWITCH), (nb.SHIFT2, nb.VSWITCH),
                                      (nb.SWITCH, nb.VSWITCH), (nb.SHIFT1, nb.NOVDW),
                                      (nb.NOELEC, nb.VSWITCH)])
@pytest.mark.parametrize("which", ["small", "link"])
def test_energy_dropin_cutoff_coulomb(gpu, which, elec, vdw):
    """energy() with keyEwald = 0: the drop-in's nonbond_energy (cut-off
    Coulomb forms, FP64 on the GPU) against MDBas's own, in either mode."""
    s = systems.config_small(4) if which == "small" else systems.water_box_for_atoms(18558, 6)
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    r = oracle.Reference(s)
    r.set_nonbond(elec, vdw)
    r.makelist()
    rfx, rfy, rfz, re = r.energy()
    r.close()
    L = nb.bind_dropin()
    for mode in (0, 1):
        L.mdbas_nb_set_mode(mode)
        try:
            d = DropinSystem(s, keyEwald=0)
            d.ctrl.elecType = elec
            d.ctrl.vdwType = vdw
            d.makelist()
            fx, fy, fz, e = d.energy()
        finally:
            L.mdbas_nb_set_mode(0)
        assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < 1e-12
        for k in ("elec", "vdw", "virelec", "virvdw", "pot", "virpot"):
            assert abs(e[k] - re[k]) <= 1e-12 * abs(re[k]), (mode, k)
        d.free()


@pytest.mark.parametrize("key", ["ewald", "shift1"])
def test_energy_dropin_pairs14(gpu, key):
    """energy() with keyNb14: the drop-in's 1-4 list (from the dihedrals) and
    its ewald14_energy / nonbond14_energy (scal14 = 0.5) against MDBas's."""
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    s = systems.flexible_chains(4, 26.0, seed=7, jitter=0.08)
    dihe = np.asarray(s.meta["dihedrals"])
    r = oracle.Reference(s)
    if key == "shift1":
        r.set_nonbond(nb.SHIFT1, nb.VSWITCH)
    r.set_nb14(0.5, dihe)
    r.makelist()
    rl14 = r.list14()
    rfx, rfy, rfz, re = r.energy()
    r.close()
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    d = DropinSystem(s, keyEwald=3 if key == "ewald" else 0)
    if key == "shift1":
        d.ctrl.elecType = nb.SHIFT1
    d.ctrl.keyNb14 = 1
    d.param.scal14 = 0.5
    arr = (nb.DIHE * len(dihe))()
    for k, (a, b, c, e4) in enumerate(dihe.tolist()):
        arr[k].a, arr[k].b, arr[k].c, arr[k].d = a, b, c, e4
    d.dihe = arr
    d.param.nDihedral = len(dihe)
    d.makelist()
    n14 = d.neigh.nPair14
    assert n14 == len(rl14) // 2 > 0
    assert [d.neighList14[k] for k in range(2 * n14)] == rl14.tolist()
    d.param.nDihedral = 0      # the dihedral terms themselves stay off, as in the reference
    fx, fy, fz, e = d.energy()
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < 1e-12
    for k in ("elec", "vdw", "virelec", "virvdw"):
        assert abs(e[k] - re[k]) <= 1e-12 * abs(re[k]), k
    d.free()


def _excl_rows(start, flat):
    """MDBas-style exclusion rows (int **, int *) from CSR arrays."""
    n = len(start) - 1
    rows = [(C.c_int * max(1, int(start[i + 1] - start[i])))(*flat[start[i]:start[i + 1]])
            for i in range(n)]
    lst = (C.POINTER(C.c_int) * n)(*[C.cast(r, C.POINTER(C.c_int)) for r in rows])
    pair = np.diff(start).astype(np.int32)
    return rows, lst, pair


def test_plugin_follows_list_rebuilt_in_place(gpu):
    """Behind the plugin entry MDBas's own list.c owns the list and refills
    the same arrays in place (src/list.c:2276-2279, 2565-2574).  Two water
    molecules swap places: the update keeps the arrays and the entry count
    but changes which atoms pair up, and the plugin must use the new list."""
    s = systems.water_box_for_atoms(18558, 3)
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    r = oracle.Reference(s)
    assert r.makelist() == 1
    x, y, z = r.positions()
    es, ef = r.get_excl()
    rows, excl, epair = _excl_rows(es, ef)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    d = DropinSystem(s)
    assert L.mdbas_nb_plugin_init(s.n, nb.as_dp(d.q), nb.as_dp(d.eps), nb.as_dp(d.sig),
                                  nb.as_ip(epair), excl, 0.34, 1) == 0
    lst, pair, order = r.list_ptrs()
    none = C.POINTER(C.c_int)()

    def plugin(xa, ya, za):
        fx, fy, fz = np.zeros(s.n), np.zeros(s.n), np.zeros(s.n)
        xa, ya, za = (np.ascontiguousarray(a, dtype=np.float64) for a in (xa, ya, za))
        L.mdbas_nb_user_energy(C.byref(d.param), C.byref(d.box), nb.as_dp(xa), nb.as_dp(ya),
                               nb.as_dp(za), nb.as_dp(fx), nb.as_dp(fy), nb.as_dp(fz), lst,
                               pair, order, none)
        return fx, fy, fz

    f1 = plugin(x, y, z)
    rfx, rfy, rfz, _ = r.energy()
    assert force_rel_rms(f1, (rfx, rfy, rfz)) < 1e-12
    before = r.get_list()
    # swap two molecules far apart (every atom keeps its role: O with O)
    m1, m2 = 10, s.n // 3 - 10
    for a in (x, y, z):
        t = a[3 * m1:3 * m1 + 3].copy()
        a[3 * m1:3 * m1 + 3] = a[3 * m2:3 * m2 + 3]
        a[3 * m2:3 * m2 + 3] = t
    r.update_list(x, y, z)
    after = r.get_list()
    assert len(after[0]) == len(before[0]), "the swap keeps the entry count"
    assert not np.array_equal(after[0], before[0]), "the swap changes the list"
    addr = [C.cast(q, C.c_void_p).value for q in (lst, pair, order)]
    assert [C.cast(q, C.c_void_p).value for q in r.list_ptrs()] == addr, "same arrays"
    f2 = plugin(x, y, z)
    rfx, rfy, rfz, _ = r.energy()
    assert force_rel_rms(f2, (rfx, rfy, rfz)) < 1e-12
    d.free()
    r.close()
