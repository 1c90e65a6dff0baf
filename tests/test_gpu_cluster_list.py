"""The mixed form's cluster-pair list against MDBas's own list (oracle/_ref).

The list the timed mixed path builds (precision 1: cell sort, cluster-pair
search) holds, at the list radius rc + delr = 14 A, exactly the unordered
pairs of MDBas's list builder on the same coordinates: the link-cell builder
(src/list.c:1793-2619) where MDBas's makelist picks it, the all-pairs one
(src/list.c:896-1123) otherwise.  Pairs within FP32 rounding of 14 A are
settled by MDBas's own FP64 expression on the GPU, so the sets are equal,
not merely close.
"""
import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems
from dropin_util import DropinSystem, force_rel_rms

pytestmark = pytest.mark.gpu

BIG = 1e30  # export every pair of the list masks


def _reference(s, **kw):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    return oracle.Reference(s, **kw)


def _mdbas_pairs(r):
    """MDBas's list as sorted unordered pairs (int64 keys i * n + j, i < j)."""
    lst, pair, order = r.get_list()
    i = np.repeat(order, pair[order]).astype(np.int64)
    j = lst.astype(np.int64)
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    return np.sort(lo * r.n + hi)


def _engine_pairs(eng, n):
    p = eng.export_pairs(BIG).astype(np.int64)
    keys = np.minimum(p[:, 0], p[:, 1]) * n + np.maximum(p[:, 0], p[:, 1])
    return np.sort(keys)


def _same(a, b):
    assert len(a) == len(b), (len(a), len(b))
    assert np.array_equal(a, b)
    assert len(np.unique(a)) == len(a), "a pair listed twice"


def _images_of_thin_box(keys, n, x, y, z, lengths, rlist=14.0):
    """The cluster list keeps a pair once per periodic image within the list
    radius, with the image's shift in the entry; in a box thinner than twice
    the list radius (but thicker than twice the cut-off, so the pair kernel
    still sees one image) a pair can have two.  MDBas's list holds the
    minimum image only.  Checks that every pair listed twice has a second
    image within the list radius, and returns the keys once each."""
    u, cnt = np.unique(keys, return_counts=True)
    assert cnt.max(initial=1) <= 2
    dup = u[cnt == 2]
    i, j = dup // n, dup % n
    L = np.asarray(lengths, dtype=np.float64)
    d = np.stack([x[j] - x[i], y[j] - y[i], z[j] - z[i]], 1)
    d -= L * np.rint(d / L)
    alt = np.full(len(dup), np.inf)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                if sx == sy == sz == 0:
                    continue
                e = d + L * np.array([sx, sy, sz])
                alt = np.minimum(alt, (e * e).sum(1))
    assert (alt <= (rlist + 1e-3) ** 2).all()
    return u


def _engine_on(r, s, **kw):
    x, y, z = r.positions()
    s2 = systems.System(s.name, s.box, x, y, z, s.q, s.eps, s.sig, s.mass, s.bonds, s.angles)
    return nb.Engine(s2, precision=1, **kw)


def test_cluster_list_link_cells(gpu):
    s = systems.water_box_for_atoms(18558, seed=3)
    r = _reference(s)
    assert r.makelist() == 1
    eng = _engine_on(r, s)
    eng.build()
    _same(_engine_pairs(eng, s.n), _mdbas_pairs(r))
    eng.close()
    r.close()


def test_cluster_list_link_cells_after_motion(gpu):
    s = systems.water_box_for_atoms(18558, seed=4)
    r = _reference(s)
    r.makelist()
    eng = _engine_on(r, s)
    rng = np.random.default_rng(7)
    x, y, z = r.positions()
    # every atom moved up to 0.45 A, some just outside the box (MDBas's list
    # update does not wrap them)
    x = x + rng.uniform(-0.45, 0.45, len(x))
    y = y + rng.uniform(-0.45, 0.45, len(y))
    z = z + rng.uniform(-0.45, 0.45, len(z))
    r.update_list(x, y, z)
    eng.set_positions(x, y, z)
    eng.build()
    _same(_engine_pairs(eng, s.n), _mdbas_pairs(r))
    eng.close()
    r.close()


def test_cluster_list_all_pairs_half_exclusions(gpu):
    # 31 A box: MDBas takes the all-pairs builder, whose exclusion rows are
    # half rows (j > i); the engine is given exactly those rows
    s = systems.config_small(seed=1)
    r = _reference(s)
    assert r.makelist() == 0
    es, ef = r.get_excl()
    eng = _engine_on(r, s, exclusions=(es, ef))
    eng.build()
    _same(_engine_pairs(eng, s.n), _mdbas_pairs(r))
    eng.close()
    r.close()


def test_cluster_list_frozen_atoms(gpu):
    s = systems.config_small(seed=2)
    fz = (np.random.default_rng(3).random(s.n) < 0.1).astype(np.int32)
    r = _reference(s, frozen=fz)
    r.makelist()
    eng = _engine_on(r, s, frozen=fz)
    eng.build()
    _same(_engine_pairs(eng, s.n), _mdbas_pairs(r))
    eng.close()
    r.close()


def test_cluster_list_96k(gpu):
    s = systems.config_96k(seed=1, temperature=None)
    r = _reference(s)
    assert r.makelist() == 1
    eng = _engine_on(r, s)
    eng.build()
    a, b = _engine_pairs(eng, s.n), _mdbas_pairs(r)
    _same(a, b)
    assert len(a) > 55_000_000
    eng.close()
    r.close()


def test_cluster_list_tall_columns(gpu):
    """A 25 x 25 x 700 A water box: 36 columns of ~1,200 atoms, so the
    column sort ranks the columns over 1,024 atoms and sorts the others with
    its 1,024-key network, and the search reads long z tables.  MDBas takes
    its all-pairs builder (fewer than three link cells across x and y).  The
    cluster list's pairs are MDBas's (the box is thinner than twice the list
    radius: some pairs are listed in two images, MDBas's list has their
    minimum image), and the forces and energies match its energy() within
    the mixed tolerance."""
    s = systems.water_box_ortho((25.0, 25.0, 700.0), seed=2)
    cell = s.cell()
    r = _reference(s, box_type=nb.ORBIC, cell=cell)
    assert r.makelist() == 0
    eng = _engine_on(r, s, box_type=nb.ORBIC, cell=cell)
    eng.build()
    x, y, z = r.positions()
    got = _images_of_thin_box(_engine_pairs(eng, s.n), s.n, x, y, z, (25.0, 25.0, 700.0))
    _same(got, _mdbas_pairs(r))
    eng.compute()
    f, e = eng.forces(), eng.energies()
    rfx, rfy, rfz, re = r.energy()
    assert force_rel_rms(f, (rfx, rfy, rfz)) < 1e-5
    elec = e["elec_direct"] + e["elec_corr"]
    assert abs(elec - re["elec"]) <= 1e-5 * abs(re["elec"])
    assert abs(e["vdw"] - re["vdw"]) <= 1e-5 * abs(re["vdw"])
    eng.close()
    r.close()


def test_cluster_list_very_tall_columns(gpu):
    """A 25 x 25 x 2,600 A water box: columns of ~4,500 atoms (over 512
    clusters each, more than the z-table kernel stages in shared memory).
    Too large for MDBas's all-pairs builder on one core, so the cluster list
    is compared with the FP64 form's list (MDBas's own order and pair set,
    pinned to MDBas by the list tests) and the forces with the FP64 form's."""
    s = systems.water_box_ortho((25.0, 25.0, 2600.0), seed=3)
    cell = s.cell()
    eng = nb.Engine(s, precision=1, box_type=nb.ORBIC, cell=cell)
    ref = nb.Engine(s, precision=0, box_type=nb.ORBIC, cell=cell)
    eng.build()
    ref.build()
    got = _images_of_thin_box(_engine_pairs(eng, s.n), s.n, s.x, s.y, s.z, (25.0, 25.0, 2600.0))
    _same(got, _engine_pairs(ref, s.n))
    eng.compute()
    ref.compute()
    assert force_rel_rms(eng.forces(), ref.forces()) < 1e-5
    e, e0 = eng.energies(), ref.energies()
    # the mixed form counts the pairs within its FP32 rc^2: a few at 12 A
    # fall on the other side of the FP64 test
    assert abs(e["n_pairs"] - e0["n_pairs"]) <= 1e-6 * e0["n_pairs"]
    assert abs(e["vdw"] - e0["vdw"]) <= 1e-5 * abs(e0["vdw"])
    eng.close()
    ref.close()


def test_mixed_dropin_all_pairs_half_rows(gpu):
    # the mixed drop-in on MDBas's all-pairs path: half exclusion rows from
    # exclude_list reach the cluster search, which must still drop every
    # excluded pair from the direct sum
    s = systems.config_small(seed=2)
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(1)
    try:
        d = DropinSystem(s)
        assert d.makelist() == 0
        fx, fy, fz, e = d.energy()
    finally:
        L.mdbas_nb_set_mode(0)
    r = _reference(s)
    r.makelist()
    rfx, rfy, rfz, re = r.energy()
    assert force_rel_rms((fx, fy, fz), (rfx, rfy, rfz)) < 1e-5
    for k in ("elec", "vdw"):
        assert abs(e[k] - re[k]) <= 1e-5 * abs(re[k]), k
    d.free()
    r.close()
