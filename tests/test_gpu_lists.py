"""GPU list builders against MDBas: same entries, same order (bit-exact)."""
import numpy as np
import pytest

import oracle
from mdbas_b200 import systems
from dropin_util import DropinSystem

pytestmark = pytest.mark.gpu


def _reference(s, **kw):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    r = oracle.Reference(s, **kw)
    return r


def _compare(d, r):
    lst, pair, order = d.get_list()
    rl, rp, ro = r.get_list()
    assert len(lst) == len(rl)
    assert np.array_equal(pair, rp)
    assert np.array_equal(order, ro)
    assert np.array_equal(lst, rl)
    assert d.neigh.sizeList == r.size_list
    return len(lst)


def test_all_pairs_list_small_box(gpu):
    s = systems.config_small(seed=1)
    d = DropinSystem(s)
    r = _reference(s)
    assert d.makelist() == 0 and r.makelist() == 0
    # entries, order and sizeList equal MDBas's (asserted inside _compare);
    # the 31 A box holds ~582 list pairs per atom at 14 A
    n = _compare(d, r)
    assert 1_700_000 < n < 1_800_000, n
    es, ef = d.get_excl()
    rs, rf = r.get_excl()
    assert np.array_equal(es, rs) and np.array_equal(ef, rf)
    d.free()


@pytest.mark.parametrize("ratio", [1, 2])
def test_link_cell_list(gpu, ratio):
    s = systems.water_box_for_atoms(18558, seed=3)
    d = DropinSystem(s, linkRatio=ratio)
    r = _reference(s, linkRatio=ratio)
    assert d.makelist() == 1 and r.makelist() == 1
    assert d.neigh.nCells == r.n_cells
    _compare(d, r)
    # the first build wraps the caller's coordinates in place, like MDBas
    rx, ry, rz = r.positions()
    assert np.array_equal(d.x, rx) and np.array_equal(d.y, ry) and np.array_equal(d.z, rz)
    es, ef = d.get_excl()
    rs, rf = r.get_excl()
    assert np.array_equal(es, rs) and np.array_equal(ef, rf)
    d.free()


def test_link_cell_update_after_motion(gpu):
    s = systems.water_box_for_atoms(18558, seed=4)
    d = DropinSystem(s)
    r = _reference(s)
    d.makelist()
    r.makelist()
    rng = np.random.default_rng(7)
    x, y, z = r.positions()
    # move every atom up to 0.45 A, some of them just outside the box
    x = x + rng.uniform(-0.45, 0.45, len(x))
    y = y + rng.uniform(-0.45, 0.45, len(y))
    z = z + rng.uniform(-0.45, 0.45, len(z))
    d.update(x, y, z)
    r.update_list(x, y, z)
    _compare(d, r)
    d.free()


def test_list_growth_matches_reference(gpu):
    # denser second configuration forces the 1% growth path of the update
    s = systems.water_box_for_atoms(18558, seed=5)
    d = DropinSystem(s)
    r = _reference(s)
    d.makelist()
    r.makelist()
    x, y, z = r.positions()
    f = 0.985
    d.update(x * f, y * f, z * f)
    r.update_list(x * f, y * f, z * f)
    _compare(d, r)
    d.free()


def test_frozen_atoms(gpu):
    s = systems.config_small(seed=2)
    fz = (np.random.default_rng(3).random(s.n) < 0.1).astype(np.int32)
    d = DropinSystem(s, frozen=fz)
    r = _reference(s, frozen=fz)
    d.makelist()
    r.makelist()
    _compare(d, r)
    d.free()


def test_link_cell_96k(gpu):
    s = systems.config_96k(seed=1, temperature=None)
    d = DropinSystem(s)
    r = _reference(s)
    assert d.makelist() == 1 and r.makelist() == 1
    n = _compare(d, r)
    assert n > 50_000_000
    d.free()
