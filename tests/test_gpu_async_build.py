"""The engine's rebuilds of an unchanged grid run without waiting for the
list counts (precision 1): errors surface at the next call that returns
results.  A rebuild whose list no longer fits is built again with room and
the evaluation redone, so the caller sees the same forces as a fresh engine;
non-finite positions report MDBAS_NB_ERR_NONFINITE."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu


def _squeezed(s, factor):
    """The same atoms pulled towards the box centre (more pairs per atom)."""
    t = systems.System(**{**s.__dict__})
    t.x, t.y, t.z = s.x * factor, s.y * factor, s.z * factor
    return t


def test_overflowing_rebuild_matches_fresh_engine(gpu):
    s = systems.lj_fluid(8000, 50.0, seed=11, min_sep=2.0)
    # soft, weakly charged particles, so that the packed state below keeps
    # its forces far inside the fixed-point range
    s.eps = s.eps * 1e-2
    s.sig = s.sig * 0.3
    s.q = s.q * 0.1
    dense = _squeezed(s, 0.25)           # 64x the density: past the list's room
    e = nb.Engine(s, precision=1)
    e.build()
    e.compute()
    cap0 = e.list_stats()[3]
    e.set_positions(dense.x, dense.y, dense.z)
    e.build()                            # same grid: no wait for the counts
    e.compute()
    f = e.forces()                       # settles the build: rebuilt with room
    en = e.energies()
    stats = e.list_stats()
    assert stats[1] > cap0 and stats[3] > cap0   # the list outgrew its room and grew
    ref = nb.Engine(dense, precision=1)
    ref.build()
    ref.compute()
    rf = ref.forces()
    ren = ref.energies()
    for k in range(3):
        assert np.array_equal(f[k], rf[k])
    assert en == ren
    # and again without overflow: the grown list is reused
    e.build()
    e.compute()
    f2 = e.forces()
    for k in range(3):
        assert np.array_equal(f2[k], rf[k])
    e.close()
    ref.close()


def test_nonfinite_position_reported(gpu):
    s = systems.water_box(1000, 31.0, seed=2)
    e = nb.Engine(s, precision=1)
    e.build()
    e.compute()
    x = s.x.copy()
    x[17] = np.nan
    e.set_positions(x, s.y, s.z)
    e.build()
    e.compute()
    with pytest.raises(nb.MdbasNbError) as err:
        e.energies()
    assert err.value.status == 11    # MDBAS_NB_ERR_NONFINITE
    # finite positions again: the engine recovers
    e.set_positions(s.x, s.y, s.z)
    e.build()
    e.compute()
    e.energies()
    e.close()
