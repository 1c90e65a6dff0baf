"""Explicit reciprocal-space Ewald sum on the GPU (mdbas_b200/csrc/ewald_rec.cu)
against MDBas's own init_ewald + ewald_rec (src/ewald.c, compiled into
oracle/_ref).  Same k set (checked through mmax), the same per-(atom, k)
arithmetic; the sums over atoms run in another order, so energies, virials
and stresses agree to 1e-12 relative and forces to 1e-11 of the largest."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

import ewald_util

pytestmark = pytest.mark.gpu

CELLS = [(nb.CUBIC, None), (nb.TCLIN, [31.0, 0.0, 0.0, 1.5, 31.0, 0.0, 1.0, 2.0, 31.0])]


def _ref(s, prec, alpha, mmax, cell, btype, forces=None):
    import oracle
    lib = oracle.Reference.lib()
    ew = ewald_util.init(lib, s, prec, alpha, mmax, cell=cell, box_type=btype)
    out = ewald_util.rec(lib, s, ew, forces, cell=cell, box_type=btype)
    lib.ewald_free(ew)
    return ew, out


def _close(got, ref):
    e, fx, fy, fz, vir, st = got
    re_, rfx, rfy, rfz, rvir, rst = ref
    scale = max(np.max(np.abs(a)) for a in (rfx, rfy, rfz))
    ferr = max(np.max(np.abs(a - b)) for a, b in zip((fx, fy, fz), (rfx, rfy, rfz)))
    serr = max(abs(a - b) for a, b in zip(st, rst)) / max(abs(v) for v in rst)
    print(f"E {e:.12e} vs {re_:.12e}; vir {vir:.6e} vs {rvir:.6e}; "
          f"max|dF| {ferr / scale:.2e}; stress {serr:.2e}")
    assert abs(e - re_) <= 1e-12 * abs(re_)
    assert abs(vir - rvir) <= 1e-12 * abs(rvir)
    assert serr <= 1e-12
    assert ferr <= 1e-11 * scale


@pytest.mark.parametrize("btype,cell", CELLS)
def test_ewald_rec_matches_mdbas(gpu, ref_available, btype, cell):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.config_small(2)
    ew, ref = _ref(s, 1e-6, 0.34, None, cell, btype)
    assert ew.mmax > 1000
    got = nb.ewald_rec(s, 0.34, (ew.m1max, ew.m2max, ew.m3max), cell=cell, box_type=btype)
    _close(got, ref)


def test_ewald_rec_dropin_prototype(gpu, ref_available):
    """The library's ewald_rec (MDBas's prototype) after its own init_ewald,
    on force arrays that already hold values: MDBas multiplies the whole
    arrays by 4 pi C / V after adding the reciprocal forces, and so does the
    drop-in."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.water_box(500, 25.0, seed=6)
    rng = np.random.default_rng(3)
    f0 = [rng.normal(size=s.n) for _ in range(3)]
    ew, ref = _ref(s, 1e-5, None, None, None, nb.CUBIC, f0)
    L = nb.bind_dropin()
    mine_ew = ewald_util.init(L, s, 1e-5, None, None)
    assert (mine_ew.m1max, mine_ew.mmax, mine_ew.alpha) == (ew.m1max, ew.mmax, ew.alpha)
    got = ewald_util.rec(L, s, mine_ew, f0)
    L.ewald_free(mine_ew)
    _close(got, ref)


def test_ewald_rec_large_m_range(gpu, ref_available):
    """m up to 24 per dimension (29k k-vectors on a 1,200-atom box)."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    s = systems.water_box(400, 22.0, seed=8)
    ew, ref = _ref(s, 1e-6, 0.34, (24, 24, 24), None, nb.CUBIC)
    assert ew.mmax > 20000
    got = nb.ewald_rec(s, 0.34, (24, 24, 24))
    _close(got, ref)


def test_ewald_rec_no_k_vectors(gpu):
    """m-range 0: no k-vector, only the self and non-neutral terms of
    src/ewald.c:166-172 and :323 (MDBas's own ewald_rec is not run here: its
    tables hold mmax = 0 rows and it writes rows 0 and 1)."""
    s = systems.water_box(50, 15.0, seed=1)
    s.q = s.q.copy()
    s.q[0] += 0.1  # non-neutral
    e, fx, fy, fz, vir, st = nb.ewald_rec(s, 0.34, (0, 0, 0))
    systq = float(np.sum(s.q))
    eself = -systems.CHARGE_CONST * 0.34 * float(np.sum(s.q * s.q)) / 1.772453850905516
    enn = -(0.5 * np.pi * systems.CHARGE_CONST) * ((systq / 0.34) ** 2 / 15.0 ** 3)
    assert e == pytest.approx(eself + enn, rel=1e-13)
    assert not (fx.any() or fy.any() or fz.any())
