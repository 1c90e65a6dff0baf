"""Pin of the numpy SPME restatement (oracle/spme_oracle.py) against MDBas's
own explicit Ewald sum (ewald_rec, src/ewald.c:131-354, compiled in
oracle/_ref): with a fine grid (64^3, order 8) SPME converges to the exact
reciprocal sum, which MDBas gives with m1max = m2max = m3max = 32."""
import numpy as np
import pytest

from mdbas_b200 import systems


@pytest.fixture(scope="module")
def water():
    return systems.water_box(1000, 31.0, seed=2)


def test_spme_grid_rule(oracle_lib, water):
    from oracle import spme_oracle as so
    box = oracle_lib.box(water.cell())
    # init_spme: nint(0.25 + pa alpha tol1 / pi) = 11 -> next power of two 16 -> 32
    assert so.spme_grid(box, 1e-6, 12.0, 0.34) == (32, 32, 32)


def test_spme_restatement_converges_to_mdbas_ewald(ref_available, oracle_lib, water):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    from oracle import spme_oracle as so
    r = oracle.Reference(water, cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
    e, fx, fy, fz, vir, mm, nk = r.ewald_rec(1e-6, (32, 32, 32))
    r.close()
    assert mm == (32, 32, 32) and nk > 70000
    box = oracle_lib.box(water.cell())
    es, sx, sy, sz, svir = so.spme_energy(box, water.x, water.y, water.z, water.q, 0.34,
                                          systems.CHARGE_CONST, (64, 64, 64), 8)
    f = np.stack([fx, fy, fz], 1)
    sf = np.stack([sx, sy, sz], 1)
    assert abs(es - e) <= 1e-9 * abs(e)
    assert abs(svir - vir) <= 1e-6 * abs(vir)
    assert np.sqrt(((f - sf) ** 2).sum() / (f ** 2).sum()) < 1e-7
