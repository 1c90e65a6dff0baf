"""init_ewald of the library (MDBas's prototype, host code) against MDBas's
own (src/ewald.c:10-99, compiled in oracle/_ref): tolerances, alpha, the
m-range and the k-vector count, bit for bit, for cubic, orthorhombic and
triclinic boxes, with and without the alpha / m-range keywords.  CPU only."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

import ewald_util

CELLS = [(nb.CUBIC, [31.0, 0, 0, 0, 31.0, 0, 0, 0, 31.0]),
         (nb.ORBIC, [40.0, 0, 0, 0, 35.5, 0, 0, 0, 33.25]),
         (nb.TCLIN, [31.0, 0.0, 0.0, 1.5, 31.0, 0.0, 1.0, 2.0, 31.0])]


@pytest.mark.parametrize("btype,cell", CELLS)
@pytest.mark.parametrize("alpha,mmax,prec", [(None, None, 1e-6), (0.34, None, 1e-5),
                                             (0.30, (5, 6, 7), 1e-6)])
def test_init_ewald_matches_mdbas(ref_available, btype, cell, alpha, mmax, prec):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s = systems.water_box(200, 31.0, seed=4)
    ref = ewald_util.init(oracle.Reference.lib(), s, prec, alpha, mmax, cell=cell,
                          box_type=btype)
    mine = ewald_util.init(nb.bind_dropin(), s, prec, alpha, mmax, cell=cell, box_type=btype)
    fields = ["prec", "tol", "alpha", "tol1", "m1max", "m2max", "m3max", "mmax"]
    got = [getattr(mine, f) for f in fields]
    want = [getattr(ref, f) for f in fields]
    oracle.Reference.lib().ewald_free(ref)
    print(dict(zip(fields, want)))
    assert got == want
    assert ref.mmax > 0
