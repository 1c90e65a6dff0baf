"""Cut-off electrostatics (MDBas's nonbond_energy: energy() with keyEwald = 0,
coulomb_shift1 / shift2 / switch and vdw_switch or none, src/energy.c:216-345,
src/elec.c:137-263): the C restatement (oracle/mdbas_oracle.c) against MDBas
itself, on MDBas's own list.  Bit for bit: the restatement keeps MDBas's
operation order and is compiled without FP contraction."""
import numpy as np
import pytest

import oracle
from mdbas_b200 import nb, systems

CASES = [(nb.SHIFT1, nb.VSWITCH), (nb.SHIFT2, nb.VSWITCH), (nb.SWITCH, nb.VSWITCH),
         (nb.SHIFT1, nb.NOVDW), (nb.NOELEC, nb.VSWITCH), (nb.FULL, nb.VFULL)]


@pytest.mark.parametrize("elec,vdw", CASES)
def test_restatement_matches_mdbas(oracle_lib, elec, vdw):
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    s = systems.config_small(4)
    r = oracle.Reference(s)
    r.set_nonbond(elec, vdw)
    r.makelist()
    lst, pair, order = r.get_list()
    x, y, z = r.positions()
    rfx, rfy, rfz, re = r.energy()
    r.close()
    s.x, s.y, s.z = x, y, z
    box = oracle_lib.box(s.cell())
    p = oracle_lib.param(vdwSwitch=1 if vdw == nb.VSWITCH else 0, elecType=elec)
    fx, fy, fz, e = oracle_lib.nonbond_energy(box, s, lst, pair, order, p)
    assert np.array_equal(fx, rfx) and np.array_equal(fy, rfy) and np.array_equal(fz, rfz)
    for k in ("elec", "vdw", "virelec", "virvdw"):
        assert e[k] == re[k], k
    if elec in (nb.NOELEC, nb.FULL):
        assert re["elec"] == 0.0      # coulomb_none without Ewald
    else:
        assert re["elec"] != 0.0


def test_rejects_unknown_types():
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    r = oracle.Reference(systems.config_small(1))
    with pytest.raises(ValueError):
        r.set_nonbond(7, nb.VSWITCH)
    r.close()
