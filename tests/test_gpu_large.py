"""The 999,999-atom water box (333,333 molecules, 215 A cube).

The mixed-precision forces are checked against the FP64 oracle restatement
(oracle/mdbas_oracle.c, itself bit-exact with MDBas's ewald_energy on the
pairs it evaluates) on a seeded 10,000-atom subset, and the energies and the
in-cut-off pair count against the plain FP64 GPU form on the whole box.
"""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    return systems.config_1m(seed=1)


def test_large_box_subset_forces_vs_oracle(gpu, oracle_lib, big):
    e = nb.Engine(big, precision=1)
    e.build()
    e.compute()
    fx, fy, fz = e.forces()
    stats = e.list_stats()
    e.close()
    rng = np.random.default_rng(11)
    sub = np.sort(rng.choice(big.n, 10000, replace=False)).astype(np.int32)
    box = oracle_lib.box(big.cell())
    gx, gy, gz = oracle_lib.forces_subset(box, big, big.exclusions(symmetric=True), sub)
    num = ((fx[sub] - gx) ** 2 + (fy[sub] - gy) ** 2 + (fz[sub] - gz) ** 2).sum()
    den = (gx ** 2 + gy ** 2 + gz ** 2).sum()
    rel = float(np.sqrt(num / den))
    print(f"1M box: {stats[1]} cluster pairs; subset force rel RMS {rel:.3e}")
    assert rel < 1e-5


def test_large_box_energy_vs_fp64_form(gpu, big):
    out = {}
    for prec in (1, 0):
        e = nb.Engine(big, precision=prec)
        e.build()
        e.compute()
        out[prec] = e.energies()
        e.close()
    a, b = out[1], out[0]
    ta = a["elec_direct"] + a["elec_corr"] + a["vdw"]
    tb = b["elec_direct"] + b["elec_corr"] + b["vdw"]
    print(f"1M box: pairs {a['n_pairs']:.0f} vs {b['n_pairs']:.0f}; energy rel "
          f"{abs(ta - tb) / abs(tb):.3e}")
    assert abs(ta - tb) / abs(tb) < 1e-6
    assert abs(a["n_pairs"] - b["n_pairs"]) <= 1e-6 * b["n_pairs"]
