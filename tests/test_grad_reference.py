"""The plain-PyTorch FP64 energy of the gradient harness (mdbas_b200.grad.
reference_energy), used as the reference gradient by the adjoint tests, is
pinned here against MDBas's own energy() (oracle/_ref) on CPU."""
import numpy as np
import pytest
import torch

from mdbas_b200 import grad, systems


@pytest.fixture(scope="module")
def fluid():
    return systems.lj_fluid(3000, 33.0, seed=6)


def test_reference_energy_matches_mdbas(ref_available, oracle_lib, fluid):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s = fluid
    r = oracle.Reference(s, cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
    r.makelist()
    _, _, _, e = r.energy()
    e_mdbas = e["elec"] + e["vdw"] + r.self_energy()
    r.close()
    box = oracle_lib.box(s.cell())
    excl = s.exclusions(symmetric=True)
    pairs = oracle_lib.pairs_within(box, s.x, s.y, s.z, excl, 144.0)
    pos = torch.tensor(np.stack([s.x, s.y, s.z], 1))
    e_ref = grad.reference_energy(pos, torch.tensor(s.q), torch.tensor(s.type_eps_kcal),
                                  torch.tensor(s.type_sigma), s.types, pairs, None, s.box)
    assert abs(float(e_ref) - e_mdbas) <= 1e-10 * abs(e_mdbas)


def test_reference_energy_water_exclusions(ref_available, oracle_lib):
    """With exclusions (water): the erf correction term of the reference."""
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    s = systems.water_box(1000, 31.0, seed=2)
    # one LJ type for O, one for H (eps = sigma = 0)
    types = np.tile([0, 1, 1], 1000)
    eps_t = torch.tensor([systems.WATER_EPS_KCAL, 0.0], dtype=torch.float64)
    sig_t = torch.tensor([systems.WATER_SIGMA, 0.0], dtype=torch.float64)
    r = oracle.Reference(s, cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
    r.makelist()
    _, _, _, e = r.energy()
    e_mdbas = e["elec"] + e["vdw"] + r.self_energy()
    r.close()
    box = oracle_lib.box(s.cell())
    start, flat = s.exclusions(symmetric=True)
    pairs = oracle_lib.pairs_within(box, s.x, s.y, s.z, (start, flat), 144.0)
    rows = np.repeat(np.arange(s.n), np.diff(start))
    excl = np.stack([rows, flat], 1)
    excl = excl[excl[:, 1] > excl[:, 0]]
    pos = torch.tensor(np.stack([s.x, s.y, s.z], 1))
    e_ref = grad.reference_energy(pos, torch.tensor(s.q), eps_t, sig_t, types, pairs, excl,
                                  s.box)
    assert abs(float(e_ref) - e_mdbas) <= 1e-10 * abs(e_mdbas)
