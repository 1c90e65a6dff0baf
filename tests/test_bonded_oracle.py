"""The numpy restatement of MDBas's bonded terms (oracle/bonded_oracle.py)
against MDBas's own compiled routines (src/internal.c in oracle/_ref), and
its forces against finite differences of its energies.  CPU only."""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

import bonded_util
from oracle import bonded_oracle as bo

KINDS = list(enumerate(nb.BONDED_KINDS))


@pytest.fixture(scope="module")
def chains():
    # 64 chains in a 26 A box: many cross the periodic boundary
    return systems.flexible_chains(4, 26.0, seed=3, jitter=0.08)


def _oracle_kind(kind, spec, s):
    name = nb.BONDED_KINDS[kind]
    L = (s.box, s.box, s.box)
    t = spec[name]
    if name in ("bonds", "ub"):
        e, v, f = bo.bonds(t, s.x, s.y, s.z, L, ub=name == "ub")
        return e, v, f
    if name == "angles":
        e, f = bo.angles(t, s.x, s.y, s.z, L)
    else:
        e, f = bo.torsions(t, s.x, s.y, s.z, L)
    return e, 0.0, f


@pytest.mark.parametrize("kind,name", KINDS)
def test_restatement_matches_mdbas(ref_available, chains, kind, name):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    spec = chains.meta["bonded"]
    structs = nb.bonded_structs(spec)
    e_ref, v_ref, fx, fy, fz = bonded_util.call(oracle.Reference.lib(), kind, chains, structs)
    e, v, f = _oracle_kind(kind, spec, chains)
    fref = np.stack([fx, fy, fz], 1)
    scale = np.max(np.abs(fref))
    print(f"{name}: E {e_ref:.6e} vs {e:.6e}, max|dF| {np.max(np.abs(f - fref)) / scale:.2e}")
    assert scale > 0 and e_ref != 0.0
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    assert abs(v - v_ref) <= 1e-12 * max(abs(v_ref), 1.0)
    assert np.max(np.abs(f - fref)) <= 1e-12 * scale


@pytest.mark.parametrize("kind,name", KINDS)
def test_restatement_forces_are_gradients(chains, kind, name):
    spec = chains.meta["bonded"]
    e0, _, f = _oracle_kind(kind, spec, chains)
    rng = np.random.default_rng(kind)
    atoms = rng.choice(chains.n, 6, replace=False)
    h = 1e-6
    for a in atoms:
        for axis, arr in enumerate(("x", "y", "z")):
            plus = systems.System(**{**chains.__dict__})
            minus = systems.System(**{**chains.__dict__})
            for s_, sgn in ((plus, 1.0), (minus, -1.0)):
                v = getattr(chains, arr).copy()
                v[a] += sgn * h
                setattr(s_, arr, v)
            ep = _oracle_kind(kind, spec, plus)[0]
            em = _oracle_kind(kind, spec, minus)[0]
            fd = -(ep - em) / (2 * h)
            assert abs(fd - f[a, axis]) <= 1e-5 * (abs(f[a, axis]) + 1e-3 * np.max(np.abs(f)))


def test_restatement_empty_kinds(chains):
    out, f = bo.all_terms({}, chains.x, chains.y, chains.z, (chains.box,) * 3)
    assert all(v == 0.0 for v in out.values())
    assert not f.any()
