"""Host-side logic that needs no GPU: generators, exclusion CSR, the FP32 erfc
fit, status handling without a device."""
import math

import numpy as np
import pytest

from mdbas_b200 import systems


def test_water_generator_deterministic_and_neutral():
    a = systems.config_small(seed=4)
    b = systems.config_small(seed=4)
    c = systems.config_small(seed=5)
    assert np.array_equal(a.x, b.x) and not np.array_equal(a.x, c.x)
    assert a.n == 3000 and abs(a.q.sum()) < 1e-12
    assert np.all(np.abs(a.x) <= 15.5) and np.all(np.abs(a.z) <= 15.5)
    # rigid geometry: O-H bond lengths (minimum image)
    d = np.stack([a.x[1::3] - a.x[0::3], a.y[1::3] - a.y[0::3], a.z[1::3] - a.z[0::3]], 1)
    d -= 31.0 * np.round(d / 31.0)
    assert np.allclose(np.sqrt((d * d).sum(1)), 0.9572, atol=1e-12)


def test_orthorhombic_water_box():
    L = np.array([25.0, 27.0, 70.0])
    a = systems.water_box_ortho(L, seed=2)
    b = systems.water_box_ortho(L, seed=2)
    assert np.array_equal(a.z, b.z)
    m = a.meta["molecules"]
    # a full lattice at the water density, n_a = round(L_a * density^(1/3))
    nl = np.rint(L * systems.WATER_DENSITY ** (1.0 / 3.0)).astype(int)
    assert m == int(np.prod(nl)) and a.n == 3 * m and abs(a.q.sum()) < 1e-9
    assert np.array_equal(a.cell(), [25.0, 0, 0, 0, 27.0, 0, 0, 0, 70.0])
    for v, edge in ((a.x, L[0]), (a.y, L[1]), (a.z, L[2])):
        assert np.all(np.abs(v) <= 0.5 * edge)
    # rigid geometry under the minimum image of each axis
    for h in (1, 2):
        d = np.stack([a.x[h::3] - a.x[0::3], a.y[h::3] - a.y[0::3], a.z[h::3] - a.z[0::3]], 1)
        d -= L * np.round(d / L)
        assert np.allclose(np.sqrt((d * d).sum(1)), 0.9572, atol=1e-12)
    assert len(a.bonds) == 2 * m and len(a.angles) == m


def test_96k_box_density_and_velocities():
    s = systems.config_96k(seed=1)
    assert s.n == 96000 and s.box == 98.6
    ke = 0.5 * (s.mass * (s.vx ** 2 + s.vy ** 2 + s.vz ** 2)).sum()
    temp = 2 * ke / (3 * s.n * systems.RBOLTZ_IU)
    assert abs(temp - 300.0) < 5.0


def test_lj_fluid_min_separation():
    s = systems.lj_fluid(3000, 31.0, seed=3)
    from scipy.spatial import cKDTree
    pos = np.stack([s.x, s.y, s.z], 1) + 15.5
    pos = np.mod(pos, 31.0)
    assert len(cKDTree(pos, boxsize=31.0).query_pairs(1.9999)) == 0
    assert abs(s.q.sum()) < 1e-10
    assert len(set(s.types.tolist())) == 4
    assert np.allclose(s.eps, np.sqrt(s.type_eps_kcal[s.types] * 418.4))


def test_replica_sizes():
    sz = systems.replica_sizes(64, seed=1)
    assert len(sz) == 64 and all(1500 <= v <= 30000 and v % 3 == 0 for v in sz)


def test_exclusion_csr_forms():
    s = systems.config_small(seed=1)
    st, fl = s.exclusions(symmetric=True)
    assert st[-1] == 6 * 1000
    sth, flh = s.exclusions(symmetric=False)
    assert sth[-1] == 3 * 1000
    for i in range(0, 30):
        row = flh[sth[i]:sth[i + 1]]
        assert all(j > i for j in row)


def test_fp32_erfc_fit_accuracy():
    """The pair kernel's erfc = t P(t) exp(-x^2) evaluated in FP32 (Horner,
    coefficients rounded to FP32) stays within 6e-7 relative of erfc on the
    range the 12 A cut-off reaches (alpha r <= 4.08)."""
    from scipy.special import erfc
    p = np.float32(3.225531683e-01)
    c = [np.float32(v) for v in (1.826605733e-01, 1.717395874e-01, 2.389294945e-01,
                                 -8.776152576e-02, 6.608865734e-01, -6.320509922e-01,
                                 6.305108379e-01, -1.649145727e-01)]
    x = np.linspace(0, 4.2, 100001).astype(np.float32)
    t = (np.float32(1) / (np.float32(1) + p * x)).astype(np.float32)
    poly = c[7]
    for k in range(6, -1, -1):
        poly = (poly * t + c[k]).astype(np.float32)
    approx = (t * poly * np.exp(-(x.astype(np.float64) ** 2)).astype(np.float32))
    rel = np.abs(approx.astype(np.float64) - erfc(x.astype(np.float64))) / erfc(x)
    assert rel.max() < 6e-7


def test_fit_script_constants_match_kernel():
    import os
    import re
    src = open(os.path.join(os.path.dirname(systems.__file__), "csrc", "pair_fp32.cu")).read()
    consts = dict(re.findall(r"constexpr float kErfc(\w+) = ([-0-9.e+]+)f;", src))
    assert float(consts["P"]) == pytest.approx(0.3225531683, rel=1e-9)
    assert len(consts) == 9


def test_engine_without_device_reports(nb_lib):
    from conftest import has_gpu
    from mdbas_b200 import nb
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(nb.MdbasNbError) as ei:
        nb.Engine(systems.config_small(1), precision=1)
    assert ei.value.status == 3


def test_make_param_derived_terms():
    from mdbas_b200 import nb
    p = nb.make_param(10, cutOff=12.0, cutOn=10.0)
    assert p.cutOff2 == 144.0 and p.cutOn2 == 100.0
    assert p.switch2 == 1.0 / (44.0 * 44.0 * 44.0)
    assert math.isclose(p.chargeConst, 332.0716 * 418.4)


def test_concat_batch_layout():
    from mdbas_b200 import systems
    a = systems.water_box_for_atoms(1500, seed=1, temperature=300.0)
    b = systems.water_box_for_atoms(2100, seed=2, temperature=300.0)
    c = systems.concat([a, b])
    assert c.n == a.n + b.n
    assert c.meta["offsets"] == [0, a.n, a.n + b.n]
    assert [n for _, n in c.meta["replicas"]] == [a.n, b.n]
    assert np.array_equal(c.x[a.n:], b.x)
    # bonds renumbered into the second replica's range
    assert c.bonds.min() == 0 and c.bonds[len(a.bonds):].min() == a.n
    start, flat = c.exclusions(symmetric=True)
    sa, fa = a.exclusions(symmetric=True)
    assert np.array_equal(start[:a.n + 1], sa)
    assert np.array_equal(flat[:len(fa)], fa)
    pairs, len2 = c.water_constraints()
    assert len(pairs) == c.n and pairs.max() == c.n - 1
    sizes = systems.replica_sizes(64, seed=1)
    assert len(sizes) == 64 and all(s % 3 == 0 and 1500 <= s <= 30000 for s in sizes)
