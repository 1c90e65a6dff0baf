"""Batches of independent water boxes in one engine (one launch per stage).

A replica's cluster layout, list and fixed-point sums do not depend on the
other replicas, so the batch's forces equal those of separate engines bit for
bit; the batch is also checked against the plain FP64 form per replica, and
its dynamics (CUDA-graph steps, every replica with its own box) against
separate engines.
"""
import numpy as np
import pytest

from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)
SIZES = [1500, 4203, 2700, 9000, 1998]


@pytest.fixture(scope="module")
def parts():
    return [systems.water_box_for_atoms(n, seed=20 + i, temperature=300.0)
            for i, n in enumerate(SIZES)]


def test_batch_forces_equal_separate_engines(gpu, parts):
    batch = systems.concat(parts)
    e = nb.Engine(batch, precision=1, **POT)
    e.build()
    e.compute()
    fb = e.forces()
    eb = e.energies()
    e.close()
    tot = {k: 0.0 for k in ("elec_direct", "elec_corr", "vdw", "elec_self", "n_pairs")}
    for r, (p, got) in enumerate(zip(parts, nb.Engine.split_arrays(fb, batch))):
        s = nb.Engine(p, precision=1, **POT)
        s.build()
        s.compute()
        fs = s.forces()
        es = s.energies()
        s.close()
        for k in range(3):
            assert np.array_equal(got[k], fs[k]), f"replica {r} component {k}"
        for k in tot:
            tot[k] += es[k]
    for k in tot:
        assert abs(eb[k] - tot[k]) <= 1e-12 * max(1.0, abs(tot[k])), k


def test_batch_per_replica_error_vs_fp64(gpu, parts):
    batch = systems.concat(parts)
    e = nb.Engine(batch, precision=1, **POT)
    e.build()
    tune = e.autotune()
    e.compute()
    fb = e.forces()
    e.close()
    worst = 0.0
    for p, got in zip(parts, nb.Engine.split_arrays(fb, batch)):
        s = nb.Engine(p, precision=0, **POT)
        s.build()
        s.compute()
        ref = s.forces()
        s.close()
        num = sum(((a - b) ** 2).sum() for a, b in zip(got, ref))
        den = sum((b ** 2).sum() for b in ref)
        worst = max(worst, float(np.sqrt(num / den)))
    print(f"batch of {len(parts)}: autotune {tune}; worst replica force rel RMS {worst:.3e}")
    assert worst < 1e-5


def test_batch_dynamics_tracks_separate_engines(gpu, parts):
    batch = systems.concat(parts)
    vel = (batch.vx, batch.vy, batch.vz)
    e = nb.Engine(batch, precision=1, **POT)
    e.md_set_graph(20)
    e.md_init(batch.mass, vel, time_step=0.001, list_update=0,
              constraints=batch.water_constraints())
    rows = e.md_run(60, energy_every=10)
    pos = e.positions()
    st = e.md_stats()
    e.close()
    worst = 0.0
    for p, got in zip(parts, nb.Engine.split_arrays(pos, batch)):
        s = nb.Engine(p, precision=1, **POT)
        s.md_init(p.mass, (p.vx, p.vy, p.vz), time_step=0.001, list_update=0,
                  constraints=p.water_constraints())
        s.md_run(60)
        ref = s.positions()
        s.close()
        for k in range(3):
            d = got[k] - ref[k]
            d -= p.box * np.round(d / p.box)
            worst = max(worst, float(np.max(np.abs(d))))
    print(f"batch dynamics: {st['rebuilds']} rebuilds, worst position difference {worst:.3e} A")
    assert st["molecules"] == sum(SIZES) // 3
    assert worst < 1e-3
    assert np.all(np.isfinite(rows))


def test_batch_rejects_small_box(gpu):
    small = systems.water_box(300, 20.0, seed=1)   # 20 A < 2 * 12 A
    big = systems.water_box_for_atoms(3000, seed=2)
    e = nb.Engine(systems.concat([big, small]), precision=1, **POT)
    with pytest.raises(nb.MdbasNbError):
        e.build()
    e.close()
