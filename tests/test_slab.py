"""Slab decomposition of one box over ranks (mdbas_b200/slab.py), on CPU:
geometry, the local frame's exclusion rows, and whole decomposed
evaluations against the single-domain oracle (FP64, MDBas's expressions) --
one rank (the box exchanging its halo with itself) in-process, two and
three ranks as gloo processes."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch

from mdbas_b200 import slab

import slab_util


def test_geometry():
    g = slab.SlabGeometry((90.0, 50.0, 40.0), 3, 14.0)
    assert g.width == 30.0
    assert [g.lo(r) for r in range(3)] == [-45.0, -15.0, 15.0]
    x = np.array([-45.0, -15.0001, -15.0, 14.999, 15.0, 44.999, 45.0, 100.0, -46.0])
    assert g.owner(x).tolist() == [0, 0, 1, 1, 2, 2, 0, 1, 2]
    assert g.local_lengths() == (30.0 + 28.0 + 1.0, 50.0, 40.0)
    # window [lo, lo + w + r_halo) centred in the local box
    assert g.local_center(1) == -15.0 + 22.0
    with pytest.raises(ValueError):
        slab.SlabGeometry((90.0, 50.0, 40.0), 7, 14.0)   # 12.9 A slabs < 14 A halo
    with pytest.raises(ValueError):
        slab.SlabGeometry((90.0, 50.0, 40.0), 0, 14.0)


def test_partition_covers_every_atom_once():
    s, _ = slab_util.system("water")
    g = slab.SlabGeometry((s.box,) * 3, 3, 14.0)
    parts = slab.partition(g, s.x)
    flat = np.sort(np.concatenate(parts))
    assert np.array_equal(flat, np.arange(s.n))


def test_local_exclusions_pick_the_near_copy():
    # one molecule across the periodic x face, one rank: the partner's halo
    # copy (above the upper face) is the excluded one, not its owned copy
    s, _ = slab_util.system("water")
    L = s.box
    g = slab.SlabGeometry((L,) * 3, 1, 14.0)
    m = 0
    o, h1, h2 = 3 * m, 3 * m + 1, 3 * m + 2
    x = s.x.copy()
    x[o], x[h1], x[h2] = 0.5 * L - 0.3, -0.5 * L + 0.4, 0.5 * L - 1.0
    topo = slab.Topology.of(s)
    owned = np.arange(s.n)
    run = slab.SlabRunner(g, 0, topo, None)
    run.repartition(owned, x, s.y, s.z)
    loc = run.loc
    n_own = loc.n_owned
    halo_of = {int(gi): n_own + k for k, gi in enumerate(loc.gidx[n_own:])}
    assert h1 in halo_of and o not in halo_of
    row_o = loc.excl_flat[loc.excl_start[o]:loc.excl_start[o + 1]].tolist()
    assert sorted(row_o) == sorted([halo_of[h1], h2])
    # the owned copy of h1 keeps no exclusion with o's owned copy
    row_h1 = loc.excl_flat[loc.excl_start[h1]:loc.excl_start[h1 + 1]].tolist()
    assert o not in row_h1
    # rows are symmetric
    n = loc.n
    rows = np.repeat(np.arange(n), np.diff(loc.excl_start))
    pairs = set(zip(rows.tolist(), loc.excl_flat.tolist()))
    assert all((b, a) in pairs for a, b in pairs)
    # no halo-halo exclusions
    assert not any(a >= n_own and b >= n_own for a, b in pairs)


def _compare(s, cell, results):
    rfx, rfy, rfz, re = slab_util.reference(s, cell)
    fx, fy, fz = np.zeros(s.n), np.zeros(s.n), np.zeros(s.n)
    seen = np.zeros(s.n, np.int64)
    for owned, a, b, c, _ in results:
        fx[owned], fy[owned], fz[owned] = a, b, c
        seen[owned] += 1
    assert np.all(seen == 1)
    num = np.sqrt(((fx - rfx) ** 2 + (fy - rfy) ** 2 + (fz - rfz) ** 2).sum())
    den = np.sqrt((rfx ** 2 + rfy ** 2 + rfz ** 2).sum())
    assert num / den < 1e-12, num / den
    e = results[0][4]
    assert int(e["n_pairs"]) == int(re["n_pairs"])
    for k in ("e_dir", "e_corr", "e_vdw", "vir_dir", "vir_corr", "vir_vdw", "e_self"):
        assert abs(e[k] - re[k]) <= 1e-11 * max(abs(re[k]), 1.0), (k, e[k], re[k])


@pytest.mark.parametrize("kind", ["water", "ortho"])
def test_one_rank_self_halo(kind):
    s, cell = slab_util.system(kind)
    res = slab_util.rank_forces(s, cell, 0, 1, slab_util.OracleBackend())
    _compare(s, cell, [res])


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, kind):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        s, cell = slab_util.system(kind)
        res = slab_util.rank_forces(s, cell, rank, world, slab_util.OracleBackend())
        got = [None] * world
        dist.all_gather_object(got, res)
        if rank == 0:
            _compare(s, cell, got)
        # every rank holds the same energies
        assert all(g[4] == res[4] for g in got)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind", [(2, "water"), (3, "water"), (4, "ortho")])
def test_gloo_ranks(world, kind):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), kind), nprocs=world, join=True)


def test_moved_halo_atom_is_refused():
    s, _ = slab_util.system("water")
    g = slab.SlabGeometry((s.box,) * 3, 1, 14.0)
    run = slab.SlabRunner(g, 0, slab.Topology.of(s), slab_util.OracleBackend())
    owned = np.arange(s.n)
    run.repartition(owned, s.x, s.y, s.z)
    run.step(s.x, s.y, s.z)
    # an atom not in the halo moves close to the lower face: the rank below
    # (here the box itself) would miss its pairs, so a repartition is needed
    x = s.x.copy()
    unsent = np.setdiff1d(np.arange(s.n), run.send_idx)
    k = int(unsent[np.argmin(np.abs(x[unsent]))])
    x[k] = g.lo(0) + 1.0
    with pytest.raises(RuntimeError):
        run.step(x, s.y, s.z)
    # with two slabs an atom leaving its slab by more than half the skin too
    g2 = slab.SlabGeometry((s.box,) * 3, 2, 14.0)
    own0 = slab.partition(g2, s.x)[0]
    run2 = slab.SlabRunner(g2, 0, slab.Topology.of(s), slab_util.OracleBackend())
    run2.send_t = torch.zeros(0, dtype=torch.int64)
    x0 = s.x[own0].copy()
    x0[np.argmax(x0)] = g2.lo(1) + 1.5
    with pytest.raises(RuntimeError):
        run2._check_drift(torch.from_numpy(x0))
