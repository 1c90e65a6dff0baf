"""Shared pieces of the slab-decomposition tests: the FP64 CPU restatement
(oracle) as the per-rank evaluator, the single-domain reference, and one
rank's whole evaluation."""
import numpy as np

import oracle
from mdbas_b200 import slab, systems

ORBIC = 2


class OracleBackend:
    """Local evaluation by the oracle's all-pairs list and ewald_energy (FP64,
    MDBas's expressions) in the rank's orthorhombic box, halo atoms frozen."""

    def __init__(self):
        self.o = oracle.Oracle()

    def prepare(self, loc):
        self.loc = loc
        self.box = self.o.box(loc.cell(), box_type=ORBIC)
        self.half = loc.exclusions(symmetric=False)

    def evaluate(self, x, y, z):
        import torch
        o, loc = self.o, self.loc
        x, y, z = (v.cpu().numpy() for v in (x, y, z))
        lst, pair, order = o.verlet_list(self.box, x, y, z, self.half, frozen=loc.frozen,
                                         box_type=ORBIC)
        fx, fy, fz, e = o.ewald_energy(self.box, loc, lst, pair, order, self.half,
                                       box_type=ORBIC, x=x, y=y, z=z)
        return (torch.from_numpy(fx), torch.from_numpy(fy), torch.from_numpy(fz), e)


def reference(s, cell=None):
    """Forces and energies of the whole periodic box in one domain (oracle)."""
    o = oracle.Oracle()
    cell = s.cell() if cell is None else cell
    bt = 1 if cell[4] == cell[0] and cell[8] == cell[0] else ORBIC
    box = o.box(cell, box_type=bt)
    half = s.exclusions(symmetric=False)
    lst, pair, order = o.verlet_list(box, s.x, s.y, s.z, half, box_type=bt)
    fx, fy, fz, e = o.ewald_energy(box, s, lst, pair, order, half, box_type=bt)
    e["e_self"] = o.self_energy(s.q, systems.CHARGE_CONST, 0.34)
    return fx, fy, fz, e


def system(kind: str):
    if kind == "water":
        return systems.water_box_for_atoms(9000, seed=3), None
    # orthorhombic water: a 3,000-molecule cube stretched along x
    s = systems.water_box(2000, 40.0, seed=5)
    s.x = s.x * 1.5
    return s, np.array([60.0, 0, 0, 0, 40.0, 0, 0, 0, 40.0])


def rank_forces(s, cell, rank: int, world: int, backend, device="cpu", moves=1):
    """One rank's owned forces and the box's energies; ``moves`` extra
    evaluations at slightly moved positions (same partition) precede the
    returned one, which is at the original positions."""
    lengths = (cell[0], cell[4], cell[8]) if cell is not None else (s.box,) * 3
    geom = slab.SlabGeometry(lengths, world, 14.0)
    owned = slab.partition(geom, s.x)[rank]
    run = slab.SlabRunner(geom, rank, slab.Topology.of(s), backend, device=device)
    run.repartition(owned, s.x[owned], s.y[owned], s.z[owned])
    rng = np.random.default_rng(rank)
    for _ in range(moves):
        d = rng.uniform(-0.05, 0.05, size=(3, len(owned)))
        run.step(s.x[owned] + d[0], s.y[owned] + d[1], s.z[owned] + d[2])
    fx, fy, fz, e = run.step(s.x[owned], s.y[owned], s.z[owned])
    return owned, fx.cpu().numpy(), fy.cpu().numpy(), fz.cpu().numpy(), e
