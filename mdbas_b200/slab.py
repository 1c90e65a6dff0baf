"""Spatial decomposition of one periodic box into slabs along x, one slab per
rank (one process per GPU), for the real-space nonbonded forces.

MDBas itself has no working domain decomposition (src/parallel.c holds an
MPI stub that nothing calls); this module splits the force evaluation of one
large box over ranks so that each GPU holds a slab of it.

Scheme (half shell, one exchange step each way):

* Rank r owns the atoms whose wrapped x lies in [lo_r, lo_r + w), w = Lx /
  world.  Every rank keeps the whole topology (charges, LJ parameters,
  exclusion rows by global atom index); only positions travel.
* Forward exchange: rank r sends to rank r - 1 (periodically) the owned atoms
  within ``r_halo`` of its lower face, with their global indices; rank r - 1
  places them above its upper face (adding Lx when the sender is rank 0 and
  the receiver the last rank, or with one rank, when the box sends to itself).
* Each rank evaluates, in its own orthorhombic box ``Lx_loc = w + 2 r_halo +
  1`` by Ly by Lz (no periodic image within reach along x), every pair with
  at least one owned atom: halo atoms are marked frozen, so halo-halo pairs
  drop out as MDBas drops pairs of two frozen atoms (src/list.c:2057-2075),
  and only excluded pairs with an owned atom are corrected.
* Reverse exchange: the forces on halo atoms go back to their owner (rank
  r + 1), which adds them to its own.

Every pair within the cut-off (minimum image) is evaluated by exactly one
rank, the owner of the atom lying lower along x in the pair's minimum-image
placement: with ``w >= r_halo`` the other atom lies in the same slab or in
that rank's halo, and no other rank holds the pair with an owned lower atom.
Excluded pairs follow the same rule (the local copy of a partner is the one
within ``r_halo``), so the exclusion correction of each excluded pair is
also added once.  The self term is summed over owned charges only.

Positions between two repartitions: ``SlabRunner.repartition`` fixes the
owned and halo atoms (as MDBas fixes its list at a rebuild); ``step`` then
moves the same atoms' positions through the exchange every evaluation.
Repartition at every list rebuild, with ``r_halo = cutOff + delr`` as the
list radius, so that atoms moving less than half the skin stay covered.

Communication uses torch.distributed point-to-point operations on tensors
of ``device`` (CUDA tensors over NCCL on GPUs, CPU tensors over gloo in
tests).  No TMA or bulk copy ever reads a peer's memory: halo data land in
this rank's own buffers before any kernel reads them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

ENERGY_KEYS = ("e_dir", "e_corr", "e_vdw", "vir_dir", "vir_corr", "vir_vdw", "n_pairs")


@dataclass
class SlabGeometry:
    """Slabs of an orthorhombic (or cubic) box along x."""

    lengths: tuple  # (Lx, Ly, Lz)
    world: int
    r_halo: float

    def __post_init__(self):
        self.lengths = tuple(float(v) for v in self.lengths)
        if self.world < 1:
            raise ValueError("world must be >= 1")
        if self.width < self.r_halo:
            raise ValueError(f"slab width {self.width:.3f} A is below the halo width "
                             f"{self.r_halo:.3f} A: at most {int(self.lengths[0] // self.r_halo)}"
                             " ranks for this box")

    @property
    def width(self) -> float:
        return self.lengths[0] / self.world

    def lo(self, rank: int) -> float:
        """Lower face of rank's slab (the box spans [-Lx/2, Lx/2))."""
        return -0.5 * self.lengths[0] + rank * self.width

    def wrap(self, v: np.ndarray, axis: int) -> np.ndarray:
        """Coordinates along axis wrapped into [-L/2, L/2)."""
        L = self.lengths[axis]
        s = (np.asarray(v, dtype=np.float64) + 0.5 * L) / L
        return (s - np.floor(s)) * L - 0.5 * L

    def owner(self, x: np.ndarray) -> np.ndarray:
        """Rank owning each atom, from its x coordinate."""
        xw = self.wrap(x, 0)
        r = np.floor((xw + 0.5 * self.lengths[0]) / self.width).astype(np.int64)
        return np.clip(r, 0, self.world - 1)

    def local_lengths(self) -> tuple:
        """The local box: owned slab + halo + r_halo + 1 A along x, so that no
        periodic image along x lies within r_halo of any local atom."""
        return (self.width + 2.0 * self.r_halo + 1.0, self.lengths[1], self.lengths[2])

    def local_center(self, rank: int) -> float:
        """x of the local box's centre in the global frame (the window
        [lo, lo + w + r_halo) is centred in the local box)."""
        return self.lo(rank) + 0.5 * (self.width + self.r_halo)


def partition(geom: SlabGeometry, x: np.ndarray) -> list:
    """Global indices owned by each rank (ascending)."""
    own = geom.owner(x)
    return [np.nonzero(own == r)[0] for r in range(geom.world)]


@dataclass
class LocalSystem:
    """One rank's owned + halo atoms in its local frame (owned first)."""

    gidx: np.ndarray          # global index of each local atom
    n_owned: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    q: np.ndarray
    eps: np.ndarray
    sig: np.ndarray
    frozen: np.ndarray        # 1 on halo atoms
    excl_start: np.ndarray    # symmetric exclusion rows over local indices
    excl_flat: np.ndarray
    lengths: tuple            # local orthorhombic box

    @property
    def n(self) -> int:
        return int(self.gidx.shape[0])

    @property
    def meta(self) -> dict:
        return {}

    def cell(self) -> np.ndarray:
        Lx, Ly, Lz = self.lengths
        return np.array([Lx, 0, 0, 0, Ly, 0, 0, 0, Lz], dtype=np.float64)

    def exclusions(self, symmetric: bool = True):
        """(start, flat) rows: symmetric, or half rows (j > i) as MDBas's
        all-pairs builder keeps them."""
        if symmetric:
            return self.excl_start, self.excl_flat
        n = self.n
        rows = np.repeat(np.arange(n), np.diff(self.excl_start))
        keep = self.excl_flat > rows
        counts = np.bincount(rows[keep], minlength=n)
        start = np.zeros(n + 1, np.int32)
        start[1:] = np.cumsum(counts)
        return start, self.excl_flat[keep].astype(np.int32)


class Topology:
    """Per-atom parameters and exclusion rows by global index (every rank
    holds all of it: it does not change during a run)."""

    def __init__(self, q, eps, sig, excl_start, excl_flat):
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.eps = np.ascontiguousarray(eps, dtype=np.float64)
        self.sig = np.ascontiguousarray(sig, dtype=np.float64)
        self.excl_start = np.ascontiguousarray(excl_start, dtype=np.int64)
        self.excl_flat = np.ascontiguousarray(excl_flat, dtype=np.int64)

    @classmethod
    def of(cls, system, exclusions=None):
        start, flat = system.exclusions(symmetric=True) if exclusions is None else exclusions
        return cls(system.q, system.eps, system.sig, start, flat)

    @property
    def n(self) -> int:
        return int(self.q.shape[0])


def local_system(geom: SlabGeometry, rank: int, topo: Topology, owned: np.ndarray,
                 ox, oy, oz, halo: np.ndarray, hx, hy, hz) -> LocalSystem:
    """The local frame of one rank: owned atoms (global indices ``owned`` at
    wrapped positions) then halo atoms (placed above the upper face), x
    shifted by the local box centre, y and z wrapped.  Exclusion rows keep,
    for each owned atom and each partner, the partner's local copy within
    r_halo (none when the partner lies below the slab: the rank below holds
    that pair), mirrored so the rows are symmetric."""
    n_own, n_halo = len(owned), len(halo)
    gidx = np.concatenate([owned, halo]).astype(np.int64)
    c = geom.local_center(rank)
    x = np.concatenate([geom.wrap(ox, 0), np.asarray(hx, np.float64)]) - c
    y = geom.wrap(np.concatenate([oy, hy]), 1)
    z = geom.wrap(np.concatenate([oz, hz]), 2)
    n = n_own + n_halo
    frozen = np.zeros(n, np.int32)
    frozen[n_own:] = 1

    # local copies of every global atom: owned index, halo index (-1: none)
    own_map = np.full(topo.n, -1, np.int64)
    own_map[owned] = np.arange(n_own)
    halo_map = np.full(topo.n, -1, np.int64)
    halo_map[halo] = n_own + np.arange(n_halo)
    s0, s1 = topo.excl_start[owned], topo.excl_start[owned + 1]
    cnt = s1 - s0
    a = np.repeat(np.arange(n_own), cnt)
    if len(a):
        off = np.arange(len(a)) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        partner = topo.excl_flat[np.repeat(s0, cnt) + off]
    else:
        partner = np.zeros(0, np.int64)
    Ly, Lz = geom.lengths[1], geom.lengths[2]

    def near(i, j):
        ok = j >= 0
        jj = np.where(ok, j, 0)
        dx = x[jj] - x[i]
        dy = y[jj] - y[i]
        dy -= Ly * np.rint(dy / Ly)
        dz = z[jj] - z[i]
        dz -= Lz * np.rint(dz / Lz)
        return ok & (dx * dx + dy * dy + dz * dz < geom.r_halo * geom.r_halo)

    co, ch = own_map[partner], halo_map[partner]
    use_o, use_h = near(a, co), near(a, ch)
    if np.any(use_o & use_h):
        raise ValueError("an excluded pair has two local copies within the halo width")
    rows_a = np.concatenate([a[use_o], a[use_h]])
    rows_b = np.concatenate([co[use_o], ch[use_h]])
    # symmetric: both directions, each pair once per direction
    ii = np.concatenate([rows_a, rows_b])
    jj = np.concatenate([rows_b, rows_a])
    key = np.unique(ii * n + jj)
    ii, jj = key // n, key % n
    start = np.zeros(n + 1, np.int32)
    start[1:] = np.cumsum(np.bincount(ii, minlength=n))
    return LocalSystem(gidx=gidx, n_owned=n_own, x=x, y=y, z=z, q=topo.q[gidx],
                       eps=topo.eps[gidx], sig=topo.sig[gidx], frozen=frozen,
                       excl_start=start, excl_flat=jj.astype(np.int32),
                       lengths=geom.local_lengths())


class Exchange:
    """Point-to-point exchanges between a rank and its two slab neighbours:
    forward to rank - 1 / from rank + 1, reverse to rank + 1 / from rank - 1,
    on torch tensors of the runner's device.  With one rank both neighbours
    are the rank itself and nothing is sent."""

    def __init__(self, rank: int, world: int, device="cpu"):
        self.rank, self.world, self.device = rank, world, device
        self.prev = (rank - 1) % world
        self.next = (rank + 1) % world

    def _swap(self, send, to: int, frm: int, recv_shape, dtype):
        import torch
        import torch.distributed as dist
        buf = torch.empty(recv_shape, dtype=dtype, device=self.device)
        ops = [dist.P2POp(dist.isend, send.contiguous(), to), dist.P2POp(dist.irecv, buf, frm)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        return buf

    def count(self, k: int) -> int:
        """Send this rank's row count to rank - 1; return rank + 1's."""
        if self.world == 1:
            return k
        import torch
        t = torch.tensor([k], dtype=torch.int64, device=self.device)
        return int(self._swap(t, self.prev, self.next, (1,), torch.int64).item())

    def forward(self, rows, k_in: int):
        """Send (k, m) float64 rows to rank - 1; return the (k_in, m) rows
        rank + 1 sent."""
        if self.world == 1:
            return rows
        import torch
        return self._swap(rows, self.prev, self.next, (k_in, rows.shape[1]), torch.float64)

    def reverse(self, rows, n_back: int):
        """Send (k, m) float64 rows to rank + 1 (the owner of this rank's halo
        atoms); return the (n_back, m) rows rank - 1 sent back for the atoms
        this rank forwarded to it."""
        if self.world == 1:
            return rows
        import torch
        return self._swap(rows, self.next, self.prev, (n_back, rows.shape[1]), torch.float64)


class EngineBackend:
    """Local evaluation on this rank's GPU through the engine (nb.Engine:
    mixed precision 1 or the plain FP64 form 0), positions and forces as
    device pointers of CUDA tensors, on the current torch stream.  The engine
    is made for a local system at repartition and kept while the local atoms
    stay the same."""

    def __init__(self, precision: int = 1, device: int = 0, **engine_kw):
        self.precision, self.device, self.kw = precision, device, engine_kw
        self.eng = None
        self._key = None

    def prepare(self, loc: LocalSystem):
        import torch

        from . import nb
        key = (loc.n, loc.n_owned, loc.gidx.tobytes())
        if self.eng is None or key != self._key:
            if self.eng is not None:
                self.eng.close()
            self.eng = nb.Engine(loc, precision=self.precision, device=self.device,
                                 frozen=loc.frozen, box_type=nb.ORBIC, cell=loc.cell(),
                                 exclusions=(loc.excl_start, loc.excl_flat), **self.kw)
            self.eng.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
            self._key = key
            self.f = torch.empty((3, loc.n), dtype=torch.float64, device=f"cuda:{self.device}")

    def evaluate(self, x, y, z):
        e = self.eng
        e.set_positions_device(x.data_ptr(), y.data_ptr(), z.data_ptr())
        e.build()
        e.compute()
        f = self.f
        e.forces_device(f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
        en = e.energies()
        return f[0], f[1], f[2], {"e_dir": en["elec_direct"], "e_corr": en["elec_corr"],
                                  "e_vdw": en["vdw"], "vir_dir": en["vir_direct"],
                                  "vir_corr": en["vir_corr"], "vir_vdw": en["vir_vdw"],
                                  "n_pairs": en["n_pairs"]}

    def close(self):
        if self.eng is not None:
            self.eng.close()
            self.eng = None


class SlabRunner:
    """One rank's part of the decomposed force evaluation.

    ``repartition(owned, x, y, z)`` takes this rank's owned atoms (global
    indices and FP64 positions), exchanges the halo atoms and prepares the
    local system (host work, once per list rebuild); ``step(x, y, z)``
    evaluates at new positions of the same owned atoms: forward exchange of
    the halo positions, local evaluation, reverse exchange of the halo
    forces -- torch tensors on ``device`` throughout (CUDA tensors and the
    engine's device-pointer calls on GPUs).  Returns the owned atoms'
    forces (tensors, in the order of ``owned``) and the whole box's
    energies (identical on every rank)."""

    def __init__(self, geom: SlabGeometry, rank: int, topo: Topology, backend,
                 device="cpu", alpha: float = 0.34, charge_const: float | None = None,
                 r_cut: float = 12.0):
        from .systems import CHARGE_CONST
        if not 0.0 < r_cut <= geom.r_halo:
            raise ValueError("the cut-off must lie within the halo width")
        self.geom, self.rank, self.topo, self.backend = geom, rank, topo, backend
        # half the skin: how far atoms may move between two repartitions
        self.drift = 0.5 * (geom.r_halo - r_cut)
        self.ex = Exchange(rank, geom.world, device)
        self.device = device
        self.self_coef = -(CHARGE_CONST if charge_const is None else charge_const) * alpha \
            / math.sqrt(math.pi)
        self.owned = None

    def _t(self, a):
        import torch
        return torch.as_tensor(a, dtype=torch.float64, device=self.device)

    def _wrap_t(self, v, axis: int):
        import torch
        L = self.geom.lengths[axis]
        s = (v + 0.5 * L) / L
        return (s - torch.floor(s)) * L - 0.5 * L

    def _send_rows(self, x, y, z):
        import torch
        xw = self._wrap_t(x.index_select(0, self.send_t), 0)
        if self.rank == 0:
            xw = xw + self.geom.lengths[0]   # above the last rank's upper face
        return torch.stack([xw, y.index_select(0, self.send_t), z.index_select(0, self.send_t)], 1)

    def repartition(self, owned: np.ndarray, x, y, z):
        import torch
        self.owned = np.asarray(owned, dtype=np.int64)
        xh, yh, zh = (np.asarray(v.cpu() if hasattr(v, "cpu") else v, dtype=np.float64)
                      for v in (x, y, z))
        xw = self.geom.wrap(xh, 0)
        self.send_idx = np.nonzero(xw - self.geom.lo(self.rank) < self.geom.r_halo)[0]
        self.send_t = torch.as_tensor(self.send_idx, dtype=torch.int64, device=self.device)
        # halo membership: global indices travel once per repartition
        k_in = self.ex.count(len(self.send_idx))
        gid = self._t(self.owned[self.send_idx].astype(np.float64)).reshape(-1, 1)
        got = torch.cat([gid, self._send_rows(self._t(xh), self._t(yh), self._t(zh))], 1)
        got = self.ex.forward(got, k_in).cpu().numpy()
        self.halo = got[:, 0].astype(np.int64)
        self.loc = local_system(self.geom, self.rank, self.topo, self.owned, xh, yh, zh,
                                self.halo, got[:, 1], got[:, 2], got[:, 3])
        self.n_halo = len(self.halo)
        qo = self.topo.q[self.owned]
        self.e_self = self.self_coef * float(np.dot(qo, qo))
        if hasattr(self.backend, "prepare"):
            self.backend.prepare(self.loc)

    def _check_drift(self, x):
        # owned atoms still within half the skin of the slab, and atoms not in
        # the halo sent below still beyond the cut-off plus half the skin from
        # the lower face; otherwise the partition no longer covers every pair
        import torch
        rel = self._wrap_t(x, 0) - self.geom.lo(self.rank)
        w, h = self.geom.width, self.drift
        bad = torch.zeros_like(rel, dtype=torch.bool)
        if self.geom.world > 1:
            bad |= (rel < -h) | (rel >= w + h)
        near = rel < self.geom.r_halo - h
        near[self.send_t] = False
        if bool((bad | near).any()):
            raise RuntimeError("atoms moved more than half the skin since the last "
                               "repartition: repartition first")

    def step(self, x, y, z):
        import torch
        x, y, z = self._t(x), self._t(y), self._t(z)
        self._check_drift(x)
        got = self.ex.forward(self._send_rows(x, y, z), self.n_halo)
        c = self.geom.local_center(self.rank)
        lx = (torch.cat([self._wrap_t(x, 0), got[:, 0]]) - c).contiguous()
        ly = self._wrap_t(torch.cat([y, got[:, 1]]), 1).contiguous()
        lz = self._wrap_t(torch.cat([z, got[:, 2]]), 2).contiguous()
        fx, fy, fz, en = self.backend.evaluate(lx, ly, lz)
        no = self.loc.n_owned
        back = self.ex.reverse(torch.stack([fx[no:], fy[no:], fz[no:]], 1), len(self.send_idx))
        ofx, ofy, ofz = fx[:no].clone(), fy[:no].clone(), fz[:no].clone()
        ofx.index_add_(0, self.send_t, back[:, 0])
        ofy.index_add_(0, self.send_t, back[:, 1])
        ofz.index_add_(0, self.send_t, back[:, 2])
        vals = [float(en[k]) for k in ENERGY_KEYS] + [self.e_self]
        tot = _sum_over_ranks(vals, self.device)
        out = dict(zip(ENERGY_KEYS, tot[:len(ENERGY_KEYS)]))
        out["e_self"] = tot[-1]
        return ofx, ofy, ofz, out


def _sum_over_ranks(values, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu().tolist()]
