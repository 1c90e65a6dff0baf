"""Gradient harness: the real-space energy and forces as a differentiable
function of positions, per-atom charges and per-type LJ parameters.

``RealSpaceModel(system, types)`` wraps an FP64-form engine.  ``model(pos, q,
eps_t, sig_t)`` returns (E, F) through ``RealSpaceFunction``, a
``torch.autograd.Function`` whose backward is one call of the hand-written
adjoint kernel (``mdbas_nb_engine_adjoint``): for upstream gradients (gE, gF)
it returns

    dL/dpos = -gE F + d(gF.F)/dpos          (d(gF.F)/dpos = -H gF)
    dL/dq   =  gE dE/dq + d(gF.F)/dq
    dL/deps_t, dL/dsig_t likewise, reduced from the per-atom eps_i, sig_i
    through eps_i = sqrt(418.4 eps_t) and sig_i = sig_t / 2 (MDBas's FORF
    convention, src/io.c:1174-1175).

Units: positions in A, charges in e, eps_t in kcal/mol, sig_t in A (the LJ
sigma), energies in MDBas internal units (10 J/mol), forces in those per A.

``reference_energy`` restates the same energy in plain PyTorch FP64 on an
explicit pair list, for the gradient checks (autograd through it gives the
FP64 reference gradient).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import nb
from .systems import CHARGE_CONST, KCAL_TO_IU

POTENTIAL = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)


class RealSpaceModel:
    """One system (fixed topology and box) evaluated on the GPU's FP64 form."""

    def __init__(self, system, types, device: int = 0, **pot):
        self.pot = dict(POTENTIAL, **pot)
        self.system = system
        self.types = np.asarray(types, dtype=np.int64)
        self.n_types = int(self.types.max()) + 1
        self.engine = nb.Engine(system, precision=0, device=device, **self.pot)
        self.n = system.n

    def per_atom(self, eps_t: np.ndarray, sig_t: np.ndarray):
        return (np.sqrt(np.asarray(eps_t)[self.types] * KCAL_TO_IU),
                0.5 * np.asarray(sig_t)[self.types])

    def evaluate(self, pos: np.ndarray, q: np.ndarray, eps_t: np.ndarray, sig_t: np.ndarray):
        """Set parameters and positions, rebuild the list, compute: (E, F[n, 3])."""
        eps_i, sig_i = self.per_atom(eps_t, sig_t)
        self.engine.set_parameters(q, eps_i, sig_i)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.engine.set_positions(pos[:, 0], pos[:, 1], pos[:, 2])
        self.engine.build()
        self.engine.compute()
        e = self.engine.energies()
        energy = e["elec_direct"] + e["elec_corr"] + e["elec_self"] + e["vdw"]
        f = np.stack(self.engine.forces(), axis=1)
        return energy, f

    def type_sum(self, per_atom: np.ndarray) -> np.ndarray:
        return np.bincount(self.types, weights=per_atom, minlength=self.n_types)

    def __call__(self, pos, q, eps_t, sig_t):
        return RealSpaceFunction.apply(pos, q, eps_t, sig_t, self)


class RealSpaceFunction(torch.autograd.Function):
    """(pos [n,3], q [n], eps_t [T], sig_t [T], model) -> (E, F [n,3]), FP64."""

    @staticmethod
    def forward(ctx, pos, q, eps_t, sig_t, model):
        args = [t.detach().cpu().numpy().astype(np.float64) for t in (pos, q, eps_t, sig_t)]
        energy, f = model.evaluate(*args)
        ctx.model = model
        ctx.args = args
        ctx.forces = f
        dev = pos.device
        return (torch.tensor(energy, dtype=torch.float64, device=dev),
                torch.from_numpy(f).to(dev))

    @staticmethod
    def backward(ctx, gE, gF):
        model = ctx.model
        pos, q, eps_t, sig_t = ctx.args
        # the engine may have served other calls since the forward
        model.evaluate(pos, q, eps_t, sig_t)
        ge = 0.0 if gE is None else float(gE)
        v = None if gF is None else gF.detach().cpu().numpy().astype(np.float64)
        adj = model.engine.adjoint(None if v is None else (v[:, 0], v[:, 1], v[:, 2]))
        dpos = -ge * ctx.forces
        dq = ge * adj["gq"]
        deps_i = ge * adj["geps"]
        dsig_i = ge * adj["gsig"]
        if v is not None:
            dpos = dpos + np.stack([adj["hx"], adj["hy"], adj["hz"]], axis=1)
            dq = dq + adj["pq"]
            deps_i = deps_i + adj["peps"]
            dsig_i = dsig_i + adj["psig"]
        eps_i, _ = model.per_atom(eps_t, sig_t)
        with np.errstate(divide="ignore", invalid="ignore"):
            chain = np.where(eps_i > 0, KCAL_TO_IU / (2.0 * eps_i), 0.0)
        deps_t = model.type_sum(deps_i * chain)
        dsig_t = model.type_sum(0.5 * dsig_i)
        dev = gF.device if gF is not None else gE.device
        out = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
               for a in (dpos, dq, deps_t, dsig_t)]
        return out[0], out[1], out[2], out[3], None


def reference_energy(pos, q, eps_t, sig_t, types, pairs, excl_pairs, box, alpha=0.34,
                     cutOff=12.0, cutOn=10.0, chargeConst=CHARGE_CONST):
    """The same energy in plain PyTorch FP64 on explicit pair lists (test
    reference): erfc direct term over `pairs` (i < j, within the cut-off),
    erf correction over `excl_pairs`, switched LJ (src/vdw.c:144-184) with
    eps_ij = sqrt(eps_i eps_j) * 418.4 and sig_ij = (sig_i + sig_j) / 2, and
    the self term."""
    types = torch.as_tensor(types, device=pos.device)
    eps_i = torch.sqrt(eps_t[types] * KCAL_TO_IU)
    sig_i = 0.5 * sig_t[types]

    def disp(p):
        i, j = p[:, 0], p[:, 1]
        d = pos[j] - pos[i]
        d = d - box * torch.round(d / box)
        r = torch.sqrt((d * d).sum(1))
        return i, j, r

    i, j, r = disp(torch.as_tensor(pairs, device=pos.device, dtype=torch.long))
    e = (chargeConst * q[i] * q[j] * torch.special.erfc(alpha * r) / r).sum()
    veps = eps_i[i] * eps_i[j]
    s6 = ((sig_i[i] + sig_i[j]) / r) ** 6
    lj = 4.0 * veps * (s6 * s6 - s6)
    r2 = r * r
    rc2, ron2 = cutOff * cutOff, cutOn * cutOn
    sw2 = 1.0 / (rc2 - ron2) ** 3
    sw = torch.where(r2 <= ron2, torch.ones_like(r2),
                     (rc2 - r2) ** 2 * (rc2 + 2.0 * r2 - 3.0 * ron2) * sw2)
    e = e + (lj * sw).sum()
    if excl_pairs is not None and len(excl_pairs):
        i, j, r = disp(torch.as_tensor(excl_pairs, device=pos.device, dtype=torch.long))
        e = e - (chargeConst * q[i] * q[j] * torch.erf(alpha * r) / r).sum()
    e = e - chargeConst * alpha / math.sqrt(math.pi) * (q * q).sum()
    return e
