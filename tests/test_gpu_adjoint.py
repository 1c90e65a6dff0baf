"""Adjoint kernel (mdbas_nb_engine_adjoint) behind torch.autograd.Function,
on the gradient case: 12,000-atom charged LJ fluid, 4 types, 50 A cube.

Checked against (a) the FP64 reference gradient: autograd through the plain
PyTorch FP64 restatement of the energy (mdbas_b200.grad.reference_energy,
itself pinned to MDBas's energy() on CPU) on the engine's own pair set, and
(b) finite differences with MDBas's numderiv.c 4-point stencil
(-(8(c-b)-(d-a))/(12h), src/numderiv.c:102) at h = 1e-4.
"""
import numpy as np
import pytest
import torch

from mdbas_b200 import grad, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    s = systems.lj_fluid(12000, 50.0, seed=1)
    model = grad.RealSpaceModel(s, s.types)
    pos = torch.tensor(np.stack([s.x, s.y, s.z], 1), dtype=torch.float64)
    q = torch.tensor(s.q, dtype=torch.float64)
    eps_t = torch.tensor(s.type_eps_kcal, dtype=torch.float64)
    sig_t = torch.tensor(s.type_sigma, dtype=torch.float64)
    return s, model, pos, q, eps_t, sig_t


def _ref(case, pos, q, eps_t, sig_t):
    s, model = case[0], case[1]
    model.evaluate(pos.detach().numpy(), q.detach().numpy(), eps_t.detach().numpy(),
                   sig_t.detach().numpy())
    pairs = model.engine.export_pairs(144.0)
    dev = "cuda"
    args = [t.detach().to(dev).requires_grad_(True) for t in (pos, q, eps_t, sig_t)]
    e = grad.reference_energy(*args, s.types, pairs, None, s.box)
    return e, args


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_energy_gradient_vs_fp64_reference(gpu, case):
    s, model, pos, q, eps_t, sig_t = case
    qg, eg, sg = (t.clone().requires_grad_(True) for t in (q, eps_t, sig_t))
    pg = pos.clone().requires_grad_(True)
    e, f = model(pg, qg, eg, sg)
    e.backward()
    er, args = _ref(case, pos, q, eps_t, sig_t)
    er.backward()
    e, er = float(e.detach()), float(er.detach())
    print(f"E {e:.10e} ref {er:.10e}")
    assert abs(e - er) <= 1e-11 * abs(er)
    assert _rel(qg.grad, args[1].grad.cpu()) < 1e-10
    assert _rel(eg.grad, args[2].grad.cpu()) < 1e-10
    assert _rel(sg.grad, args[3].grad.cpu()) < 1e-10
    assert _rel(pg.grad, args[0].grad.cpu()) < 1e-10        # dE/dx = -F


def test_energy_gradient_vs_numderiv(gpu, case):
    s, model, pos, q, eps_t, sig_t = case
    qg, eg, sg = (t.clone().requires_grad_(True) for t in (q, eps_t, sig_t))
    e, _ = model(pos.clone(), qg, eg, sg)
    e.backward()
    h = 1e-4
    x0 = pos.numpy()

    def energy(qq, ee, ss):
        return model.evaluate(x0, qq, ee, ss)[0]

    def stencil(fn):
        a, b, c, d = fn(-2 * h), fn(-h), fn(h), fn(2 * h)
        return (8.0 * (c - b) - (d - a)) / (12.0 * h)

    # the FP64 form sums the energy with FP64 atomics in no fixed order, so
    # each evaluation carries ~E * 1e-16 of noise: the stencil's noise floor
    # is ~E * 1e-16 / h
    e0 = abs(float(e.detach()))
    floor = 10.0 * e0 * 2.2e-16 / h
    worst = 0.0
    for t in range(len(eps_t)):
        for which, vec, g in (("eps", eps_t, eg.grad), ("sig", sig_t, sg.grad)):
            def fn(dh, t=t, which=which, vec=vec):
                v = vec.numpy().copy()
                v[t] += dh
                return energy(q.numpy(), v, sig_t.numpy()) if which == "eps" else \
                    energy(q.numpy(), eps_t.numpy(), v)
            fd = stencil(fn)
            worst = max(worst, abs(fd - float(g[t])) / max(abs(fd), floor / 1e-6))
    for i in (0, 17, 4711, 11999):
        def fn(dh, i=i):
            v = q.numpy().copy()
            v[i] += dh
            return energy(v, eps_t.numpy(), sig_t.numpy())
        fd = stencil(fn)
        worst = max(worst, abs(fd - float(qg.grad[i])) / max(abs(fd), floor / 1e-6))
    print(f"worst relative difference to the 4-point stencil: {worst:.3e}")
    assert worst < 1e-6


def test_force_matching_loss_vs_fp64_reference(gpu, case):
    """L = mean |F(theta, x) - F_ref|^2 against forces of parameters perturbed
    by seeded factors in [0.95, 1.05]; dL/d(q, eps, sig) and dL/dx (a
    Hessian-vector product) from the adjoint vs double backward through the
    FP64 reference."""
    s, model, pos, q, eps_t, sig_t = case
    rng = np.random.default_rng(5)
    pert = [t * torch.tensor(rng.uniform(0.95, 1.05, t.shape[0])) for t in (q, eps_t, sig_t)]
    _, f_ref = model(pos.clone(), *pert)
    f_ref = f_ref.detach()
    n = s.n
    pg, qg, eg, sg = (t.clone().requires_grad_(True) for t in (pos, q, eps_t, sig_t))
    _, f = model(pg, qg, eg, sg)
    loss = ((f - f_ref) ** 2).sum() / n
    loss.backward()
    # reference: F = -dE/dx with create_graph, then the same loss
    er, args = _ref(case, pos, q, eps_t, sig_t)
    (dedx,) = torch.autograd.grad(er, args[0], create_graph=True)
    lr = ((-dedx - f_ref.to("cuda")) ** 2).sum() / n
    lr.backward()
    loss, lr = float(loss.detach()), float(lr.detach())
    print(f"loss {loss:.10e} ref {lr:.10e}")
    assert abs(loss - lr) <= 1e-9 * abs(lr)
    for mine, ref in ((qg.grad, args[1].grad), (eg.grad, args[2].grad),
                      (sg.grad, args[3].grad), (pg.grad, args[0].grad)):
        assert _rel(mine, ref.cpu()) < 1e-8


def test_hessian_vector_product_vs_numderiv(gpu, case):
    """d(v.F)/dx along a random direction w against the 4-point stencil of
    v.F(x + h w)."""
    s, model, pos, q, eps_t, sig_t = case
    rng = np.random.default_rng(9)
    v = rng.normal(size=(s.n, 3))
    w = rng.normal(size=(s.n, 3))
    model.evaluate(pos.numpy(), q.numpy(), eps_t.numpy(), sig_t.numpy())
    adj = model.engine.adjoint((v[:, 0], v[:, 1], v[:, 2]))
    hv = np.stack([adj["hx"], adj["hy"], adj["hz"]], 1)
    analytic = float((hv * w).sum())
    h = 1e-4
    x0 = pos.numpy()

    def vf(dh):
        _, f = model.evaluate(x0 + dh * w, q.numpy(), eps_t.numpy(), sig_t.numpy())
        return float((v * f).sum())

    a, b, c, d = vf(-2 * h), vf(-h), vf(h), vf(2 * h)
    fd = (8.0 * (c - b) - (d - a)) / (12.0 * h)
    print(f"w.d(v.F)/dx analytic {analytic:.10e} stencil {fd:.10e}")
    assert abs(analytic - fd) <= 1e-6 * abs(fd)
