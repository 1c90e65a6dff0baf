"""TEST INFRASTRUCTURE ONLY: numpy restatement of MDBas's smooth particle-mesh
Ewald (src/spme.c), the checker of the GPU SPME (mdbas_b200/csrc/spme.cu).

MDBas's spme.c includes <fftw3.h> and cannot be compiled here (FFTW3 is
absent), so this restatement follows its source step by step:

* grid sizes (init_spme, src/spme.c:32-68): the explicit-Ewald m_max of
  src/ewald.c's rule, each rounded up to a power of two p (p < 256) and
  doubled;
* B-spline moduli (epl_cplx/bspcoef, src/spme.c:170-267);
* per-atom B-splines and derivatives (bspgen, src/spme.c:269-355);
* charge spreading, FFTW_BACKWARD transform (unnormalised, e^{+i}),
  influence function with the reciprocal cut-off, FFTW_FORWARD transform,
  force interpolation, removal of the mean force, energy, self and
  non-neutral terms and the virial (spme_energy, src/spme.c:357-700).

It is pinned against MDBas's own explicit Ewald sum (ewald_rec,
src/ewald.c:131-354, compiled in oracle/_ref) by tests/test_spme_oracle.py.
"""
from __future__ import annotations

import math

import numpy as np


def nint(x: float) -> int:
    """MDBas nint (src/utils.c:606-609)."""
    return int(x + 0.5) if x >= 0 else int(x - 0.5)


def ewald_params(prec: float, cutoff: float, alpha: float | None = None):
    """tol, alpha, tol1 of init_ewald/init_spme (src/ewald.c:19-28)."""
    prec = min(abs(prec), 0.5)
    tol = math.sqrt(abs(math.log(prec * cutoff)))
    if alpha is None:
        alpha = math.sqrt(abs(math.log(prec * cutoff * tol))) / cutoff
    tol1 = math.sqrt(-math.log(prec * cutoff * (2.0 * tol * alpha) ** 2))
    return tol, alpha, tol1


def spme_grid(box, prec: float, cutoff: float, alpha: float):
    """Grid sizes of init_spme from the box's perpendicular widths pa, pb, pc
    (box = the 23-value layout of oracle.Oracle.box)."""
    _, _, tol1 = ewald_params(prec, cutoff, alpha)
    pa, pb, pc = box[18], box[19], box[20]
    out = []
    for p in (pa, pb, pc):
        m = nint(0.25 + p * alpha * tol1 / math.pi)
        p2 = 1
        while m > p2 and p2 < 256:
            p2 *= 2
        out.append(2 * p2)
    return tuple(out)


def _bsp_moduli(m: int, nbsp: int) -> np.ndarray:
    """|bspc[i]|^2 of bspcoef for one dimension."""
    bsp = np.zeros(nbsp)
    bsp[1] = 1.0
    for k in range(2, nbsp):
        bsp[k] = 0.0
        for j in range(k, 0, -1):
            bsp[j] = (j * bsp[j] + (k + 1 - j) * bsp[j - 1]) / k
    h = m // 2
    epl = np.zeros(m, dtype=complex)
    epl[0] = 1.0
    for i in range(1, h + 1):
        epl[i] = np.exp(1j * 2.0 * math.pi * i / m)
        epl[m - i] = np.conj(epl[i])
    out = np.zeros(m)
    for i in range(m):
        coeff = 0.0 + 0.0j
        for k in range(nbsp - 1):
            coeff += bsp[k + 1] * epl[(i * k) % m]
        c = epl[(i * (nbsp - 1)) % m] / coeff
        out[i] = (c * np.conj(c)).real
    return out


def _bspgen(s: np.ndarray, nbsp: int):
    """bspgen for one dimension: bsp[n, nbsp], bsd[n, nbsp]."""
    n = len(s)
    frac = s - np.trunc(s)
    bsp = np.zeros((n, nbsp))
    bsd = np.zeros((n, nbsp))
    bsd[:, 0] = 1.0
    bsd[:, 1] = -1.0
    bsp[:, 0] = frac
    bsp[:, 1] = 1.0 - frac
    for k in range(2, nbsp):
        bsp[:, k] = 0.0
        for j in range(k, 0, -1):
            if k == nbsp - 1:
                bsd[:, j] = bsp[:, j] - bsp[:, j - 1]
            ts = s + j - np.trunc(s)
            bsp[:, j] = (ts * bsp[:, j] + ((k + 1) - ts) * bsp[:, j - 1]) / k
        if k == nbsp - 1:
            bsd[:, 0] = bsp[:, 0]
        bsp[:, 0] = frac * bsp[:, 0] / k
    return bsp, bsd


def spme_energy(box, x, y, z, q, alpha: float, chargeConst: float, grid, nbsp: int = 8):
    """(energy, fx, fy, fz, virial) of spme_energy; energy includes the self
    and non-neutral terms, forces are the reciprocal ones alone."""
    x, y, z, q = (np.asarray(a, dtype=np.float64) for a in (x, y, z, q))
    n = len(x)
    m1, m2, m3 = grid
    # box layout of oracle.Oracle.box: a1..c3 = 0..8, u1..w3 = 9..17,
    # pa, pb, pc = 18..20, vol = 21; MDBas's box->u = 1/pa (src/init.c:873)
    u1, u2, u3, v1, v2, v3, w1, w2, w3 = box[9:18]
    vol = box[21]
    u, v, w = 1.0 / box[18], 1.0 / box[19], 1.0 / box[20]
    systq = q.sum()
    eself = -chargeConst * alpha * (q * q).sum() / math.sqrt(math.pi)
    rvol = 2.0 * math.pi / vol
    ralpha2 = -0.25 / (alpha * alpha)
    rc = min(min(m1 * u, m2 * v), m3 * w) * 1.05 * 2.0 * math.pi
    rc2 = rc * rc
    sx = m1 * (x * u1 + y * u2 + z * u3 + 0.5)
    sy = m2 * (x * v1 + y * v2 + z * v3 + 0.5)
    sz = m3 * (x * w1 + y * w2 + z * w3 + 0.5)
    b1, d1 = _bspgen(sx, nbsp)
    b2, d2 = _bspgen(sy, nbsp)
    b3, d3 = _bspgen(sz, nbsp)

    def wrap(idx, m):
        idx = np.where(idx >= m, 0, idx)
        return np.where(idx < 0, idx + m, idx)

    i0 = np.trunc(sx).astype(np.int64)
    j0 = np.trunc(sy).astype(np.int64)
    k0 = np.trunc(sz).astype(np.int64)
    ii = wrap(i0[:, None] - np.arange(nbsp)[None, :], m1)
    jj = wrap(j0[:, None] - np.arange(nbsp)[None, :], m2)
    kk = wrap(k0[:, None] - np.arange(nbsp)[None, :], m3)
    qsp = np.zeros((m1, m2, m3))
    for a in range(nbsp):
        for b in range(nbsp):
            wab = q * b1[:, a] * b2[:, b]
            for c in range(nbsp):
                np.add.at(qsp, (ii[:, a], jj[:, b], kk[:, c]), wab * b3[:, c])
    # FFTW_BACKWARD (e^{+i}, unnormalised) = N * numpy's ifftn
    ft = np.fft.ifftn(qsp) * (m1 * m2 * m3)
    bm1, bm2, bm3 = _bsp_moduli(m1, nbsp), _bsp_moduli(m2, nbsp), _bsp_moduli(m3, nbsp)
    i_ = np.arange(m1)
    j_ = np.arange(m2)
    k_ = np.arange(m3)
    iis = np.where(i_ > m1 // 2, i_ - m1, i_)
    jjs = np.where(j_ > m2 // 2, j_ - m2, j_)
    kks = np.where(k_ > m3 // 2, k_ - m3, k_)
    tw = 2.0 * math.pi
    rmx = (tw * iis[:, None, None] * u1 + tw * jjs[None, :, None] * v1 + tw * kks[None, None, :] * w1)
    rmy = (tw * iis[:, None, None] * u2 + tw * jjs[None, :, None] * v2 + tw * kks[None, None, :] * w2)
    rmz = (tw * iis[:, None, None] * u3 + tw * jjs[None, :, None] * v3 + tw * kks[None, None, :] * w3)
    rm = rmx * rmx + rmy * rmy + rmz * rmz
    bm = bm1[:, None, None] * bm2[None, :, None] * bm3[None, None, :]
    ok = (rm > np.finfo(float).eps) & (rm <= rc2)
    with np.errstate(divide="ignore", invalid="ignore"):
        rrm = np.where(ok, 1.0 / np.where(ok, rm, 1.0), 0.0)
        cam = np.where(ok, bm * np.exp(ralpha2 * rm) * rrm * ft, 0.0)
        vam = np.where(ok, 2.0 * (rrm - ralpha2) * (cam * np.conj(ft)).real, 0.0)
    stress = [-(vam * rmx * rmx).sum(), -(vam * rmx * rmy).sum(), -(vam * rmx * rmz).sum(),
              -(vam * rmy * rmy).sum(), -(vam * rmy * rmz).sum(), -(vam * rmz * rmz).sum()]
    # FFTW_FORWARD (e^{-i}, unnormalised) = numpy's fftn
    conv = np.fft.fftn(cam)
    qt = conv.real
    fact1 = -2.0 * rvol * chargeConst
    fx = np.zeros(n)
    fy = np.zeros(n)
    fz = np.zeros(n)
    for a in range(nbsp):
        for b in range(nbsp):
            for c in range(nbsp):
                g = qt[ii[:, a], jj[:, b], kk[:, c]]
                fbx = g * d1[:, a] * b2[:, b] * b3[:, c] * m1
                fby = g * b1[:, a] * d2[:, b] * b3[:, c] * m2
                fbz = g * b1[:, a] * b2[:, b] * d3[:, c] * m3
                fx += fact1 * q * (fbx * u1 + fby * v1 + fbz * w1)
                fy += fact1 * q * (fbx * u2 + fby * v2 + fbz * w2)
                fz += fact1 * q * (fbx * u3 + fby * v3 + fbz * w3)
    fx -= fx.mean()
    fy -= fy.mean()
    fz -= fz.mean()
    erec = (conv * qsp).sum().real
    enn = -(0.5 * math.pi * chargeConst) * ((systq / alpha) ** 2 / vol)
    f1 = rvol * chargeConst
    s0 = f1 * (stress[0] + erec) + enn
    s3 = f1 * (stress[3] + erec) + enn
    s5 = f1 * (stress[5] + erec) + enn
    energy = f1 * erec + eself + enn
    return energy, fx, fy, fz, -(s0 + s3 + s5)
