"""Slab decomposition on the GPU engine (mdbas_b200/slab.py, EngineBackend):
one rank whose halo is its own lower face moved above the upper face, so
the local box is non-periodic along x and every pair across the periodic
face goes through the halo path (forward exchange, frozen halo atoms,
reverse force exchange).  Against the single-domain oracle (FP64, MDBas's
expressions): the plain FP64 form to 1e-12, the mixed form to 1e-5."""
import numpy as np
import pytest

from mdbas_b200 import slab

import slab_util


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["water", "ortho"])
@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_slab_self_halo_on_gpu(gpu, kind, precision, tol):
    s, cell = slab_util.system(kind)
    backend = slab.EngineBackend(precision=precision, device=gpu)
    try:
        owned, fx, fy, fz, e = slab_util.rank_forces(s, cell, 0, 1, backend, device="cuda:0")
    finally:
        backend.close()
    rfx, rfy, rfz, re = slab_util.reference(s, cell)
    order = np.argsort(owned)
    assert np.array_equal(owned[order], np.arange(s.n))
    fx, fy, fz = fx[order], fy[order], fz[order]
    num = np.sqrt(((fx - rfx) ** 2 + (fy - rfy) ** 2 + (fz - rfz) ** 2).sum())
    den = np.sqrt((rfx ** 2 + rfy ** 2 + rfz ** 2).sum())
    assert num / den < tol, num / den
    for k in ("e_dir", "e_corr", "e_vdw", "vir_dir", "vir_corr", "vir_vdw", "e_self"):
        assert abs(e[k] - re[k]) <= tol * max(abs(re[k]), 1.0), (k, e[k], re[k])
    if precision == 0:
        assert int(e["n_pairs"]) == int(re["n_pairs"])
    else:
        # FP32 distances at the cut-off may settle a pair or two otherwise
        assert abs(int(e["n_pairs"]) - int(re["n_pairs"])) <= 4
