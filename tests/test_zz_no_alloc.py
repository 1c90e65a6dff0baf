"""The allocation-free entry point mdbas_nb_ewald_fp64_noalloc.

It exists for callers that cannot let the library allocate device memory
(programs that own all GPU memory through their own allocator, or loops that
must avoid the device-wide synchronisation of cudaMalloc/cudaFree).  This
test calls it through the C ABI twice in a row -- the second call reuses the
library's fixed scratch area with whatever the first call left in it -- and
checks both results against the ordinary FP64 entry point
(mdbas_nb_ewald_energy_status) on the same system and list, within the 1e-12
relative tolerance of the other FP64 tests.  It also checks that a system
larger than the fixed scratch area is refused before any GPU work.
"""
import ctypes as C

import numpy as np
import pytest

from mdbas_b200 import nb, systems
from dropin_util import DropinSystem, force_rel_rms

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _bind(L):
    P = C.POINTER
    f = L.mdbas_nb_ewald_fp64_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, P(nb.PBC), C.c_double, C.c_double, C.c_double, C.c_double, C.c_int] + \
        [C.c_void_p] * 14 + [P(C.c_double), C.c_void_p]
    return f


def test_noalloc_matches_regular_entry_point_twice(gpu):
    import torch
    L = nb.bind_dropin()
    L.mdbas_nb_set_mode(0)
    fn = _bind(L)
    s = systems.water_box_for_atoms(18558, seed=9)
    d = DropinSystem(s)
    d.makelist()  # link-cell list (wraps positions in place) + symmetric exclusions
    lst, pair, order = d.get_list()
    start, flat = d.get_excl()
    assert not np.array_equal(order, np.arange(s.n))  # exercise neighOrder

    # regular entry point on host arrays
    fx, fy, fz = np.zeros(s.n), np.zeros(s.n), np.zeros(s.n)
    ener = nb.ENERGY()
    assert L.mdbas_nb_ewald_energy_status(
        C.byref(d.ctrl), C.byref(d.param), C.byref(ener), C.byref(d.ewald), C.byref(d.box),
        nb.as_dp(d.x), nb.as_dp(d.y), nb.as_dp(d.z), nb.as_dp(fx), nb.as_dp(fy), nb.as_dp(fz),
        nb.as_dp(d.q), nb.as_dp(d.eps), nb.as_dp(d.sig), d.neighList, d.neighPair,
        d.neighOrder, d.exclList, d.exclPair) == 0

    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in dict(
        x=d.x, y=d.y, z=d.z, q=d.q, eps=d.eps, sig=d.sig, lst=lst, pair=pair, order=order,
        start=start, flat=flat if len(flat) else np.zeros(1, np.int32)).items()}
    outs = [[torch.zeros(s.n, dtype=torch.float64, device=dev) for _ in range(3)]
            for _ in range(2)]
    torch.cuda.synchronize()
    free = []
    for call in range(2):
        out = outs[call]
        en = (C.c_double * 6)()
        free.append(torch.cuda.mem_get_info(dev)[0])
        st = fn(s.n, C.byref(d.box), d.param.cutOff, d.param.cutOn, d.ewald.alpha,
                d.param.chargeConst, 1, *(t[k].data_ptr() for k in
                                          ("x", "y", "z", "q", "eps", "sig", "lst", "pair",
                                           "order", "start", "flat")),
                *(o.data_ptr() for o in out), en, None)
        assert st == 0, call
        torch.cuda.synchronize()
        f = [o.cpu().numpy() for o in out]
        assert force_rel_rms(f, (fx, fy, fz)) < TOL, call
        elec = en[0] + en[1]
        assert abs(elec - ener.elec) <= TOL * abs(ener.elec), call
        assert abs(en[2] - ener.vdw) <= TOL * abs(ener.vdw), call
        assert abs((en[3] + en[4]) - ener.virelec) <= TOL * abs(ener.virelec), call
        assert abs(en[5] - ener.virvdw) <= TOL * abs(ener.virvdw), call
    # the point of the entry point: the second call (set-up done by the
    # first) leaves the device's free memory exactly as it found it
    assert torch.cuda.mem_get_info(dev)[0] == free[1]
    d.free()


def test_noalloc_refuses_systems_beyond_its_scratch(gpu):
    import torch
    L = nb.bind_dropin()
    fn = _bind(L)
    box = nb.make_pbc([300.0, 0, 0, 0, 300.0, 0, 0, 0, 300.0])
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    en = (C.c_double * 6)()
    st = fn(131072 + 1, C.byref(box), 12.0, 10.0, 0.34, 1.0, 1,
            *([dummy.data_ptr()] * 14), en, None)
    assert st == 5  # MDBAS_NB_ERR_CAPACITY
    L.mdbas_nb_last_message.restype = C.c_char_p
    assert b"scratch limit" in L.mdbas_nb_last_message()
