"""MDBas's files (mdbas_b200/mdbas_files.py) against MDBas's own readers and
writers (src/io.c, compiled into oracle/_ref): the same fields from the same
SIMU / CONF / FORF files, and byte-identical RCON, REST, PROP and DCD output.
CPU only."""
import math
import os

import numpy as np
import pytest

from mdbas_b200 import mdbas_files as mf
from mdbas_b200 import nb, systems

import io_util

SIMU_LINES = [
    "mdbas", "timestep 0.0005", "nsteps 100", "cutoff 10.0", "cuton 8.0", "delr 1.5",
    "ewald prec 1e-5", "Ewald ALPHA 0.3", "ewald nbsp 6", "ewald recvec 7 8.9 9", "elec spme",
    "vdw switch", "nb14 0.5", "list 10", "link 2", "ensemble nvt beren", "taut 0.2",
    "taup 1.0", "temperature 310", "pressure 1.5", "compressibility 4.5e-5",
    "shake tol 1e-7", "shake maxcycle 200", "seed 42", "print 10", "prop 5", "traj 20",
    "resconf 50", "write field", "file conf CONF_T", "file forf FORF_T", "file rest REST_T",
    "file rcon RCON_T", "file prop PROP_T", "file traj TRAJ_T", "minim tol 0.01",
    "integrator velocity", "consth", "numforce", "",
]
CELL = [20.0, 0.0, 0.0, 1.0, 20.0, 0.0, 0.5, 1.5, 20.0]


@pytest.fixture(scope="module")
def ref_lib(ref_available):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    return io_util.bind(oracle.Reference.lib())


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("mdbas_files")
    s = systems.flexible_chains(3, 20.0, seed=2)
    n = s.n
    conf = mf.Conf(s.x, s.y, s.z, np.repeat(np.arange(1, n // 6 + 1), 6).astype(np.int32),
                   np.repeat(np.arange(1, n // 6 + 1), 6).astype(np.int32),
                   [f"C{k % 6 + 1}" for k in range(n)], ["CHN"] * n, ["SEGA"] * n)
    mf.write_conf(str(d / "CONF_T"), conf)
    frozen = np.zeros(n, np.int32)
    frozen[[3, 17, 40]] = 1
    cons = (s.bonds[4::5].copy(), np.full(len(s.bonds[4::5]), 1.53 ** 2))
    mf.write_forf(str(d / "FORF_T"), [f"C{k % 6 + 1}" for k in range(n)],
                  np.tile([1, 2, 2, 2, 2, 1], n // 6), s.q, s.mass, frozen,
                  s.eps ** 2 / mf.KCAL_TO_IU, s.sig, bonded=s.meta["bonded"], constraints=cons)
    mf.write_simu(str(d / "SIMU"), CELL, mf.TCLIN, SIMU_LINES)
    return d, s


def test_read_simu_matches_mdbas(ref_lib, files):
    d, _ = files
    io = io_util.io_with(simu=d / "SIMU")
    ctrl, param, bath, neigh, ewald, pbc = (nb.CTRL(), nb.PARAM(), io_util.BATH(), nb.NEIGH(),
                                            nb.EWALD(), nb.PBC())
    cwd = os.getcwd()
    ref_lib.read_SIMU(io, ctrl, param, bath, neigh, ewald, pbc)
    mine = mf.read_simu(str(d / "SIMU"))
    for want, got in ((ctrl, mine.ctrl), (param, mine.param), (ewald, mine.ewald),
                      (neigh, mine.neigh), (bath, mine.bath)):
        for k, v in got.items():
            assert getattr(want, k) == v, k
    assert pbc.type == mine.box_type
    assert [pbc.a1, pbc.a2, pbc.a3, pbc.b1, pbc.b2, pbc.b3, pbc.c1, pbc.c2, pbc.c3] == \
        list(mine.cell)
    for k, v in mine.files.items():
        assert getattr(io, f"{k}Name").decode() == v
    assert os.getcwd() == cwd
    assert mine.ewald["m2max"] == 8 and mine.ctrl["keyEwald"] == 2 and mine.ctrl["ens"] == mf.NVT_B


def _mdbas_conf_forf(ref_lib, d):
    import ctypes as C
    io = io_util.io_with(conf=d / "CONF_T", forf=d / "FORF_T")
    param = nb.PARAM()
    atom = C.POINTER(io_util.ATOM)()
    px, py, pz = (C.POINTER(C.c_double)() for _ in range(3))
    ref_lib.read_CONF(io, param, C.byref(atom), C.byref(px), C.byref(py), C.byref(pz))
    n = param.nAtom
    a = {k: np.zeros(n) for k in ("eps", "sig", "eps14", "sig14", "mass", "q")}
    fr, nat = np.zeros(n, np.int32), np.zeros(n, np.int32)
    cons = C.POINTER(nb.CONSTRAINT)()
    bond, ub = C.POINTER(nb.BOND)(), C.POINTER(nb.BOND)()
    angle = C.POINTER(nb.ANGLE)()
    dihe, impr = C.POINTER(nb.DIHE)(), C.POINTER(nb.DIHE)()
    ref_lib.read_FORF(io, param, atom, C.byref(cons), C.byref(bond), C.byref(angle),
                      C.byref(dihe), C.byref(impr), C.byref(ub),
                      *(a[k].ctypes.data for k in ("eps", "sig", "eps14", "sig14", "mass", "q")),
                      fr.ctypes.data, nat.ctypes.data)
    return dict(param=param, atom=atom, x=io_util.arr(px, n), y=io_util.arr(py, n),
                z=io_util.arr(pz, n), arrays=a, frozen=fr, nat=nat, cons=cons, bond=bond,
                ub=ub, angle=angle, dihe=dihe, impr=impr)


def test_read_conf_and_forf_match_mdbas(ref_lib, files):
    d, s = files
    ref = _mdbas_conf_forf(ref_lib, d)
    conf = mf.read_conf(str(d / "CONF_T"))
    forf = mf.read_forf(str(d / "FORF_T"), conf.n)
    n = conf.n
    assert ref["param"].nAtom == n == s.n
    for k in "xyz":
        assert np.array_equal(getattr(conf, k), ref[k])
    for i in range(n):
        at = ref["atom"][i]
        assert (at.label.decode(), at.resn.decode(), at.segn.decode(), at.ires, at.resi) == \
            (conf.label[i], conf.resn[i], conf.segn[i], conf.ires[i], conf.resi[i])
        assert at.type == forf.type[i]
    for k in ("eps", "sig", "eps14", "sig14", "mass", "q"):
        assert np.array_equal(getattr(forf, k), ref["arrays"][k]), k
    assert np.array_equal(forf.frozen, ref["frozen"])
    assert np.array_equal(forf.n_at_const, ref["nat"])
    p = ref["param"]
    pairs, len2 = forf.constraints
    assert p.nConst == len(len2) > 0
    for k in range(p.nConst):
        c = ref["cons"][k]
        assert (c.a, c.b, c.rc2) == (pairs[k][0], pairs[k][1], len2[k])
    structs = nb.bonded_structs(forf.bonded)
    counts = (p.nBond, p.nAngle, p.nUb, p.nDihedral, p.nImproper)
    refs = (ref["bond"], ref["angle"], ref["ub"], ref["dihe"], ref["impr"])
    for (m, arr), cnt, rp in zip(structs, counts, refs):
        assert m == cnt > 0
        for k in range(m):
            for f, _ in arr[k]._fields_:
                assert getattr(arr[k], f) == getattr(rp[k], f), f
    # the values survived the kcal/degree round trip to within a few ulps
    spec = s.meta["bonded"]
    assert np.allclose(forf.bonded["angles"]["theta0"], spec["angles"]["theta0"], rtol=1e-15)
    assert np.allclose(forf.eps, s.eps, rtol=1e-15)


def test_dihedral_order_field_kept(files):
    d, _ = files
    forf = mf.read_forf(str(d / "FORF_T"), systems.flexible_chains(3, 20.0, seed=2).n)
    assert "order" in forf.bonded["dihedrals"]


def test_write_conf_matches_mdbas(ref_lib, files, tmp_path):
    d, _ = files
    ref = _mdbas_conf_forf(ref_lib, d)
    io = io_util.io_with(rcon=tmp_path / "RCON_MDBAS")
    ref_lib.write_CONF(io, ref["param"], ref["atom"], ref["x"].ctypes.data,
                       ref["y"].ctypes.data, ref["z"].ctypes.data)
    conf = mf.read_conf(str(d / "CONF_T"))
    mf.write_conf(str(tmp_path / "RCON_MINE"), conf)
    assert (tmp_path / "RCON_MINE").read_bytes() == (tmp_path / "RCON_MDBAS").read_bytes()
    # and it reads back to the same coordinates at 1e-5 A
    back = mf.read_conf(str(tmp_path / "RCON_MINE"))
    assert np.max(np.abs(back.x - conf.x)) <= 5e-6


def test_write_conf_large_numbers_read_back(tmp_path):
    """Atom numbers past 99,999: MDBas's %5d%5d would join the atom and
    residue numbers; the writer keeps them apart."""
    n = 100002
    rng = np.random.default_rng(1)
    x, y, z = (rng.uniform(-50, 50, n) for _ in range(3))
    conf = mf.Conf(x, y, z, np.arange(1, n + 1, dtype=np.int32) // 3,
                   np.arange(1, n + 1, dtype=np.int32) // 3, ["OH2"] * n, ["TIP3"] * n,
                   ["W"] * n)
    mf.write_conf(str(tmp_path / "BIG"), conf)
    back = mf.read_conf(str(tmp_path / "BIG"))
    assert back.n == n and np.array_equal(back.ires, conf.ires)
    assert np.max(np.abs(back.z - z)) <= 5e-6


def test_restart_round_trip_with_mdbas(ref_lib, files, tmp_path):
    import ctypes as C
    d, s = files
    ref = _mdbas_conf_forf(ref_lib, d)
    n = s.n
    rng = np.random.default_rng(5)
    v = [rng.normal(size=n) for _ in range(6)]
    ener = nb.ENERGY()
    for i, (f, _) in enumerate(ener._fields_):
        setattr(ener, f, 0.25 * i - 1.0)
    bath = io_util.BATH(0.1, 0.02, 0.5, -0.03, 4e-5)
    param = ref["param"]
    param.step = 1234
    io = io_util.io_with(rest=tmp_path / "REST_MDBAS")
    ref_lib.write_rest(io, param, ener, bath, ref["atom"], ref["x"].ctypes.data,
                       ref["y"].ctypes.data, ref["z"].ctypes.data,
                       *(a.ctypes.data for a in v))
    mine = mf.read_rest(str(tmp_path / "REST_MDBAS"))
    assert mine.step == 1234 and len(mine.atoms) == n
    assert np.array_equal(mine.x, ref["x"]) and np.array_equal(mine.fz, v[5])
    assert mine.energy["virtot"] == ener.virtot and (mine.chiT, mine.chiP) == (0.02, -0.03)
    mf.write_rest(str(tmp_path / "REST_MINE"), mine)
    assert (tmp_path / "REST_MINE").read_bytes() == (tmp_path / "REST_MDBAS").read_bytes()
    # MDBas reads ours back
    io2 = io_util.io_with(rest=tmp_path / "REST_MINE")
    p2, e2, b2 = nb.PARAM(), nb.ENERGY(), io_util.BATH()
    atom2 = C.POINTER(io_util.ATOM)()
    ptrs = [C.POINTER(C.c_double)() for _ in range(9)]
    ref_lib.read_rest(io2, p2, e2, b2, C.byref(atom2), *(C.byref(p) for p in ptrs))
    assert p2.step == 1234 and p2.nAtom == n and e2.consv == ener.consv
    assert np.array_equal(io_util.arr(ptrs[3], n), v[0])
    with pytest.raises(mf.MdbasFileError):
        (tmp_path / "SHORT").write_bytes((tmp_path / "REST_MINE").read_bytes()[:100])
        mf.read_rest(str(tmp_path / "SHORT"))


def test_write_prop_matches_mdbas(ref_lib, tmp_path):
    pbc = nb.make_pbc(CELL, nb.TCLIN)
    ener = nb.ENERGY()
    for i, (f, _) in enumerate(ener._fields_):
        setattr(ener, f, 1000.0 * math.sin(i + 1))
    param = nb.PARAM()
    param.step, param.timeStep, param.nDegFree = 250, 0.001, 1791
    io = io_util.io_with(prop=tmp_path / "PROP_MDBAS")
    ref_lib.write_prop(io, param, ener, pbc)
    ref_lib.write_prop(io, param, ener, pbc)
    e = {f: getattr(ener, f) for f, _ in ener._fields_}
    for _ in range(2):
        mf.write_prop(str(tmp_path / "PROP_MINE"), 250, 0.001, 1791, e, pbc)
    assert (tmp_path / "PROP_MINE").read_bytes() == (tmp_path / "PROP_MDBAS").read_bytes()


def test_dcd_matches_mdbas(ref_lib, files, tmp_path):
    d, s = files
    n = s.n
    frozen = np.zeros(n, np.int32)
    frozen[[1, 2, 30]] = 1
    pbc = nb.make_pbc(CELL, nb.TCLIN)
    ctrl, param = nb.CTRL(), nb.PARAM()
    ctrl.printTraj = 10
    param.nSteps, param.nDegFree, param.nFrozen, param.nAtom = 105, 2 * n, 3, n
    io = io_util.io_with(traj=tmp_path / "TRAJ_MDBAS")
    ref_lib.write_DCD_header(io, ctrl, param, pbc, frozen.ctypes.data)
    x, y, z = (np.ascontiguousarray(a) for a in (s.x, s.y, s.z))
    for k in range(2):  # MDBas's first frame holds every atom, later ones the free atoms
        xk = x + k
        ref_lib.write_DCD_traj(io, param, pbc, xk.ctypes.data, y.ctypes.data, z.ctypes.data,
                               frozen.ctypes.data)
    mf.write_dcd_header(str(tmp_path / "TRAJ_MINE"), 105, 10, 2 * n, frozen, nb.TCLIN)
    for k in range(2):
        mf.write_dcd_frame(str(tmp_path / "TRAJ_MINE"), pbc, x + k, y, z, frozen, first=k == 0)
    a = (tmp_path / "TRAJ_MINE").read_bytes()
    b = (tmp_path / "TRAJ_MDBAS").read_bytes()
    assert len(a) == len(b)
    # the first title holds the creation time (seconds): compare around it
    assert a[:100] == b[:100] and a[180:] == b[180:]


def test_reader_errors(tmp_path):
    (tmp_path / "S").write_text("timestep 0.001\nbogus 1\nend\n")
    with pytest.raises(mf.MdbasFileError, match="SIMU_KEYWORD_ERROR"):
        mf.read_simu(str(tmp_path / "S"))
    (tmp_path / "S2").write_text("pbc 1\n-10 0 0\n0 10 0\n0 0 10\nend\n")
    with pytest.raises(mf.MdbasFileError, match="SIMU_PARAM_ERROR"):
        mf.read_simu(str(tmp_path / "S2"))
    (tmp_path / "F").write_text("atoms 2\n1 A 1 0.0 1.0 0\n2 B 1 0.0 1.0 2\nend\n")
    with pytest.raises(mf.MdbasFileError, match="21"):
        mf.read_forf(str(tmp_path / "F"), 2)
    with pytest.raises(mf.MdbasFileError, match="CONF_ATNUM_ERROR"):
        mf.read_forf(str(tmp_path / "F"), 3)
    (tmp_path / "C").write_text("* t\n    2\n    1    1 WAT  OH2    1.0 2.0 3.0 W 1 0.0\n")
    with pytest.raises(mf.MdbasFileError):
        mf.read_conf(str(tmp_path / "C"))


def test_load_builds_the_system(files):
    d, s = files
    sys2, simu, conf, forf = mf.load(str(d / "SIMU"))
    assert sys2.n == s.n and simu.box_type == mf.TCLIN
    assert np.array_equal(sys2.cell(), np.array(CELL))
    assert np.array_equal(sys2.bonds, s.bonds) and np.array_equal(sys2.angles, s.angles)
    assert sys2.meta["frozen"].sum() == 3 and len(sys2.meta["constraints"][1]) == len(s.bonds) // 5
    assert np.allclose(sys2.q, s.q, rtol=0, atol=0)
    # the engine side takes the spec as it is
    structs = nb.bonded_structs(sys2.meta["bonded"])
    assert [m for m, _ in structs] == [len(s.meta["bonded"][k]["atoms"])
                                       for k in nb.BONDED_KINDS]
