"""A run set up from MDBas's own input files: SIMU / CONF / FORF written for
flexible chains with every bonded kind and one constraint per chain, read
back by mdbas_b200.mdbas_files.load, then 20 steps of GPU dynamics against
MDBas's integrator on the same system (FP64 form; SHAKE stops each molecule
at its own convergence, MDBas all at the worst one's: positions within 1e-6
A)."""
import numpy as np
import pytest

from mdbas_b200 import mdbas_files as mf
from mdbas_b200 import nb, systems

pytestmark = pytest.mark.gpu

POT = dict(cutOff=12.0, cutOn=10.0, delr=2.0, alpha=0.34)


def _write_inputs(d, s):
    n = s.n
    labels = [f"C{k % 6 + 1}" for k in range(n)]
    conf = mf.Conf(s.x, s.y, s.z, np.repeat(np.arange(1, n // 6 + 1), 6).astype(np.int32),
                   np.repeat(np.arange(1, n // 6 + 1), 6).astype(np.int32), labels,
                   ["CHN"] * n, ["SEGA"] * n)
    mf.write_conf(str(d / "CONF"), conf)
    cons = (s.bonds[4::5].copy(), np.full(len(s.bonds[4::5]), 1.53 ** 2))
    mf.write_forf(str(d / "FORF"), labels, np.ones(n, np.int32), s.q, s.mass,
                  np.zeros(n, np.int32), s.eps ** 2 / mf.KCAL_TO_IU, s.sig,
                  bonded=s.meta["bonded"], constraints=cons)
    mf.write_simu(str(d / "SIMU"), s.cell(), mf.CUBIC,
                  ["timestep 0.0005", "nsteps 20", "list 10", "elec full", "vdw switch"])


def test_md_from_mdbas_files_matches_mdbas(gpu, ref_available, tmp_path):
    if not ref_available:
        pytest.skip("MDBas harness library not built")
    import oracle
    src = systems.flexible_chains(4, 26.0, seed=5, temperature=300.0)
    _write_inputs(tmp_path, src)
    s, simu, conf, forf = mf.load(str(tmp_path / "SIMU"))
    vel = (src.vx, src.vy, src.vz)
    dt = simu.param["timeStep"]
    cons = s.meta["constraints"]
    structs = nb.bonded_structs(s.meta["bonded"])
    r = oracle.Reference(s, **POT)
    r.set_bonded(structs)
    r.makelist()
    excl = r.get_excl()
    r.md_init(s.mass, vel, time_step=dt, list_update=simu.neigh["update"], constraints=cons)
    rrows = r.md_run(simu.param["nSteps"])
    rp, rself = r.positions(), r.self_energy()
    r.close()
    e = nb.Engine(s, precision=0, exclusions=excl, **POT)
    e.set_bonded(s.meta["bonded"])
    e.md_init(s.mass, vel, time_step=dt, list_update=simu.neigh["update"], constraints=cons)
    grows = e.md_run(simu.param["nSteps"], energy_every=1)
    gp = e.positions()
    st = e.md_stats()
    e.close()
    d = max(np.max(np.abs((gp[k] - rp[k]) - s.box * np.round((gp[k] - rp[k]) / s.box)))
            for k in range(3))
    tot = np.max(np.abs(grows[:, 3] - (rrows[:, 3] + rself))) / np.max(np.abs(rrows[:, 3]))
    print(f"files -> GPU dynamics: pos {d:.3e} A, total energy {tot:.3e}, "
          f"constrained molecules {st['molecules']}")
    assert st["molecules"] == s.n // 6
    assert d < 1e-6
    assert tot < 1e-7
