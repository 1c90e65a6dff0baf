"""MDBas's own driver (src/mdbas.c) on the GPU library: the link recipe.

The same unmodified driver source is linked twice (oracle/Makefile, target
drivers): with all of MDBas's sources (oracle/_ref/mdbas_stock; src/spme.c
stubbed, FFTW3 is absent), and with energy.c, list.c, internal.c, ewald.c
and spme.c replaced by libmdbas_nb.so (oracle/_ref/mdbas_nb_linked, the
Makefile change INTEGRATION.md gives).  Both run the same SIMU / CONF / FORF
(3,000-atom flexible water, explicit Ewald, switched LJ, velocity Verlet, an
energy row every step) and their OUTPUT energy tables are compared: the
plain FP64 mode to MDBas's printed digits, the mixed mode within 1e-5 of
each printed total.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from mdbas_b200 import mdbas_files as mf
from mdbas_b200 import systems

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
STOCK = os.path.join(REF, "mdbas_stock")
LINKED = os.path.join(REF, "mdbas_nb_linked")
STEPS = 6


def _write_inputs(d):
    s = systems.config_small(seed=1)
    n = s.n
    labels = ["OT" if k % 3 == 0 else "HT" for k in range(n)]
    types = np.array([1 if k % 3 == 0 else 2 for k in range(n)], np.int32)
    mol = np.repeat(np.arange(1, n // 3 + 1), 3).astype(np.int32)
    mf.write_conf(str(d / "CONF"), mf.Conf(s.x, s.y, s.z, mol, mol, labels, ["TIP3"] * n,
                                          ["WAT"] * n))
    # flexible water: harmonic O-H bonds and H-O-H angle (internal units)
    bonded = {
        "bonds": {"atoms": s.bonds, "k": np.full(len(s.bonds), 450.0 * mf.KCAL_TO_IU),
                  "r0": np.full(len(s.bonds), systems.WATER_ROH)},
        "angles": {"atoms": s.angles, "k": np.full(len(s.angles), 55.0 * mf.KCAL_TO_IU),
                   "theta0": np.full(len(s.angles), systems.WATER_THETA)},
    }
    mf.write_forf(str(d / "FORF"), labels, types, s.q, s.mass, np.zeros(n, np.int32),
                  s.eps ** 2 / mf.KCAL_TO_IU, s.sig, bonded=bonded)
    mf.write_simu(str(d / "SIMU"), s.cell(), mf.CUBIC,
                  ["integrator velocity", "ensemble nve", "timestep 0.0005", f"nsteps {STEPS}",
                   "temperature 300.0", "seed 7", "print 1", "list 3", "cutoff 12.0",
                   "cuton 10.0", "delr 2.0", "elec ewald", "ewald alpha 0.34", "ewald prec 1e-6",
                   "vdw switch"])


def _energy_rows(path):
    """The energy table of an OUTPUT file: per printed step, its 15 numbers."""
    rows, cur = [], []
    with open(path) as fh:
        for ln in fh:
            parts = ln.split()
            if len(parts) != 5:
                continue
            try:
                vals = [float(p) for p in parts]
            except ValueError:
                continue
            cur.extend(vals)
            if len(cur) == 15:
                rows.append(cur)
                cur = []
    return np.array(rows)


def _run(exe, d, out, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([exe, "-i", "SIMU", "-o", out], cwd=str(d), env=e, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return _energy_rows(str(d / out))


@pytest.fixture(scope="module")
def stock_rows(tmp_path_factory):
    if not (os.path.exists(STOCK) and os.path.exists(LINKED)):
        pytest.skip("MDBas drivers not built (make -C oracle drivers with MDBAS_REF)")
    d = tmp_path_factory.mktemp("relink")
    _write_inputs(d)
    return d, _run(STOCK, d, "OUTPUT_stock")


def test_relinked_driver_fp64_matches_mdbas(gpu, stock_rows):
    d, ref = stock_rows
    got = _run(LINKED, d, "OUTPUT_nb", {"MDBAS_NB_MODE": "fp64"})
    assert ref.shape == (STEPS + 1, 15) and got.shape == ref.shape
    # every printed number (6 significant digits) agrees to its last digit
    scale = np.maximum(np.abs(ref), 1e-30)
    assert np.all(np.abs(got - ref) <= 1.001e-5 * scale + 1e-300), (got - ref) / scale


def test_relinked_driver_mixed_within_tolerance(gpu, stock_rows):
    d, ref = stock_rows
    got = _run(LINKED, d, "OUTPUT_mixed", {"MDBAS_NB_MODE": "mixed"})
    assert got.shape == ref.shape
    # step, time, volume exactly; totals (Etot, Ekin, Epot, Ecoul, Evdw, bonded)
    # within 1e-5 of MDBas's
    assert np.array_equal(got[:, [0, 1, 4]], ref[:, [0, 1, 4]])
    # (Ecoul is a small difference of large terms: its error is taken against
    # the potential energy's magnitude)
    epot = np.abs(ref[:, 7])
    for c in (5, 6, 7, 8, 9, 10, 11):
        rel = np.abs(got[:, c] - ref[:, c]) / np.maximum(np.abs(ref[:, c]), epot)
        assert np.all(rel <= 1e-5), (c, rel)
