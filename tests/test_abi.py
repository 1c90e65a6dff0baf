"""The C ABI: the library loads without a GPU, exports every entry point
include/*.h declares, and its struct layouts are MDBas's."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mdbas_nb.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text,
                         flags=re.M):
        name = m.group(1)
        if name in ("if", "while", "for", "sizeof", "return"):
            continue
        names.add(name)
    return sorted(names)


def test_library_exports_every_declared_function(nb_lib):
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(nb_lib, n)]
    assert not missing, missing


def test_no_checker_symbols_in_product():
    out = subprocess.run(["nm", "-D", "--defined-only",
                          os.path.join(ROOT, "mdbas_b200", "libmdbas_nb.so")],
                         capture_output=True, text=True, check=True).stdout
    assert " orc_" not in out and " ref_" not in out


def test_status_strings_and_mode(nb_lib):
    nb_lib.mdbas_nb_status_string.restype = C.c_char_p
    assert nb_lib.mdbas_nb_status_string(0) == b"ok"
    assert nb_lib.mdbas_nb_status_string(7).startswith(b"too few link cells")
    assert nb_lib.mdbas_nb_build_arch() == 1000
    assert nb_lib.mdbas_nb_set_mode(3) == 1
    assert nb_lib.mdbas_nb_set_mode(1) == 0 and nb_lib.mdbas_nb_get_mode() == 1
    assert nb_lib.mdbas_nb_set_mode(0) == 0 and nb_lib.mdbas_nb_get_mode() == 0


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include INCLUDE
#define OFF(T, f) (int)offsetof(T, f)
int main(void) {
  printf("PBC %d %d %d %d %d %d %d;", (int)sizeof(PBC), OFF(PBC, type), OFF(PBC, a1),
         OFF(PBC, u1), OFF(PBC, pa), OFF(PBC, vol0), OFF(PBC, stress9));
  printf("CTRL %d %d %d %d %d %d;", (int)sizeof(CTRL), OFF(CTRL, newjob), OFF(CTRL, keyLink),
         OFF(CTRL, keyEwald), OFF(CTRL, elecType), OFF(CTRL, ens));
  printf("PARAM %d %d %d %d %d %d %d %d;", (int)sizeof(PARAM), OFF(PARAM, timeStep),
         OFF(PARAM, nAtom), OFF(PARAM, tolShake), OFF(PARAM, chargeConst), OFF(PARAM, cutOff2),
         OFF(PARAM, switch2), OFF(PARAM, maxminst));
  printf("BOND %d %d %d %d;", (int)sizeof(BOND), OFF(BOND, a), OFF(BOND, k), OFF(BOND, beta));
  printf("ANGLE %d %d %d %d;", (int)sizeof(ANGLE), OFF(ANGLE, a), OFF(ANGLE, c),
         OFF(ANGLE, theta0));
  printf("DIHE %d %d %d %d;", (int)sizeof(DIHE), OFF(DIHE, order), OFF(DIHE, d),
         OFF(DIHE, mult));
  printf("NEIGH %d %d %d;", (int)sizeof(NEIGH), OFF(NEIGH, linkRatio), OFF(NEIGH, nPair14));
  printf("ENERGY %d %d %d %d;", (int)sizeof(ENERGY), OFF(ENERGY, elec), OFF(ENERGY, virelec),
         OFF(ENERGY, virtot));
  printf("CONSTRAINT %d %d;", (int)sizeof(CONSTRAINT), OFF(CONSTRAINT, rc2));
  printf("EWALD %d %d %d;", (int)sizeof(EWALD), OFF(EWALD, m3max), OFF(EWALD, alpha));
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_header_struct_layout_matches_mdbas(tmp_path):
    import oracle
    if not oracle.Reference.available():
        pytest.skip("MDBas reference library not built")
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f'-DINCLUDE="{HEADER}"', str(src), "-o", str(exe)], check=True)
    mine = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert mine == oracle.Reference.layout()


def test_ctypes_mirror_matches_header():
    from mdbas_b200 import nb
    sizes = {"PBC": nb.PBC, "CTRL": nb.CTRL, "PARAM": nb.PARAM, "BOND": nb.BOND,
             "ANGLE": nb.ANGLE, "DIHE": nb.DIHE, "NEIGH": nb.NEIGH, "ENERGY": nb.ENERGY,
             "CONSTRAINT": nb.CONSTRAINT, "EWALD": nb.EWALD}
    want = {"PBC": 320, "CTRL": 104, "PARAM": 200, "BOND": 40, "ANGLE": 32, "DIHE": 48,
            "NEIGH": 20, "ENERGY": 152, "CONSTRAINT": 16, "EWALD": 56}
    for k, t in sizes.items():
        assert C.sizeof(t) == want[k], k
    assert nb.PARAM.chargeConst.offset == 72 and nb.PBC.stress9.offset == 312
