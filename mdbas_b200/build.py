"""Build libmdbas_nb.so (all of csrc/) for sm_100a with nvcc, in tree.

Every translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` into
``mdbas_b200/_build/`` and linked into ``mdbas_b200/libmdbas_nb.so``.
pair_fp64.cu, bonded.cu and ewald_rec.cu are compiled with ``--fmad=false`` so
that the plain FP64 forms keep MDBas's uncontracted operation order.  Objects are rebuilt when their
source or any header under csrc/ or include/ is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmdbas_nb.so")
# bench-side FP32 peak probe, a library of its own (not part of libmdbas_nb.so)
PEAK_SRC = os.path.join(HERE, "peak", "fp32_peak.cu")
PEAK_LIB = os.path.join(HERE, "libmdbas_peak.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NO_FMAD = {"pair_fp64.cu", "bonded.cu", "ewald_rec.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hdrs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_time = _newest_header()
    cc = nvcc()
    objs, cmds = [], []
    for src in srcs:
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name.replace(".cu", ".o"))
        objs.append(obj)
        if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_time):
            continue
        cmd = [cc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-c", src, "-o", obj]
        if name in NO_FMAD:
            cmd.insert(1, "--fmad=false")
        cmds.append(cmd)
    procs = []
    maxjobs = jobs or min(8, os.cpu_count() or 4)
    failed = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len([p for _, p in procs if p.poll() is None]) >= maxjobs:
            procs[0][1].wait()
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((cmd, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"$ {' '.join(c)}\n{o}" for c, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if (not os.path.exists(LIB) or cmds
            or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)):
        link = [cc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-lcudart", "-lcufft",
                "-Xlinker", "-Bsymbolic"]
        if verbose:
            print(" ".join(link))
        subprocess.run(link, check=True)
    build_peak(cc, verbose)
    return LIB


def build_peak(cc: str | None = None, verbose: bool = False) -> str:
    """The FP32 peak probe library of the benchmark (libmdbas_peak.so)."""
    if (os.path.exists(PEAK_LIB)
            and os.path.getmtime(PEAK_LIB) >= os.path.getmtime(PEAK_SRC)):
        return PEAK_LIB
    cmd = [cc or nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler",
           "-fPIC", PEAK_SRC, "-o", PEAK_LIB]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return PEAK_LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
