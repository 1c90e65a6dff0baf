"""Benchmark of the real-space nonbonded hot path on B200.

Workload: the 96,000-atom rigid-water box (32,000 molecules, 98.6 A cube,
seeded lattice-plus-jitter generator), real-space Ewald (alpha 0.34 1/A)
+ CHARMM-switched LJ (10-12 A), Verlet skin 2 A.

One step = one pass of the hot path from FP64 positions: cell sort and
cluster-pair list build, then forces, energies and virial (FP32 pair kernel
with 64-bit fixed-point accumulation, FP64 exclusion corrections).  Nothing
is carried between steps but the topology; L2 is flushed (256 MiB write)
before every timed step.  ``value`` = in-cut-off pair interactions (r <= 12 A,
not excluded) per second of device time, summed over ranks; ``e2e`` is the
same through the engine's C ABI with host buffers (pinned H2D of the
positions and D2H of forces and energies inside the timed region).

Further keys: ``md`` (the device-resident velocity-Verlet step of the same box,
rigid water, rebuilds on half-skin displacement, CUDA-graph launches of 20
steps: ms per step and ns/day at 1 fs, and the NVE energy drift over
``--nve-steps``), ``md_fp64_form`` (the same loop over the plain FP64 form),
``large_box`` (999,999 atoms) and ``replicas`` (64 boxes in one engine).

``--impl reference`` times MDBas itself (oracle/_ref, its list rebuild +
energy() with real-space Ewald) on the host cores, one process per core
slot, each process evaluating its own copy of the workload per step.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ns/day & pairs/s (96k-atom real-space NB), FP32+fixed-pt vs FP64 form, 1 B200"
WORKLOAD = ("96,000-atom rigid water box (32,000 molecules, 98.6 A cube, 0.0334/A^3), "
            "real-space Ewald alpha 0.34 + switched LJ 10-12 A, skin 2 A")
# algorithmic FP32 flops per in-cut-off pair (FMA = 2): displacement 3, r^2 5,
# r 1, q_i q_j 1, exp argument 3, erfc polynomial x exp 14, E_dir 2, dE_dir 4,
# LJ core 14, switch 15, force scalar 2, force vector + i/j accumulation 9,
# energy + virial 4
FLOPS_PER_PAIR = 77
# algorithmic HBM bytes per atom of the list build's sort and layout stages:
#   bin: read FP64 x, y, z 24, write column 4 + fractional z 8
#   scatter: read column 4, write the column-ordered index 4 (+ column starts)
#   column sort: read index 4 + z 8, write the slot's atom 4
#   cluster layout, per slot (1.09 slots per atom at 96k, padding): read the
#     slot's atom 4, x, y, z 24, q, eps, sig 24; write float4 16 + float2 8,
#     their pair-interleaved copies 16 + 8, the atom's slot 4, per cluster
#     FP64 origin, FP32 origin and half extents (64 B / 8 slots) -> 112
BUILD_STAGE_BYTES = {"bin": 36, "scatter": 12, "column_sort": 16, "cluster_layout": 122}
LIST_BYTES_PER_ATOM = 36 + 12 + 16 + 122
FS_PER_STEP = 1.0


def _parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision-seeds", type=int, default=10)
    p.add_argument("--md-steps", type=int, default=1000,
                   help="timed velocity-Verlet steps (1 fs, rigid water) for ns/day")
    p.add_argument("--nve-steps", type=int, default=10000,
                   help="NVE steps (1 fs) for the energy-drift report; 0 skips it")
    p.add_argument("--pme-steps", type=int, default=200,
                   help="timed steps of the 96k dynamics with SPME in every step")
    p.add_argument("--large-steps", type=int, default=10,
                   help="timed steps of the 999,999-atom box; 0 skips it")
    p.add_argument("--replica-steps", type=int, default=100,
                   help="timed dynamics steps of the 64-replica batch (one CUDA graph); 0 skips")
    p.add_argument("--case", choices=["pair", "md", "build1m", "pair1m"], default=None,
                   help="run one case for a profiler and exit: 'pair' = 96k list build + 4 "
                        "force evaluations, 'md' = --md-steps 96k dynamics steps driven from "
                        "the host (a profiler sees no kernels inside graphs with conditional "
                        "nodes), 'build1m' = three 999,999-atom list builds, 'pair1m' = one "
                        "999,999-atom build + 2 force evaluations")
    p.add_argument("--variant", type=int, default=7, help="pair kernel variant of --case pair")
    p.add_argument("--dropin-steps", type=int, default=10,
                   help="steps of the drop-in e2e leg (0 skips it)")
    p.add_argument("--decomp", choices=["replicas", "slab"], default="replicas",
                   help="replicas: every rank runs its own copy of the 96k box (the "
                        "default line); slab: the 999,999-atom box split into slabs along "
                        "x over the ranks (halo exchange, strong scaling)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of the benchmarked GPU while the timed
    region runs.  NVML is polled every 5 ms from a thread (the GPU found by its
    PCI address, so CUDA_VISIBLE_DEVICES cannot mislead it); start() returns
    once the first sample is in, so even a region of a few milliseconds gets
    samples.  Falls back to `nvidia-smi -lms` when NVML cannot be used."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []
        self.smax = None
        self.stop_flag = False
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.dev)
        bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            first = threading.Event()

            def poll():
                while not self.stop_flag:
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                          int(get_reasons(h))))
                    except Exception:
                        pass
                    first.set()
                    time.sleep(0.005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            first.wait(timeout=2.0)
            self.source = "nvml"
            return
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(prefix="clocks", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi"
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=2.0)
            rows = list(self.rows)
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"],
                        "source": "nvml"}
            reasons = sorted({name for _, bits in rows for name, m in self.REASONS if bits & m})
            return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(rows), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = [n for n, _ in self.REASONS]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi"}


# ---------------------------------------------------------------------------
# reference arm: MDBas on the host cores
# ---------------------------------------------------------------------------
def _ref_worker(seed, steps, warmup, barrier, queue):
    import oracle
    from mdbas_b200 import systems
    s = systems.config_96k(seed=seed, temperature=None)
    r = oracle.Reference(s)
    r.makelist()
    x, y, z = r.positions()
    times = []
    for k in range(warmup + steps):
        barrier.wait()
        t0 = r.now()
        r.update_list(x, y, z)
        r.energy()
        t1 = r.now()
        if k >= warmup:
            times.append(t1 - t0)
    queue.put(times)


def _count_pairs(seed):
    import oracle
    from mdbas_b200 import systems
    s = systems.config_96k(seed=seed, temperature=None)
    o = oracle.Oracle()
    box = o.box(s.cell())
    excl = s.exclusions(symmetric=True)
    return len(o.pairs_within(box, s.x, s.y, s.z, excl, 144.0))


def run_reference(args, rank, world):
    import oracle
    if rank != 0:
        return
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libmdbas_ref.so (MDBas built from its sources) is missing"}))
        return
    cores = os.cpu_count() or 1
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    procs_n = max(1, min(cores, 32))
    pairs = _count_pairs(args.seed)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs_n)
    queue = ctx.Queue()
    steps = max(1, args.steps)
    warm = max(0, min(args.warmup, 3))
    ps = [ctx.Process(target=_ref_worker, args=(args.seed + k, steps, warm, barrier, queue))
          for k in range(procs_n)]
    for p in ps:
        p.start()
    res = [queue.get() for _ in ps]
    for p in ps:
        p.join()
    # each step: every process evaluates one copy; the step lasts as long as
    # its slowest process
    step_t = [max(r[k] for r in res) for k in range(steps)]
    t = sum(step_t) / steps
    value = procs_n * pairs / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOAD, "n_atoms": 96000, "in_cutoff_pairs": pairs,
                   "step": "MDBas link_cell_verlet_list_update + energy() (keyEwald=3)",
                   "processes": procs_n},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": procs_n, "kind": "reference",
                         "sample": f"{procs_n} processes x {steps} steps, one 96k-atom list "
                                   f"rebuild + energy() each", "host": _host_cpu()},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "ns_per_day": 86400.0 / t * FS_PER_STEP * 1e-6,
    }
    print(json.dumps(line))


def cpu_baseline_sample(seed: int, gpu_list=None, gpu_list64=None, gpu_forces=None) -> dict:
    """MDBas single-threaded on the host: list rebuild + energy(), ~3 steps.
    With gpu_list / gpu_list64 (functions of the wrapped positions returning
    a GPU list's unordered pairs: the timed mixed path's cluster list, the
    FP64 form's MDBas-order list), the result also carries "list_parity" /
    "list_parity_fp64_form": MDBas's neighbour pair set against them on the
    same 96k coordinates.  With gpu_forces (positions -> forces, energies of
    the timed mixed path), "vs_mdbas" compares them with MDBas's energy() of
    the last sample."""
    import numpy as np
    import oracle
    from mdbas_b200 import systems
    if not oracle.Reference.available():
        return {"value": None, "unit": "pairs/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    s = systems.config_96k(seed=seed, temperature=None)
    r = oracle.Reference(s)
    r.makelist()
    x, y, z = r.positions()
    pairs = _count_pairs(seed)
    ts, tl, te = [], [], []
    t_start = time.perf_counter()
    while len(ts) < 3 or (time.perf_counter() - t_start < 10 and len(ts) < 6):
        t0 = r.now()
        r.update_list(x, y, z)
        t1 = r.now()
        ref_out = r.energy()
        t2 = r.now()
        ts.append(t2 - t0)
        tl.append(t1 - t0)
        te.append(t2 - t1)
    parity = parity64 = vs = None
    if gpu_list is not None or gpu_list64 is not None:
        lst, pair, order = r.get_list()
        if gpu_list is not None:
            gp = gpu_list(x, y, z)
            parity = _same_pair_set(s.n, np.repeat(order, pair[order]), lst, gp[:, 0], gp[:, 1])
            parity["gpu_list"] = "cluster-pair list of the timed mixed path (precision 1)"
        if gpu_list64 is not None:
            gp = gpu_list64(x, y, z)
            parity64 = _same_pair_set(s.n, np.repeat(order, pair[order]), lst, gp[:, 0],
                                      gp[:, 1])
            parity64["gpu_list"] = "MDBas-order list of the plain FP64 form (precision 0)"
    if gpu_forces is not None:
        rfx, rfy, rfz, re = ref_out
        (gx, gy, gz), ge = gpu_forces(x, y, z)
        num = ((gx - rfx) ** 2 + (gy - rfy) ** 2 + (gz - rfz) ** 2).sum()
        den = (rfx ** 2 + rfy ** 2 + rfz ** 2).sum()
        elec = ge["elec_direct"] + ge["elec_corr"]
        vs = {"force_rel_rms_vs_mdbas": float(np.sqrt(num / den)),
              "elec_rel_vs_mdbas": abs(elec - re["elec"]) / abs(re["elec"]),
              "vdw_rel_vs_mdbas": abs(ge["vdw"] - re["vdw"]) / abs(re["vdw"]),
              "what": "timed mixed path vs MDBas energy() (keyEwald 3), 96k seed "
                      f"{seed}, MDBas's wrapped coordinates"}
    r.close()
    t = statistics.median(ts)
    return {"list_parity": parity, "list_parity_fp64_form": parity64, "vs_mdbas": vs,
            "value": pairs / t, "unit": "pairs/s", "cores": 1, "kind": "reference",
            "sample": f"{len(ts)} x (96k-atom link_cell_verlet_list_update + energy()), "
                      f"median {t:.2f} s",
            "list_update_s": statistics.median(tl), "energy_s": statistics.median(te),
            "host": _host_cpu()}


def mdbas_errors(nb, systems, dev) -> dict:
    """Mixed-form forces and energies against MDBas itself (oracle/_ref:
    energy() with real-space Ewald, keyEwald 3) on the small water box, the
    charged LJ fluid of the gradient case and the median box of the replica
    batch; the 999,999-atom box on a 10,000-atom subset against the FP64
    restatement; the 96k box is compared in cpu_baseline_sample."""
    import numpy as np
    import oracle
    if not oracle.Reference.available():
        return {"unavailable": "oracle/_ref not built"}
    out = {}
    for name, s in (("water_3k_seed1", systems.config_small(seed=1)),
                    ("lj_fluid_12k_seed1", systems.lj_fluid(seed=1))):
        r = oracle.Reference(s)
        r.makelist()
        x, y, z = r.positions()
        rfx, rfy, rfz, re = r.energy()
        r.close()
        sp = systems.System(s.name, s.box, x, y, z, s.q, s.eps, s.sig, s.mass, s.bonds,
                            s.angles)
        e = nb.Engine(sp, precision=1, device=dev)
        e.build()
        e.compute()
        fx, fy, fz = e.forces()
        en = e.energies()
        e.close()
        num = ((fx - rfx) ** 2 + (fy - rfy) ** 2 + (fz - rfz) ** 2).sum()
        den = (rfx ** 2 + rfy ** 2 + rfz ** 2).sum()
        elec = en["elec_direct"] + en["elec_corr"]
        out[name] = {"n_atoms": s.n, "force_rel_rms": float(np.sqrt(num / den)),
                     "elec_rel": abs(elec - re["elec"]) / abs(re["elec"]),
                     "vdw_rel": abs(en["vdw"] - re["vdw"]) / max(abs(re["vdw"]), 1e-300)}
    # one box of the replica batch (the median size) against MDBas
    sizes = systems.replica_sizes(64, seed=1)
    k = int(np.argsort(sizes)[len(sizes) // 2])
    batch = systems.config_replicas(64, seed=1)
    rep = systems.replica(batch, k)
    r = oracle.Reference(rep)
    r.makelist()
    x, y, z = r.positions()
    rfx, rfy, rfz, re = r.energy()
    r.close()
    sp = systems.System(rep.name, rep.box, x, y, z, rep.q, rep.eps, rep.sig, rep.mass,
                        rep.bonds, rep.angles)
    e = nb.Engine(sp, precision=1, device=dev)
    e.build()
    e.compute()
    fx, fy, fz = e.forces()
    en = e.energies()
    e.close()
    num = ((fx - rfx) ** 2 + (fy - rfy) ** 2 + (fz - rfz) ** 2).sum()
    den = (rfx ** 2 + rfy ** 2 + rfz ** 2).sum()
    elec = en["elec_direct"] + en["elec_corr"]
    out[f"replica_{k}_of_64"] = {"n_atoms": rep.n, "force_rel_rms": float(np.sqrt(num / den)),
                                  "elec_rel": abs(elec - re["elec"]) / abs(re["elec"]),
                                  "vdw_rel": abs(en["vdw"] - re["vdw"]) / abs(re["vdw"])}
    # the 999,999-atom box: the forces of a seeded 10,000-atom subset against
    # the FP64 restatement (bit-exact with MDBas's ewald_energy on its pairs)
    big = systems.config_1m(seed=1)
    e = nb.Engine(big, precision=1, device=dev)
    e.build()
    e.compute()
    fx, fy, fz = e.forces()
    e.close()
    o = oracle.Oracle()
    sub = np.sort(np.random.default_rng(11).choice(big.n, 10000, replace=False)).astype(np.int32)
    gx, gy, gz = o.forces_subset(o.box(big.cell()), big, big.exclusions(symmetric=True), sub)
    num = ((fx[sub] - gx) ** 2 + (fy[sub] - gy) ** 2 + (fz[sub] - gz) ** 2).sum()
    den = (gx ** 2 + gy ** 2 + gz ** 2).sum()
    out["water_1m_seed1_subset10k"] = {"n_atoms": big.n, "subset": int(len(sub)),
                                       "force_rel_rms": float(np.sqrt(num / den)),
                                       "against": "FP64 C restatement (oracle), 10,000 atoms"}
    return out


def dropin_e2e(nb, systems, seed, steps) -> dict:
    """The calls MDBas makes, timed end to end on host arrays through the C
    ABI (wall clock around each synchronous call, which copies the positions
    in and the forces out):
      * energy() (include/energy.h:30-37) in mixed mode;
      * mdbas_nb_user_energy (the UserEnergyPtr plugin, include/user.h:29-33)
        in mixed mode;
      * the plugin in the plain FP64 form over a caller-built MDBas list (the
        library's own list copied into the caller's arrays, so it is uploaded
        on every call, as a list from MDBas's list.c would be).
    Every step moves all atoms by 1.2 A (a rigid shift back and forth), past
    half the skin, so the mixed calls rebuild their cluster list each time,
    like the step of the headline figure."""
    import ctypes as C

    import numpy as np
    L = nb.bind_dropin()
    s = systems.config_96k(seed=seed, temperature=None)
    n = s.n
    P = C.POINTER
    ctrl = nb.CTRL()
    ctrl.newjob = 1
    ctrl.keyEwald = 3
    ctrl.elecType = nb.FULL
    ctrl.vdwType = nb.VSWITCH
    param = nb.make_param(n, 12.0, 10.0, 2.0)
    param.nBond = len(s.bonds)
    param.nAngle = len(s.angles)
    box = nb.make_pbc(s.cell())
    neigh = nb.NEIGH()
    neigh.update = 1
    neigh.linkRatio = 1
    ewald = nb.EWALD()
    ewald.alpha = 0.34
    ener = nb.ENERGY()
    bond = (nb.BOND * len(s.bonds))()
    for k, (a, b) in enumerate(s.bonds.tolist()):
        bond[k].a, bond[k].b = a, b
    angle = (nb.ANGLE * len(s.angles))()
    for k, (a, b, c) in enumerate(s.angles.tolist()):
        angle[k].a, angle[k].b, angle[k].c = a, b, c
    const, dihe, impr = (nb.CONSTRAINT * 1)(), (nb.DIHE * 1)(), (nb.DIHE * 1)()
    x = np.ascontiguousarray(s.x).copy()
    y = np.ascontiguousarray(s.y).copy()
    z = np.ascontiguousarray(s.z).copy()
    q, eps, sig = (np.ascontiguousarray(a, dtype=np.float64) for a in (s.q, s.eps, s.sig))
    frozen = np.zeros(n, np.int32)
    vx, vy, vz = np.zeros(n), np.zeros(n), np.zeros(n)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    lst, pair, order, l14 = (P(C.c_int)() for _ in range(4))
    excl, epair = P(P(C.c_int))(), P(C.c_int)()
    L.mdbas_nb_set_mode(0)
    L.makelist(C.byref(ctrl), C.byref(param), C.byref(box), C.byref(neigh), const, bond, angle,
               dihe, impr, nb.as_dp(x), nb.as_dp(y), nb.as_dp(z), nb.as_ip(frozen),
               C.byref(lst), C.byref(pair), C.byref(order), C.byref(l14), C.byref(excl),
               C.byref(epair))
    L.init_energy_ptrs(C.byref(ctrl))
    pe = nb.PARAM.from_buffer_copy(param)
    pe.nBond = 0  # the nonbonded path only (no bonded terms)
    pe.nAngle = 0
    assert L.mdbas_nb_plugin_init(n, nb.as_dp(q), nb.as_dp(eps), nb.as_dp(sig), epair, excl,
                                  0.34, 1) == 0
    xs = [(x, y, z), (x + 1.2, y + 1.2, z + 1.2)]
    xs = [tuple(np.ascontiguousarray(a) for a in t) for t in xs]

    def call_energy(k):
        a, b, c = xs[k & 1]
        L.energy(C.byref(ctrl), C.byref(pe), C.byref(ener), C.byref(ewald), C.byref(box),
                 C.byref(neigh), bond, bond, angle, dihe, impr, nb.as_dp(a), nb.as_dp(b),
                 nb.as_dp(c), nb.as_dp(vx), nb.as_dp(vy), nb.as_dp(vz), nb.as_dp(fx),
                 nb.as_dp(fy), nb.as_dp(fz), nb.as_dp(q), nb.as_dp(eps), nb.as_dp(sig),
                 nb.as_dp(eps), nb.as_dp(sig), nb.as_ip(frozen), lst, pair, order, l14, excl,
                 epair)

    def call_plugin(k, lists):
        a, b, c = xs[k & 1]
        fx[:] = 0.
        fy[:] = 0.
        fz[:] = 0.
        L.mdbas_nb_user_energy(C.byref(pe), C.byref(box), nb.as_dp(a), nb.as_dp(b),
                               nb.as_dp(c), nb.as_dp(fx), nb.as_dp(fy), nb.as_dp(fz), *lists)

    def timed(fn, k_steps):
        for k in range(3):
            fn(k)
        ts = []
        for k in range(k_steps):
            t0 = time.perf_counter()
            fn(k)
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts) * 1e3

    out = {}
    try:
        L.mdbas_nb_set_mode(1)
        out["energy_mixed_ms"] = timed(call_energy, steps)
        out["plugin_mixed_ms"] = timed(lambda k: call_plugin(k, (lst, pair, order, l14)), steps)
        L.mdbas_nb_set_mode(0)
        # the same list in caller-owned arrays: uploaded on every call
        tot = int(np.ctypeslib.as_array(pair, (n,)).sum())
        cl = np.ctypeslib.as_array(lst, (tot,)).copy()
        cp = np.ctypeslib.as_array(pair, (n,)).copy()
        co = np.ctypeslib.as_array(order, (n,)).copy()
        own = (nb.as_ip(cl), nb.as_ip(cp), nb.as_ip(co), l14)
        out["plugin_fp64_caller_list_ms"] = timed(lambda k: call_plugin(0, own),
                                                  max(3, steps // 4))
        out["caller_list_bytes"] = int(4 * (tot + 2 * n))
    finally:
        L.mdbas_nb_set_mode(0)
    out["h2d_bytes_per_step"] = 3 * 8 * n
    out["d2h_bytes_per_step"] = 3 * 8 * n
    out["what"] = ("96k water, host arrays, synchronous C-ABI calls timed by wall clock; each "
                   "mixed call rebuilds the cluster list (positions moved past half the skin)")
    return out


def _same_pair_set(n, ai, aj, bi, bj) -> dict:
    """Set equality of two unordered pair lists (keys min * n + max, sorted
    on the GPU)."""
    import numpy as np
    import torch
    def keys(i, j):
        i = torch.as_tensor(np.asarray(i, dtype=np.int64), device="cuda")
        j = torch.as_tensor(np.asarray(j, dtype=np.int64), device="cuda")
        return torch.sort(torch.minimum(i, j) * n + torch.maximum(i, j)).values
    ka, kb = keys(ai, aj), keys(bi, bj)
    same = ka.numel() == kb.numel() and bool(torch.equal(ka, kb))
    return {"mdbas_pairs": int(ka.numel()), "gpu_pairs": int(kb.numel()), "bit_exact": same,
            "what": "set of unordered (i, j) of MDBas's link-cell list (r <= 14 A) and the "
                    "GPU builder's, same wrapped 96k coordinates"}


def hbm_peak() -> float:
    """Measured HBM copy bandwidth (GB/s) of this pool's B200s, from the
    driver-written MEASURED_PEAKS.json, else the recipe's fallback."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def fp32_peaks(device: int) -> tuple:
    """Measured FP32 FMA throughput of the device (TFLOP/s): scalar FFMA and
    packed f32x2 FMA, from the bench-side probe library."""
    import ctypes as C

    from mdbas_b200 import build as nb_build
    lib = C.CDLL(nb_build.build_peak())
    tf, ms = (C.c_double * 2)(), (C.c_double * 2)()
    st = lib.mdbas_peak_fp32(device, tf, ms)
    if st != 0:
        raise RuntimeError(f"FP32 peak probe failed (CUDA error {st})")
    return tf[0], tf[1]


def _host_cpu() -> dict:
    """CPU model and logical core count of the host the baseline ran on."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _time_steps(torch, eng, stream, flush, steps, fn):
    evs = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def _time_split_steps(torch, stream, flush, steps, first, second):
    """Steps of first() then second(), with an event between them: per step
    (first ms, second ms), so the two parts add up to the step time."""
    evs = []
    for _ in range(steps):
        flush.zero_()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        first()
        e[1].record(stream)
        second()
        e[2].record(stream)
        evs.append(e)
    torch.cuda.synchronize()
    return [(a.elapsed_time(b), b.elapsed_time(c)) for a, b, c in evs]


def md_measure(torch, nb, systems, dev, stream, seed, precision, steps, nve_steps, world,
               kspace=None):
    """Velocity-Verlet dynamics of the 96k water box (rigid SHAKE/RATTLE
    water, list rebuilt on half-skin displacement).  The lattice-plus-jitter
    start is relaxed first (2,000 Berendsen steps at 0.5 fs toward 300 K,
    untimed); then `steps` 1 fs NVE steps are timed with CUDA events on the
    engine stream, and `nve_steps` more give the energy drift.  kspace =
    (kind, grid, order) adds reciprocal space to every step."""
    import numpy as np
    s = systems.config_96k(seed=seed, temperature=300.0)
    cons = s.water_constraints()
    e = nb.Engine(s, precision=precision, device=dev)
    e.set_stream(stream.cuda_stream)
    if kspace is not None:
        e.set_kspace(*kspace)
    e.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.0005, list_update=0, constraints=cons)
    e.md_run(2000, target_temp=300.0, tau_t=0.05)
    pos, vel = e.positions(), e.velocities()
    e.set_positions(*pos)
    e.md_init(s.mass, vel, time_step=0.001, list_update=0, constraints=cons)
    e.md_run(20)
    st0 = e.md_stats()
    launches0 = e.launches()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e.md_run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    from mdbas_b200 import ranks
    ms = ranks.max_over_ranks([e0.elapsed_time(e1) / steps], "cuda" if world > 1 else "cpu")[0]
    st1 = e.md_stats()
    out = {"ms_per_step": ms, "ns_per_day": 86400.0 / (ms * 1e-3) * 1e-6,
           "time_step_fs": 1.0, "steps_timed": steps,
           "list_builds_per_step": (st1["rebuilds"] - st0["rebuilds"]) / steps,
           "launches_per_step": (e.launches() - launches0) / steps,
           "constraints": "rigid water, SHAKE/RATTLE tol 1e-8",
           "start": "2,000 Berendsen steps (0.5 fs, tau 0.05 ps, 300 K) from the lattice start"}
    if nve_steps > 0:
        every = 100
        rows = e.md_run(nve_steps, energy_every=every)
        n = s.n
        ndf = 3 * n - len(cons[1]) - 3
        tot, kin = rows[:, 3], rows[:, 2]
        kT = 2.0 * float(np.mean(kin)) / ndf
        t_ns = nve_steps * 1e-6
        slope = float(np.polyfit(rows[:, 0] * 1e-6, tot, 1)[0])  # per ns
        out["nve"] = {
            "steps": nve_steps, "time_step_fs": 1.0, "energy_every": every,
            "temperature_K": kT / 0.83144621,
            "drift_kT_per_dof_per_ns": slope / (ndf * kT),
            "total_first_last_kcal_mol": [float(tot[0]) / 418.4, float(tot[-1]) / 418.4],
            "max_dev_over_kin": float((tot.max() - tot.min()) / np.mean(kin)),
            "rebuilds": e.md_stats()["rebuilds"] - st1["rebuilds"],
            "simulated_ns": t_ns}
    e.close()
    return out


def large_box_measure(torch, nb, systems, dev, stream, flush, seed, steps):
    """The 999,999-atom water box (333,333 molecules, 215 A cube): the mixed
    form's list build, pair kernel and whole step, and its forces against the
    plain FP64 GPU form on every atom."""
    import numpy as np
    s = systems.config_1m(seed=seed)
    n = s.n
    eng = nb.Engine(s, precision=1, device=dev)
    eng.set_stream(stream.cuda_stream)
    for _ in range(3):
        eng.build()
        eng.compute()
    torch.cuda.synchronize()
    pairs = int(eng.energies()["n_pairs"])
    stats = eng.list_stats()

    def step():
        eng.build()
        eng.compute()

    ms = _time_steps(torch, eng, stream, flush, steps, step)
    ms_build = _time_steps(torch, eng, stream, flush, steps, eng.build)
    # the build stage by stage (CUDA events between the launches, L2 flushed
    # first), with each stage's algorithmic HBM bytes
    stage_runs = []
    for _ in range(max(3, steps)):
        flush.zero_()
        torch.cuda.synchronize()
        stage_runs.append(eng.build_stages())
    stages = {}
    for k in stage_runs[0]:
        t = statistics.median(r[k] for r in stage_runs)
        b = BUILD_STAGE_BYTES.get(k)
        stages[k] = {"ms": t}
        if b is not None:
            stages[k]["bytes_per_atom"] = b
            stages[k]["hbm_gbs"] = b * n / (t * 1e-3) / 1e9
    eng.set_timing(True)
    eng.pair_kernel_ms(reset=True)
    for _ in range(steps):
        flush.zero_()
        eng.compute()
    pair_ms, _ = eng.pair_kernel_ms(reset=True)
    eng.set_timing(False)
    fa = eng.forces()
    ea = eng.energies()
    eng.close()
    e64 = nb.Engine(s, precision=0, device=dev)
    e64.set_stream(stream.cuda_stream)
    e64.build()
    e64.compute()
    fb = e64.forces()
    eb = e64.energies()
    e64.close()
    num = sum(((u - v) ** 2).sum() for u, v in zip(fa, fb))
    den = sum((v ** 2).sum() for v in fb)
    tot_a = ea["elec_direct"] + ea["elec_corr"] + ea["vdw"]
    tot_b = eb["elec_direct"] + eb["elec_corr"] + eb["vdw"]
    t_step = sum(ms) / len(ms)
    t_build = sum(ms_build) / len(ms_build)
    return {
        "workload": "999,999-atom rigid water box (333,333 molecules, 215 A cube)",
        "n_atoms": n, "in_cutoff_pairs": pairs, "cluster_pairs": stats[1],
        "ms_per_step": t_step, "pairs_per_s": pairs / (t_step * 1e-3),
        "pair_kernel": {"ms": pair_ms, "pairs_per_s": pairs / (pair_ms * 1e-3)},
        "list_build": {"ms": t_build,
                       "hbm_gbs": LIST_BYTES_PER_ATOM * n / (t_build * 1e-3) / 1e9,
                       "bytes_per_atom": LIST_BYTES_PER_ATOM, "stages": stages,
                       "stage_peak_gbs": hbm_peak()},
        "force_rel_rms_vs_fp64_form": float(np.sqrt(num / den)),
        "energy_rel_vs_fp64_form": abs(tot_a - tot_b) / abs(tot_b),
        "fp64_form_pairs": int(eb["n_pairs"]),
        "l2": "flushed before every timed step (256 MiB write)"}


def replicas_measure(torch, nb, systems, dev, stream, flush, seed, steps, world):
    """64 independent water boxes (1,500-30,000 atoms, log-uniform) in one
    engine: autotuned pair kernel, aggregate pairs/s of the build + force
    step, a `steps`-step velocity-Verlet loop captured as one CUDA graph
    (rigid water, rebuilds on half-skin displacement), and each replica's
    force error against the plain FP64 form."""
    import numpy as np

    from mdbas_b200 import ranks
    # with N ranks each takes a size-balanced share of the 64 boxes
    rank = int(os.environ.get("RANK", "0"))
    share = ranks.shard_sizes(systems.replica_sizes(64, seed=seed), world)[rank]
    batch = systems.config_replicas(64, seed=seed, temperature=300.0, subset=share)
    parts_n = [k for _, k in batch.meta["replicas"]]
    eng = nb.Engine(batch, precision=1, device=dev)
    eng.set_stream(stream.cuda_stream)
    eng.build()
    tune = eng.autotune()
    eng.compute()
    torch.cuda.synchronize()
    pairs = int(eng.energies()["n_pairs"])
    fb = eng.forces()

    def step():
        eng.build()
        eng.compute()

    for _ in range(3):
        step()
    ms = _time_steps(torch, eng, stream, flush, 10, step)
    eng.set_timing(True)
    eng.pair_kernel_ms(reset=True)
    for _ in range(10):
        flush.zero_()
        eng.compute()
    pair_ms, _ = eng.pair_kernel_ms(reset=True)
    eng.set_timing(False)
    # per-replica error against the FP64 form
    errs = []
    for r, got in enumerate(nb.Engine.split_arrays(fb, batch)):
        sub = systems.replica(batch, r)
        ref = nb.Engine(sub, precision=0, device=dev)
        ref.build()
        ref.compute()
        fr = ref.forces()
        ref.close()
        num = sum(((a - b) ** 2).sum() for a, b in zip(got, fr))
        den = sum((b ** 2).sum() for b in fr)
        errs.append(float(np.sqrt(num / den)))
    # dynamics: relax, then `steps` NVE steps as one graph launch
    cons = batch.water_constraints()
    eng.md_set_graph(20)
    eng.md_init(batch.mass, (batch.vx, batch.vy, batch.vz), time_step=0.0005, list_update=0,
                constraints=cons)
    eng.md_run(1000, target_temp=300.0, tau_t=0.05)
    pos, vel = eng.positions(), eng.velocities()
    eng.set_positions(*pos)
    eng.md_set_graph(steps)
    eng.md_init(batch.mass, vel, time_step=0.001, list_update=0, constraints=cons)
    eng.md_run(steps)                       # captures the graph
    st0 = eng.md_stats()
    l0 = eng.launches()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.md_run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    md_ms = e0.elapsed_time(e1) / steps
    st1 = eng.md_stats()
    launches = eng.launches() - l0
    eng.close()
    dv = "cuda" if world > 1 else "cpu"
    total_pairs, t_step, rate = ranks.job_rate(pairs, sum(ms) / len(ms), dv)
    md_ms = ranks.max_over_ranks([md_ms], dv)[0]
    pair_ms = ranks.max_over_ranks([pair_ms], dv)[0]
    err_max = ranks.max_over_ranks([max(errs)], dv)[0]
    n_atoms = int(ranks.sum_over_ranks([batch.n], dv)[0])
    return {
        "workload": "64 water boxes, 1,500-30,000 atoms (seeded log-uniform), one engine per "
                    "GPU holding its size-balanced share",
        "n_atoms": n_atoms, "replicas_on_rank0": len(share),
        "replica_atoms_min_max": [min(parts_n), max(parts_n)],
        "in_cutoff_pairs": int(total_pairs), "autotune": tune,
        "ms_per_step": t_step, "pairs_per_s": rate,
        "pair_kernel": {"ms": pair_ms, "pairs_per_s": total_pairs / (pair_ms * 1e-3)},
        "force_rel_rms_vs_fp64_form": {"max": err_max, "mean_rank0": float(np.mean(errs))},
        "md": {"steps_per_graph_launch": steps, "ms_per_step": md_ms,
               "pairs_per_s": total_pairs / (md_ms * 1e-3),
               "aggregate_ns_per_day": 64 * 86400.0 / (md_ms * 1e-3) * 1e-6,
               "list_builds": st1["rebuilds"] - st0["rebuilds"],
               "kernel_launches_per_step": launches / steps}}


def spme_measure(torch, nb, systems, dev, stream, seed, steps):
    """Reciprocal space of the 96k water box by the GPU SPME with MDBas's grid
    rule (init_spme, ewald prec 1e-6, alpha 0.34) and B-spline order 8."""
    import ctypes as C
    s = systems.config_96k(seed=seed, temperature=None)
    L = nb.lib()
    ctrl, param, ew = nb.CTRL(), nb.make_param(s.n), nb.EWALD()
    pbc = nb.make_pbc(s.cell())
    ctrl.keyAlpha = 1
    ew.alpha, ew.prec, ew.nbsp = 0.34, 1e-6, 8
    L.init_spme.argtypes = [C.c_void_p] * 4
    L.init_spme(C.byref(ctrl), C.byref(param), C.byref(ew), C.byref(pbc))
    grid = (ew.m1max, ew.m2max, ew.m3max)
    xyzq = [torch.tensor(a, device="cuda", dtype=torch.float64) for a in (s.x, s.y, s.z, s.q)]
    f = torch.zeros(3, s.n, device="cuda", dtype=torch.float64)
    out = (C.c_double * 8)()

    def call():
        nb.check(L.mdbas_nb_spme(s.n, C.byref(pbc), 0.34, systems.CHARGE_CONST, *grid, 8,
                                 *(C.c_void_p(a.data_ptr()) for a in xyzq),
                                 *(C.c_void_p(f[k].data_ptr()) for k in range(3)), out, 1,
                                 C.c_void_p(stream.cuda_stream)), "spme")

    for _ in range(2):
        call()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    return {"grid": list(grid), "order": 8, "ms": e0.elapsed_time(e1) / steps,
            "energy_kcal_mol": out[0] / 418.4,
            "note": "reciprocal space of the 96k box (not part of the real-space step)"}


def run_ours(args, rank, world):
    import numpy as np
    import torch
    import torch.distributed as dist

    from mdbas_b200 import nb, ranks, systems

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = local
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    s = systems.config_96k(seed=ranks.rank_seed(args.seed, rank), temperature=None)
    eng = nb.Engine(s, precision=1, device=dev)
    eng.set_stream(stream.cuda_stream)
    eng64 = nb.Engine(s, precision=0, device=dev)
    eng64.set_stream(stream.cuda_stream)

    def step32():
        eng.build()
        eng.compute()

    def step64():
        eng64.build()
        eng64.compute()

    for _ in range(max(3, args.warmup)):
        step32()
    step64()
    torch.cuda.synchronize()
    e = eng.energies()
    pairs = int(e["n_pairs"])
    stats = eng.list_stats()

    # ---- timed region (FP32 + fixed point) --------------------------------
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    launches0 = eng.launches()
    ms = _time_steps(torch, eng, stream, flush, args.steps, step32)
    launches = eng.launches() - launches0
    clk = clocks.stop()
    torch.cuda.synchronize()
    dv = "cuda" if world > 1 else "cpu"
    total_pairs, t_step, _ = ranks.job_rate(pairs, sum(ms) / len(ms), dv)
    if world > 1:
        dist.barrier()
    value = total_pairs / (t_step * 1e-3)

    # the same step with an event between the list build and the force
    # evaluation: a decomposition of the step that adds up to it
    parts = _time_split_steps(torch, stream, flush, args.steps, eng.build, eng.compute)
    step_parts = {"list_build_ms": statistics.mean(p[0] for p in parts),
                  "forces_ms": statistics.mean(p[1] for p in parts),
                  "what": "one build + one force evaluation per step, events between them "
                          "(L2 flushed before each step); the two add up to the step"}

    # ---- pair kernel alone (CUDA events on the launching stream) ----------
    eng.set_timing(True)
    eng.pair_kernel_ms(reset=True)
    for _ in range(args.steps):
        flush.zero_()
        eng.compute()
    pair_ms, _ = eng.pair_kernel_ms(reset=True)
    # the other variants of the same kernel, for comparison
    other_ms = {}
    for v, name in ((4, "half_8x4"), (6, "quad_4x4"), (5, "half_8x4_80reg"), (2, "packed_8x8"),
                    (0, "scalar_dense_8x8"), (1, "compacted_8x8")):
        eng.set_variant(v)
        for _ in range(args.steps):
            flush.zero_()
            eng.compute()
        other_ms[name], _ = eng.pair_kernel_ms(reset=True)
    eng.set_variant(7)
    eng.set_timing(False)
    # list build alone
    ms_build = _time_steps(torch, eng, stream, flush, args.steps, eng.build)
    t_build = sum(ms_build) / len(ms_build)

    # ---- plain FP64 form, same step ---------------------------------------
    ms64 = _time_steps(torch, eng64, stream, flush, args.steps, step64)
    t64 = sum(ms64) / len(ms64)
    eng64.set_timing(True)
    eng64.pair_kernel_ms(reset=True)
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        eng64.compute()
    pair64_ms, _ = eng64.pair_kernel_ms(reset=True)
    eng64.set_timing(False)

    # ---- e2e through the C ABI with pinned host buffers -------------------
    n = s.n
    hx = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hy = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hz = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    fx = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    fy = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    fz = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hx[:], hy[:], hz[:] = s.x, s.y, s.z

    def step_e2e():
        # one C-ABI call: positions H2D, list build, forces, forces D2H and
        # the energy words, one wait
        eng.evaluate(hx, hy, hz, fx, fy, fz, rebuild=True)

    for _ in range(2):
        step_e2e()
    ms_e2e = _time_steps(torch, eng, stream, flush, args.steps, step_e2e)
    t_e2e = ranks.max_over_ranks([sum(ms_e2e) / len(ms_e2e)], dv)[0]
    e2e_value = total_pairs / (t_e2e * 1e-3)

    # ---- roofline of the pair kernel ---------------------------------------
    peaks = fp32_peaks(dev)
    peak = max(peaks)
    achieved = FLOPS_PER_PAIR * pairs / (pair_ms * 1e-3) / 1e12
    traffic = None
    prof = os.path.join(ROOT, "profiles", "pair_half_lean_96k_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None

    # ---- precision vs the FP64 form over seeds ------------------------------
    prec = None
    if rank == 0 and args.precision_seeds > 0:
        errs, eerr = [], []
        for sd in range(args.precision_seeds):
            sp = systems.config_96k(seed=sd, temperature=None)
            a = nb.Engine(sp, precision=1, device=dev)
            b = nb.Engine(sp, precision=0, device=dev)
            for x in (a, b):
                x.build()
                x.compute()
            fa, fb = a.forces(), b.forces()
            num = sum(((u - v) ** 2).sum() for u, v in zip(fa, fb))
            den = sum((v ** 2).sum() for v in fb)
            errs.append(math.sqrt(num / den))
            ea, eb = a.energies(), b.energies()
            tot_a = ea["elec_direct"] + ea["elec_corr"] + ea["vdw"]
            tot_b = eb["elec_direct"] + eb["elec_corr"] + eb["vdw"]
            eerr.append(abs(tot_a - tot_b) / abs(tot_b))
            a.close()
            b.close()
        prec = {"force_rel_rms_max": max(errs), "force_rel_rms_mean": statistics.mean(errs),
                "energy_rel_max": max(eerr), "seeds": args.precision_seeds,
                "against": "plain FP64 GPU form (itself within 1e-12 of MDBas)"}

    # ---- velocity-Verlet dynamics: ns/day, mixed and FP64 forms -----------
    md = md64 = None
    if args.md_steps > 0:
        md = md_measure(torch, nb, systems, dev, stream, args.seed + rank, 1, args.md_steps,
                        args.nve_steps, world)
        md64 = md_measure(torch, nb, systems, dev, stream, args.seed + rank, 0,
                          max(50, args.md_steps // 5), 0, world)
    # full electrostatics: SPME (MDBas's grid rule at prec 1e-6: 128^3, order
    # 8) in every step of the same dynamics
    md_pme = None
    if args.pme_steps > 0:
        md_pme = md_measure(torch, nb, systems, dev, stream, args.seed + rank, 1, args.pme_steps,
                            0, world, kspace=(2, (128, 128, 128), 8))
        md_pme["kspace"] = "SPME 128^3, B-spline order 8, every step, inside the step graph"

    spme = spme_measure(torch, nb, systems, dev, stream, args.seed + rank, 5)

    large = None
    if args.large_steps > 0:
        large = large_box_measure(torch, nb, systems, dev, stream, flush, args.seed + rank,
                                  args.large_steps)

    replicas = None
    if args.replica_steps > 0:
        # one 64-box job shared by all ranks: the same seed everywhere
        replicas = replicas_measure(torch, nb, systems, dev, stream, flush, args.seed,
                                    args.replica_steps, world)

    cpu = None
    list_parity = None
    list_parity64 = vs_mdbas = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        def _engine_at(x, y, z, precision):
            sw = systems.config_96k(seed=args.seed, temperature=None)
            sw.x, sw.y, sw.z = x, y, z
            e0 = nb.Engine(sw, precision=precision, device=dev)
            e0.build()
            return e0

        def gpu_list(x, y, z):
            e0 = _engine_at(x, y, z, 1)
            p = e0.export_pairs(1e30)  # every pair of the list masks
            e0.close()
            return p

        def gpu_list64(x, y, z):
            e0 = _engine_at(x, y, z, 0)
            p = e0.export_pairs(1e30)
            e0.close()
            return p

        def gpu_forces(x, y, z):
            e0 = _engine_at(x, y, z, 1)
            e0.compute()
            f, en = e0.forces(), e0.energies()
            e0.close()
            return f, en

        cpu = cpu_baseline_sample(args.seed, gpu_list, gpu_list64, gpu_forces)
        list_parity = cpu.pop("list_parity", None)
        list_parity64 = cpu.pop("list_parity_fp64_form", None)
        vs_mdbas = cpu.pop("vs_mdbas", None)
        # the other configurations against MDBas, as checks beside the baseline
        if vs_mdbas is not None:
            vs_mdbas = {"water_96k_seed%d" % args.seed: vs_mdbas,
                        **mdbas_errors(nb, systems, dev)}

    dropin = None
    if rank == 0 and args.dropin_steps > 0:
        dropin = dropin_e2e(nb, systems, args.seed, args.dropin_steps)
        for k in ("energy_mixed_ms", "plugin_mixed_ms", "plugin_fp64_caller_list_ms"):
            if dropin.get(k):
                dropin[k.replace("_ms", "_pairs_per_s")] = pairs / (dropin[k] * 1e-3)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair arithmetic, int64 fixed-point accumulation, fp64 positions",
            "data": "synthetic (seeded lattice-plus-jitter water generator)",
            "config": {"workload": WORKLOAD, "n_atoms": n, "in_cutoff_pairs": pairs,
                       "clusters": stats[0], "cluster_pairs": stats[1],
                       "pair_efficiency": pairs / max(1, stats[2]),
                       "step": "cluster-pair list build + forces/energy/virial",
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"replicas x{world}"},
            "ns_per_day": md["ns_per_day"] if md else None,
            "md": md,
            "md_fp64_form": md64,
            "md_pme": md_pme,
            "large_box": large,
            "spme": spme,
            "replicas": replicas,
            "pair_kernel": {"ms": pair_ms, "pairs_per_s": pairs / (pair_ms * 1e-3),
                            "variant": "half clusters, lean form: 8-atom i x two 4-atom j "
                                       "halves per warp step, packed f32x2, exact inner list",
                            "other_variants_ms": other_ms},
            "step_parts": step_parts,
            "list_build": {"ms": t_build,
                           "hbm_gbs": LIST_BYTES_PER_ATOM * n / (t_build * 1e-3) / 1e9},
            "fp64_form": {"ms_per_step": t64, "pairs_per_s": pairs / (t64 * 1e-3),
                          "pair_kernel_ms": pair64_ms,
                          "pair_kernel_pairs_per_s": pairs / (pair64_ms * 1e-3)},
            "speedup_vs_fp64_form": {"step": t64 / t_step, "pair_kernel": pair64_ms / pair_ms},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured FMA probe, the larger of scalar FFMA and "
                                        "packed f32x2 FMA (mdbas_b200/peak/fp32_peak.cu)",
                         "peak_probe_tflops": {"ffma": peaks[0], "ffma2": peaks[1]},
                         "flops_per_pair": FLOPS_PER_PAIR, "kernel": "k_pair_half_lean",
                         # the same flops counted on every listed pair slot (8 x 8
                         # per cluster pair, in the cut-off or not); frac = this x
                         # the pair efficiency of the cluster list
                         "frac_of_listed_slots": achieved / peak / max(1e-30, pairs / max(1, stats[2]))},
            "precision": prec,
            "precision_vs_mdbas": vs_mdbas,
            "e2e_dropin": dropin,
            "e2e": {"value": e2e_value, "unit": "pairs/s", "ms_per_step": t_e2e,
                    "h2d_bytes_per_step": 3 * 8 * n,
                    # forces, the eight energy/flag words, the build's error word
                    "d2h_bytes_per_step": 3 * 8 * n + 8 * 8 + 8,
                    "call": "mdbas_nb_engine_evaluate (host arrays, one call per step)"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
            "list_parity": list_parity,
            "list_parity_fp64_form": list_parity64,
        }
        print(json.dumps(line))
    eng.close()
    eng64.close()


def run_slab(args, rank, world):
    """The 999,999-atom box decomposed into ``world`` slabs along x
    (mdbas_b200/slab.py): per step the forward exchange of the halo
    positions (NCCL point-to-point on device tensors), the local cluster
    build and force evaluation of owned + halo atoms, and the reverse
    exchange of the halo forces.  With one rank the box exchanges its halo
    with itself.  value = the box's in-cut-off pairs per second of the
    slowest rank's device time (strong scaling: the box is fixed)."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from mdbas_b200 import nb, ranks, slab, systems

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    s = systems.config_1m(seed=args.seed)
    geom = slab.SlabGeometry((s.box,) * 3, world, 14.0)
    owned = slab.partition(geom, s.x)[rank]
    backend = slab.EngineBackend(precision=1, device=local)
    run = slab.SlabRunner(geom, rank, slab.Topology.of(s), backend, device=dev)
    x = torch.as_tensor(s.x[owned], device=dev)
    y = torch.as_tensor(s.y[owned], device=dev)
    z = torch.as_tensor(s.z[owned], device=dev)
    run.repartition(owned, x, y, z)
    out = {}

    def step():
        out["r"] = run.step(x, y, z)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = backend.eng.launches()
    ms = _time_steps(torch, backend.eng, stream, flush, args.steps, step)
    launches = backend.eng.launches() - launches0
    t_step = ranks.max_over_ranks([sum(ms) / len(ms)], dev)[0]
    e = out["r"][3]
    pairs = int(e["n_pairs"])
    # the same box in one periodic domain on this GPU: forces of this rank's
    # atoms against the slab path's
    ref = nb.Engine(s, precision=1, device=local)
    ref.build()
    ref.compute()
    rf = [a[owned] for a in ref.forces()]
    re_ = ref.energies()
    ref.close()
    fx, fy, fz = (t.cpu().numpy() for t in out["r"][:3])
    num = ((fx - rf[0]) ** 2 + (fy - rf[1]) ** 2 + (fz - rf[2]) ** 2).sum()
    den = (rf[0] ** 2 + rf[1] ** 2 + rf[2] ** 2).sum()
    num, den = ranks.sum_over_ranks([num, den], dev)
    if rank == 0:
        line = {
            "metric": METRIC, "value": pairs / (t_step * 1e-3), "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": t_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None,
            "dtype": "fp32 pair arithmetic, int64 fixed-point accumulation, fp64 positions",
            "data": "synthetic (seeded lattice-plus-jitter water generator)",
            "config": {"workload": "999,999-atom rigid water box (215 A cube), slab "
                                   f"decomposition along x over {world} rank(s), halo 14 A",
                       "n_atoms": s.n, "in_cutoff_pairs": pairs,
                       "owned_atoms_rank0": int(len(owned)),
                       "halo_atoms_rank0": int(run.n_halo),
                       "step": "halo exchange + cluster build + forces/energy/virial + "
                               "reverse force exchange",
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"slab x{world}"},
            "force_rel_rms_vs_single_domain": math.sqrt(num / den),
            "pairs_single_domain": int(re_["n_pairs"]),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line))
    backend.close()


def run_case(args):
    from mdbas_b200 import nb, systems
    if args.case == "pair":
        s = systems.config_96k(seed=args.seed, temperature=None)
        e = nb.Engine(s, precision=1)
        e.set_variant(args.variant)
        e.build()
        for _ in range(4):
            e.compute()
        print(json.dumps({"case": "pair", "variant": args.variant,
                          "pairs": e.energies()["n_pairs"], "list": e.list_stats()}))
    elif args.case == "pair1m":
        # the 999,999-atom box: one list build, two force evaluations (for a
        # profiler capture of the pair kernel at full size)
        s = systems.config_1m(seed=args.seed)
        e = nb.Engine(s, precision=1)
        e.set_variant(args.variant)
        e.build()
        for _ in range(2):
            e.compute()
        print(json.dumps({"case": "pair1m", "variant": args.variant,
                          "pairs": e.energies()["n_pairs"], "list": e.list_stats()}))
    elif args.case == "build1m":
        # the 999,999-atom box: three list builds (for a profiler capture of
        # the build kernels at full size)
        s = systems.config_1m(seed=args.seed)
        e = nb.Engine(s, precision=1)
        for _ in range(3):
            e.build()
        print(json.dumps({"case": "build1m", "list": e.list_stats()}))
    else:
        s = systems.config_96k(seed=args.seed, temperature=300.0)
        e = nb.Engine(s, precision=1)
        e.md_set_graph(0)
        e.md_init(s.mass, (s.vx, s.vy, s.vz), time_step=0.0005, list_update=0,
                  constraints=s.water_constraints())
        e.md_run(args.md_steps)
        print(json.dumps({"case": "md", "steps": args.md_steps, "stats": e.md_stats()}))
    e.close()


def main():
    args = _parse()
    if args.case:
        run_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.decomp == "slab":
            run_slab(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
