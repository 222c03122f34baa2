#!/usr/bin/env python
"""Benchmark: I-V bias points/s of the n-MOSFET Id-Vg workload on B200.

Workload (the precision-path configuration): n-MOSFET on a 120x80x60 tensor mesh
(576,000 nodes), p-body 1e17 cm^-3, Gaussian n+ source / drain (1e20 cm^-3, sigma 20 nm),
2 nm SiO2 gate oxide as an oxide Robin face gate, velocity-saturated mobility; gate
swept 0..1.2 V in 0.05 V steps (25 points) at Vd = 0.05 V and 1.0 V.  Synthetic device
data built by semiconductor_devices_simulator_b200/devices.py (no dataset involved).

A step is the workload's two Id-Vg sweeps (24 resolved bias points each after the first,
which api3_solve solves) through the library's C ABI (api3_set_contact_V + api3_resolve
per point, the way main.py's run_sweep drives it), the two sweeps solved concurrently by
two solver instances (api3b_new / api3b_use), each on its own host thread and CUDA
stream.  The solver runs refined (FP32 Krylov / multigrid inner solves inside FP64
iterative refinement, api3b_set_precision(1)); the plain FP64 GPU path is timed on the
same steps beside it, and the refined currents are compared with the FP64 ones and with
the reference core's.  Bias points/s = converged points / time of the step (the slower stream's
CUDA-event time);
device set-up and the equilibrium + ramp to the first point (api3_solve) are outside
the timed region, as the metric defines.  `value` reads only the terminal currents per
point (state resident in HBM); `e2e` also copies psi, n and p of every point to host
buffers (api3_bulk_copy), the per-point results a caller reads.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload nmosfet|finfet|graph_mosfet|diodes64]

`--workload finfet`: the tri-gate FinFET Id-Vg family instead (96x96x64 tensor mesh, fin
10 nm wide x 40 nm tall wrapped by 1.5 nm SiO2 and three gate electrodes driven together,
gate 0..1.0 V in 0.02 V steps at 5 drain biases, one instance and stream per drain bias),
with the same refined / FP64 / learned-seed / reference-core measurements.
`--workload graph_mosfet`: the n-MOSFET's 120x80x60 mesh given as a general (graph) mesh,
solved by the graph path (ELL kernels, aggregation multigrid, FP64), the reference's own
graph path timed beside it.

Multi-GPU (torchrun, one rank per GPU): every rank solves its own sweeps (independent
devices, no data-path collective): weak scaling, time = max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from semiconductor_devices_simulator_b200 import abi, devices as D  # noqa: E402

METRIC = "I-V bias points/s on 1 B200 (refined+batched+learned vs plain FP64), dI/I<=1e-4"
UNIT = "bias points/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mesh", default=None, help="Nx,Ny,Nz (default: the workload's mesh)")
    ap.add_argument("--precision", default="refined", choices=["refined", "fp64"],
                    help="linear solves: FP32 refined in FP64 (default) or FP64 throughout")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison steps")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-predictor step")
    ap.add_argument("--no-tight", action="store_true", help="skip the tight-tolerance refined-vs-FP64 check")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64 pn-diode variants sub-block")
    ap.add_argument("--points", type=int, default=0,
                    help="points per sweep timed in a step (0: every point)")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes (no autotuner)")
    ap.add_argument("--predictor", default=None, choices=["quadratic", "secant"],
                    help="sweep predictor of the timed steps: quadratic through the last three points or the "
                         "reference's secant step (default: quadratic, secant for the FinFET, whose on-state "
                         "currents move by 1.7e-4 with the start at its production tolerances); the other one "
                         "is timed on one more step")
    ap.add_argument("--share", default="gummel", choices=["gummel", "none"],
                    help="grid shares of concurrently solved sweeps: by the first step's Gummel iterations, "
                         "or none (every persistent solve takes the whole GPU)")
    ap.add_argument("--workload", default="nmosfet", choices=["nmosfet", "finfet", "graph_mosfet", "diodes64", "power_cell"],
                    help="nmosfet: the Id-Vg workload (default); finfet: the tri-gate FinFET Id-Vg family "
                         "(96x96x64, 5 drain biases); diodes64: the 64 pn-diode variants batch")
    ap.add_argument("--batch-solves", default="per-pass", choices=["per-pass", "persistent"],
                    help="diodes64: linear solves as per-pass graphs (default: 64 concurrent instances overlap "
                         "their small launches better, 120 against 99 points/s) or persistent launches with "
                         "grid shares by node count")
    ap.add_argument("--workers", type=int, default=0, help="diodes64: concurrent host threads (0: one per variant)")
    ap.add_argument("--variants", type=int, default=0, help="diodes64: only the first n variants (0: all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="bounded CPU-baseline sample (s)")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the e2e pass (profiler captures)")
    ap.add_argument("--trace", action="store_true", help="with --probe: barrier timeline of the persistent solve")
    ap.add_argument("--probe", type=int, default=0, metavar="ITS",
                    help="profiler probe: one continuity system of the workload device at its charge-neutral "
                         "start, multigrid set-up and ITS BiCGSTAB iterations (a few hundred launches)")
    return ap.parse_args()


def run_probe(a):
    """Few-launch case for ncu: the workload's device, one electron continuity system
    (multigrid set-up and `ITS` BiCGSTAB iterations), then one learned-seed pass."""
    import semiconductor_devices_simulator_b200 as S
    mesh = mesh_of(a)
    lib = S.load()
    w = build(lib, mesh)
    lib.api3b_set_precision(1 if a.precision == "refined" else 0)
    s = w.sweeps[-1]
    for cid, vv in D.bias_vector(w, s, 0.6).items():
        lib.api3_set_contact_V(cid, vv)
    assert lib.b200x_prepare() == 1
    lib.b200x_init_state()
    l0 = lib.b200x_launches()
    lib.b200x_cont_assemble(0, None, None, None, None)
    rn, r0 = np.zeros(1), np.zeros(1)
    lib.b200x_stream_timer(0)
    its = lib.b200x_bicgstab(a.probe, 1e-12, 0.0, 1, None, None, abi.dptr(rn), abi.dptr(r0))
    solve_ms = lib.b200x_stream_timer(1)
    lib.b200x_cont_assemble(0, None, None, None, None)      # the same solve again, warm
    nk = lib.b200x_prof(1)                                  # with its algorithmic bytes per class
    lib.b200x_stream_timer(0)
    lib.b200x_bicgstab(a.probe, 1e-12, 0.0, 1, None, None, abi.dptr(rn), abi.dptr(r0))
    solve_ms2 = lib.b200x_stream_timer(1)
    lib.b200x_prof(0)
    alg = {}
    for k in range(nk):
        ms, cnt, by = (np.zeros(1) for _ in range(3))
        lib.b200x_prof_read(k, abi.dptr(ms), abi.dptr(cnt), abi.dptr(by))
        if cnt[0] > 0:
            alg[lib.b200x_prof_name(k).decode()] = {"launches": int(cnt[0]), "bytes": float(by[0]),
                                                    "ms": round(float(ms[0]), 4)}
    timeline = None
    if a.trace:                                             # barrier timeline of one more (warm) solve
        nb = 4096
        lib.b200x_persist_trace(nb, None, None)
        lib.b200x_cont_assemble(0, None, None, None, None)
        lib.b200x_bicgstab(a.probe, 1e-12, 0.0, 1, None, None, abi.dptr(rn), abi.dptr(r0))
        buf = (ctypes.c_ulonglong * (3 * nb))()
        blocks = ctypes.c_int(0)
        if lib.b200x_persist_trace(0, buf, ctypes.byref(blocks)) == 1:
            t = np.frombuffer(buf, dtype=np.uint64).reshape(nb, 3).astype(np.float64)
            used = t[:, 2] > 0
            t = t[used]
            t0 = t[0, 0]
            first, last, rel = (t[:, 0] - t0) / 1e3, (t[:, 1] - t0) / 1e3, (t[:, 2] - t0) / 1e3
            work = last - np.concatenate([[0.0], rel[:-1]])        # previous release -> last arrival
            wait = rel - last                                       # last arrival -> release
            skew = last - first
            timeline = {"blocks": blocks.value, "barriers": int(len(t)), "total_us": round(float(rel[-1]), 1),
                        "work_us": {"mean": round(float(work.mean()), 3), "median": round(float(np.median(work)), 3),
                                    "sum": round(float(work.sum()), 1)},
                        "release_us": {"mean": round(float(wait.mean()), 3), "median": round(float(np.median(wait)), 3),
                                       "sum": round(float(wait.sum()), 1)},
                        "arrival_skew_us": {"mean": round(float(skew.mean()), 3)},
                        "first_barriers": [[round(float(x), 2) for x in (work[q], skew[q], wait[q])]
                                           for q in range(min(120, len(t)))]}
    # one pass of the learned predictor's seed kernel (untrained weights) on the same device
    from semiconductor_devices_simulator_b200 import learned as LR
    LR.load(lib, LR.init_params(lib.api3b_seed_nparam(), seed=0, out_scale=1.0))
    lib.api3b_seed_enable(0)
    dv = np.array([0.0, 0.0, 0.05, 0.0])
    seed_ok = lib.b200x_seed_run(1.0, abi.dptr(dv))
    lib.b200x_stream_timer(0)
    for _ in range(10):
        lib.b200x_seed_run(1.0, abi.dptr(dv))
    seed_ms = lib.b200x_stream_timer(1) / 10
    print(json.dumps({"probe": f"{WL}_{mesh[0]}x{mesh[1]}x{mesh[2]} electron continuity", "nodes": w.N,
                      "precision": a.precision, "seed_kernel": seed_ok, "seed_ms": round(seed_ms, 4),
                      "bicgstab_its": its, "r0": r0[0], "rn": rn[0], "solve_ms": [round(solve_ms, 3), round(solve_ms2, 3)],
                      "persistent": bool(lib.api3b_set_persist(-1, -1)), "timeline": timeline,
                      "warm_solve_classes": alg,
                      "launches": int(lib.b200x_launches() - l0)}))


# ------------------------------------------------------------------ distributed plumbing
class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist, self.torch, self.backend = dist, torch, backend

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64,
                              device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self.world == 1:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64,
                              device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj):
        """Every rank's `obj` as a list on rank 0 (None on the other ranks)."""
        if self.world == 1:
            return [obj]
        objs = [None] * self.world
        self.dist.all_gather_object(objs, obj)
        return objs if self.rank == 0 else None

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def shard(items, rank, world, weights=None):
    """The units of `items` rank `rank` of `world` takes: every unit exactly once, balanced
    by `weights` (the units' node counts: a solve's cost grows with them) - the largest
    unit first, each to the rank with the least weight so far (ties to the lower rank).
    Equal weights give a round robin."""
    items = list(items)
    wts = [1.0] * len(items) if weights is None else [float(x) for x in weights]
    order = sorted(range(len(items)), key=lambda i: (-wts[i], i))
    load = [0.0] * world
    own = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        own[r].append(i)
        load[r] += wts[i]
    return [items[i] for i in sorted(own[rank])]


def sweep_order(nsw, rank, world, replicate):
    """The sweeps (drain biases) a rank solves: with `replicate` every rank solves the whole
    family (independent replicas, weak scaling), else the family is split across the ranks
    (each sweep on exactly one rank)."""
    if replicate:
        return [(q + rank) % nsw for q in range(nsw)]
    return shard(range(nsw), rank, world)


def gather_iv(dist, cur, nsw):
    """Gather every rank's terminal currents to rank 0: `cur` maps a sweep index to its
    points' (I per contact, Iflr per contact).  Returns, on rank 0, the family's array
    (sweeps x points x contacts x 2: I, Iflr) in sweep order and how many ranks solved each
    sweep; None elsewhere."""
    mine = {int(k): np.asarray([[I, F] for I, F in v], dtype=np.float64).transpose(0, 2, 1)
            for k, v in cur.items()}
    parts = dist.gather(mine)
    if parts is None:
        return None
    seen = [0] * nsw
    arr = None
    for part in parts:
        for k, a in part.items():
            seen[k] += 1
            if arr is None:
                arr = np.full((nsw,) + a.shape, np.nan)
            arr[k] = a
    return arr, seen


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.proc, self.rows = gpu, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ workload
# The Id-Vg workloads: the n-MOSFET (120x80x60, gate 0..1.2 V in 0.05 V steps at Vd = 0.05
# and 1.0 V) and the tri-gate FinFET (96x96x64, fin 10 x 40 nm, gate 0..1.0 V in 0.02 V
# steps at 5 drain biases).  Each drain bias is one sweep, solved by its own instance.
WORKLOADS = {
    "nmosfet": {"mesh": (120, 80, 60), "build": lambda lib, n: D.nmosfet(lib, n=n)},
    "finfet": {"mesh": (96, 96, 64), "build": lambda lib, n: D.finfet(lib, n=n)},
    # the large-device configuration: the vertical power cell (10 x 60 x 10 um, 8.4M nodes),
    # drain 0..50 V in 1 V steps at 16 gate biases (2.5..10 V), one instance per gate bias
    "power_cell": {"mesh": (256, 256, 128),
                   "build": lambda lib, n: D.power_cell(lib, n=n, vgs=tuple(np.round(np.arange(2.5, 10.01, 0.5), 6)))},
    # the n-MOSFET's device given as a general (graph) mesh: the graph path's ELL kernels and
    # aggregation multigrid (FP64; no launch-shape tuning or learned seed on graphs)
    "graph_mosfet": {"mesh": (120, 80, 60),
                     "build": lambda lib, n: D.graph_nmosfet(lib, n=n, models=4, vds=(0.05, 1.0), vg_max=1.2,
                                                             dvg=0.05, h0=0.5e-9)},
}
WL = "nmosfet"


def build(lib, mesh):
    return WORKLOADS[WL]["build"](lib, mesh)


def mesh_of(a):
    return tuple(int(v) for v in a.mesh.split(",")) if a.mesh else WORKLOADS[WL]["mesh"]


def workload_name(mesh):
    return f"{WL}_{mesh[0]}x{mesh[1]}x{mesh[2]}_idvg"


def workload_config(w):
    s = w.sweeps
    V = s[0]["V"]
    return {"drain_biases_V": [float(x["fixed"]["drain"]) for x in s],
            "gate_sweep_V": [float(V[0]), float(V[-1]), round(float(V[1] - V[0]), 6)],
            "models": int(w.info.get("models", 0))}


def sweep_points(lib, w, s, fields=False, npts=None, out=None):
    """Timed part of one step: every point of the sweep after the first (or the next
    npts); the first point is the one api3_solve already solved.  `out` collects the
    terminal currents and round-off floors of every point."""
    nc = lib.api3_get_ncon()
    V = s["V"][1:] if npts is None else s["V"][1:1 + npts]
    conv = 0
    bufs = [np.empty(w.N) for _ in range(3)] if fields else None
    for v in V:
        for cid, vv in D.bias_vector(w, s, v).items():
            lib.api3_set_contact_V(cid, vv)
        conv += int(lib.api3_resolve())
        I = [lib.api3_get_contact_I(c) for c in range(nc)]
        if out is not None:
            out.append((I, [lib.api3_get_contact_Ifloor(c) for c in range(nc)]))
        if fields:
            for q, which in enumerate((0, 1, 2)):
                lib.api3_bulk_copy(which, abi.dptr(bufs[q]))
    return len(V), conv


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte of a kernel
# class on the default 120x80x60 mesh, from one ncu capture of the bench's --probe 10 case:
# the persistent refined solve (k_persist<float, 2>, 10 BiCGSTAB iterations) moved 433.2 MB
# of DRAM traffic for 4516 MB of algorithmic bytes (its hierarchy stays resident in the L2)
NCU_DRAM_PER_ALG = {"persistent_solve_f32": 433.16e6 / 4516.1e6}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(mesh, seconds):
    """The reference core (oracle/_ref, built from the reference sources) on this
    host's cores: the same workload, a bounded sample of its highest-drain-bias sweep."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_ref.so")
    if not os.path.exists(path):
        return None
    ref = abi.bind(ctypes.CDLL(path))
    cores = os.cpu_count() or 1
    ref.api3_set_threads(cores)
    w = build(ref, mesh)
    s = w.sweeps[-1]
    D.start_sweep(ref, w, s)
    t0 = time.perf_counter()
    n = 0
    cur = []
    nc = ref.api3_get_ncon()
    for v in s["V"][1:]:
        for cid, vv in D.bias_vector(w, s, v).items():
            ref.api3_set_contact_V(cid, vv)
        ref.api3_resolve()
        cur.append(([ref.api3_get_contact_I(c) for c in range(nc)], [ref.api3_get_contact_Ifloor(c) for c in range(nc)]))
        n += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"first {n} resolves of the Vd={s['fixed']['drain']} V Id-Vg sweep of {WL}, "
                      f"{mesh[0]}x{mesh[1]}x{mesh[2]} mesh, "
                      f"reference core semiconductor_3d.c built from source (-O3 -fopenmp), {cores} threads, "
                      f"{dt:.1f} s"}, cur


class Sweeper:
    """One solver instance on its own host thread and CUDA stream, solving one sweep."""

    def __init__(self, lib, mesh, sweep_index, dev, precision, solver=None, npts=None):
        self.lib, self.mesh, self.si = lib, mesh, sweep_index
        self.npts_limit = npts
        self.h = lib.api3b_new()
        self.dev = dev
        self.w = None
        self.precision = precision
        self.solver = solver
        self.cur = []

    def free(self):
        self.lib.api3b_free(self.h)

    def _use(self):
        self.lib.api3b_use(self.h)
        self.lib.b200x_set_device(self.dev)

    def prepare(self):
        self._use()
        self.lib.api3b_set_precision(self.precision)
        if self.w is None:
            self.w = build(self.lib, self.mesh)
            self.lib.api3_set_verbose(0)
            if self.solver:
                self.lib.api3_set_solver(*self.solver)
        D.start_sweep(self.lib, self.w, self.w.sweeps[self.si])   # untimed: equilibrium + ramp

    def run(self, fields):
        self._use()
        self.lib.b200x_stream_timer(0)
        t0 = time.perf_counter()
        g0 = self.lib.api3_get_stat(3)
        self.cur = []
        self.npts, self.conv = sweep_points(self.lib, self.w, self.w.sweeps[self.si], fields=fields, out=self.cur,
                                            npts=self.npts_limit)
        self.gummel = self.lib.api3_get_stat(3) - g0
        self.dev_s = self.lib.b200x_stream_timer(1) / 1e3
        self.wall = time.perf_counter() - t0


def sm_count(dev):
    import torch
    return torch.cuda.get_device_properties(dev).multi_processor_count if torch.cuda.is_available() else 148


def balance_shares(lib, ws, nsm, on=True):
    """Split the GPU's co-resident blocks (one per SM) between concurrently solved sweeps in
    proportion to the Gummel iterations each took in its last step, so that every sweep's
    persistent solves run side by side with the others' (cooperative grids that together
    exceed the SMs take turns).  `on` False removes the shares.  Returns the shares."""
    if not on or len(ws) < 2:
        for w in ws:
            lib.api3b_use(w.h)
            lib.api3b_set_share(0)
        return [0] * len(ws)
    g = [max(1, getattr(w, "gummel", 1) or 1) for w in ws]
    lo = max(4, nsm // (4 * len(ws)))
    sh = [max(lo, int(nsm * x / sum(g))) for x in g]
    while sum(sh) > nsm and max(sh) > lo:                  # trim the largest to fit the SMs
        sh[sh.index(max(sh))] -= 1
    for w, b in zip(ws, sh):
        lib.api3b_use(w.h)
        lib.api3b_set_share(b)
    return sh


def concurrent(workers, fn):
    th = [threading.Thread(target=fn, args=(w,)) for w in workers]
    for t in th:
        t.start()
    for t in th:
        t.join()


def rel_dI(cur, ref, on=1e-30):
    """Largest |I - I_ref| / |I_ref| over the points both lists hold, on terminals whose
    reference current is above its own round-off floor and above `on` amperes."""
    worst = 0.0
    for (I, _), (Ir, Fr) in zip(cur, ref):
        for x, y, f in zip(I, Ir, Fr):
            if abs(y) > max(f, on):
                worst = max(worst, abs(x - y) / abs(y))
    return worst


def worst_terminal(cur, ref):
    """The terminal that sets rel_dI over a family {sweep: points}: its sweep, point and
    contact, the reference current and floor, and the distance in units of the band
    1e-4 |I_ref| + Iflr (at most 1 where the two agree to 1e-4 or to the round-off floor)."""
    best, band = None, 0.0
    for si in ref:
        for q, ((I, _), (Ir, Fr)) in enumerate(zip(cur[si], ref[si])):
            for c, (x, y, f) in enumerate(zip(I, Ir, Fr)):
                if abs(y) > f:
                    band = max(band, abs(x - y) / (1e-4 * abs(y) + f))
                    r = abs(x - y) / abs(y)
                    if best is None or r > best["rel"]:
                        best = {"sweep": si, "point": q, "contact": c, "I_ref": y, "Iflr": f, "dI": abs(x - y), "rel": r}
    return best, band


# tight tolerances: inner solves to round-off, validate.py's Gummel tolerances
TIGHT_ENV = {"SEMISIM_BRTOL": "1e-12", "SEMISIM_PCGRTOL": "1e-10"}
TIGHT_SOLVER = (2000, 1000, 500, 1e-12, 1e-9, 1.0, 1.0)


def tight_check(lib, workers, mesh):
    """The metric's accuracy clause on the workload's own sweeps: this rank's sweeps
    re-solved with both codes converged tightly, refined and FP64 (untimed); the refined
    currents' largest relative distance to the FP64 ones, over every point and every
    terminal above its round-off floor."""
    res = {}
    t0 = time.perf_counter()
    for p in (1, 0):
        old = {k: os.environ.get(k) for k in TIGHT_ENV}
        os.environ.update(TIGHT_ENV)                     # read by api3_init
        ws = [Sweeper(lib, mesh, s.si, s.dev, p, solver=TIGHT_SOLVER) for s in workers]
        try:
            concurrent(ws, lambda s: s.prepare())
        finally:
            for k, v in old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        concurrent(ws, lambda s: s.run(False))
        res[p] = {s.si: list(s.cur) for s in ws}
        conv = sum(s.conv for s in ws)
        npts = sum(s.npts for s in ws)
        for s in ws:
            s.free()
        if conv != npts:
            return {"error": f"{npts - conv} of {npts} points did not converge at tight tolerances (precision {p})"}
    worst, band = worst_terminal(res[1], res[0])
    return {"all_points": max(rel_dI(res[1][k], res[0][k]) for k in res[0]),
            "on_state_Id_gt_1nA": max(rel_dI(res[1][k], res[0][k], on=1e-9) for k in res[0]),
            "worst_terminal": worst, "max_dI_over_band": band,
            "points": sum(len(v) for v in res[0].values()), "seconds": round(time.perf_counter() - t0, 1),
            "solver": list(TIGHT_SOLVER), "env": TIGHT_ENV,
            "note": "refined vs FP64, both converged tightly, every point of the step, terminals above their "
                    "round-off floor"}


def gummel_floor(lib, workers):
    """The fewest Gummel iterations any starting guess can give one step: every point of
    this rank's sweeps solved once along the sweep (its converged state kept), then solved
    again starting from that converged state itself (api3_set_state at the point's bias,
    then api3_resolve, which runs the Gummel loop at the same bias until its acceptance test
    passes).  A learned seed can save at most (linear-guess iterations - this floor)."""
    tot = pts = 0
    for s in workers:
        s._use()
        s.prepare()
        w, sw = s.w, s.w.sweeps[s.si]
        N = w.N
        states = []
        for v in sw["V"][1:]:
            for cid, vv in D.bias_vector(w, sw, v).items():
                lib.api3_set_contact_V(cid, vv)
            lib.api3_resolve()
            st = [np.empty(N) for _ in range(3)]
            lib.api3_get_state(*(abi.dptr(x) for x in st))
            states.append(st)
        for v, st in zip(sw["V"][1:], states):
            for cid, vv in D.bias_vector(w, sw, v).items():
                lib.api3_set_contact_V(cid, vv)
            lib.api3_set_state(*(abi.dptr(x) for x in st))
            g0 = lib.api3_get_stat(3)
            lib.api3_resolve()
            tot += lib.api3_get_stat(3) - g0
            pts += 1
    return tot, pts


def learned_step(a, lib, workers, step, cur, gummel_per_step, dist, gummel_other=None, order=1):
    """Train the learned predictor on the workload device's own sweeps at gate voltages
    shifted by half a step (both drain biases), then run one step of the workload with
    it (it corrects the secant guess at the first continuation step of each point).
    Returns the measured block: Gummel iterations of one step with the headline predictor
    (`gummel_per_step`, of order `order`), with the other plain predictor
    (`gummel_other`), with the learned seed and from converged starts; points/s."""
    if not workers:                             # this rank holds no sweep: keep the collective steps
        dist.barrier()
        return None
    import torch
    from semiconductor_devices_simulator_b200 import learned as LR
    s0 = workers[0]
    s0._use()
    t0 = time.perf_counter()
    feats, targs = [], []
    for sw in s0.w.sweeps:
        s2 = dict(sw)
        s2["V"] = np.round(sw["V"] + 0.5 * (sw["V"][1] - sw["V"][0]), 12)
        Vs, Xs, ok = LR.collect(lib, s0.w, s2)
        f, t = LR.pair_data(lib, torch, Vs, Xs, per_pair=131072)
        feats.append(f)
        targs.append(t)
    t_data = time.perf_counter() - t0
    tr = LR.Trainer(lib, torch, batch=16384, seed=0)
    tr.fit(torch.cat(feats), torch.cat(targs), steps=6000, lr=1e-3, lr_end=1e-4)
    params = tr.params()
    for s in workers:                           # the workload's own points, as a held-out set
        s._use()
        s.prepare()
        LR.load(lib, params)
        lib.api3b_seed_enable(1)
    dist.barrier()
    t1 = time.perf_counter()
    concurrent(workers, lambda s: s.run(False))
    wall = time.perf_counter() - t1
    dev = max(s.dev_s for s in workers)
    pts = sum(s.npts for s in workers)
    used = []
    for s in workers:
        s._use()
        used.append(LR.stats(lib))
        lib.api3b_seed_enable(0)
    curl = {s.si: list(s.cur) for s in workers}
    floor, fpts = gummel_floor(lib, workers)
    return {"points_per_s": round(pts / dev, 4), "unit": UNIT,
            "gummel_iterations_per_step": {("quadratic_guess" if order == 2 else "secant_guess"): gummel_per_step,
                                           ("secant_guess" if order == 2 else "quadratic_guess"): gummel_other,
                                           "learned_guess": sum(s.gummel for s in workers),
                                           "converged_start_floor": int(floor)},
            "floor_note": f"Gummel iterations of the same {fpts} points when each starts from its own converged "
                          "solution (api3_set_state at its bias): the least any seed can reach under the "
                          "acceptance test",
            "seeded_steps": int(sum(u[0] for u in used)), "fallbacks": int(sum(u[1] for u in used)),
            "max_rel_dI_vs_headline_on_state": max(rel_dI(curl[k], cur[k], on=1e-9) for k in cur),
            "train": {"rows": int(sum(f.shape[0] for f in feats)), "steps": 6000, "seconds": round(tr.seconds, 2),
                      "data_seconds": round(t_data, 1)},
            "note": "not in `value`: the seed corrects the secant guess and saves no Gummel iterations "
                    "against it; the converged-start floor shows how many a perfect seed would save"}


def run_b200(a, dist):
    import semiconductor_devices_simulator_b200 as S
    mesh = mesh_of(a)
    lib = S.load()
    lib.b200x_set_device(dist.local)
    pred = a.predictor or ("secant" if WL == "finfet" else "quadratic")
    order = 2 if pred == "quadratic" else 1
    lib.api3b_set_pred_order(order)
    nsw = {"finfet": 5, "power_cell": 16}.get(WL, 2)   # the sweeps of the workload, one instance each
    graph = WL.startswith("graph")
    prec = 1 if a.precision == "refined" and not graph else 0
    # the n-MOSFET family is replicated on every GPU (independent characterisation jobs:
    # weak scaling); the FinFET's five drain-bias sweeps and the power cell's sixteen
    # gate-bias sweeps are split across the GPUs
    replicate = WL not in ("finfet", "power_cell")

    def make(p):
        return [Sweeper(lib, mesh, si, dist.local, p, npts=a.points or None)
                for si in sweep_order(nsw, dist.rank, dist.world, replicate)]
    workers = make(prec)

    def step(ws, fields=False):
        """The rank's sweeps, concurrently (one instance, thread and stream each)."""
        concurrent(ws, lambda s: s.prepare())
        dist.barrier()
        t0 = time.perf_counter()
        concurrent(ws, lambda s: s.run(fields))
        wall = time.perf_counter() - t0
        return (sum(s.npts for s in ws), sum(s.conv for s in ws), max([s.dev_s for s in ws] or [0.0]), wall)

    tune = None
    if not a.no_autotune and not graph:       # launch shapes, one instance at a time (untimed)
        for s in workers:
            s.prepare()
            us = lib.api3b_autotune(2)
        r, g, sm, zc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib.api3b_tune_get(ctypes.byref(r), ctypes.byref(g), ctypes.byref(sm), ctypes.byref(zc))
        tune = {"rows_per_block": r.value, "row_blocks_max": zc.value, "grid_cap": g.value,
                "small_level_nodes": sm.value or 2048, "vcycle_us": round(us, 2)}
    nsm = sm_count(dist.local)
    shares = []
    for i in range(a.warmup):
        step(workers)
        if i == 0:                            # grid shares from the first step's Gummel counts
            shares = balance_shares(lib, workers, nsm, on=a.share == "gummel")
    w = workers[0].w
    clocks = Clocks(dist.local)
    clocks.start()
    l0 = lib.b200x_launches()
    tot_pts = tot_conv = 0
    tot_dev = tot_wall = 0.0
    for i in range(a.steps):
        npts, conv, dev_s, wall = step(workers)
        tot_pts += npts; tot_conv += conv; tot_dev += dev_s; tot_wall += wall
    launches = int(lib.b200x_launches() - l0)
    clk = clocks.stop()
    cur = {s.si: list(s.cur) for s in workers}
    iv = gather_iv(dist, cur, nsw)            # the family's I-V arrays on rank 0
    # e2e: the same steps with every point's psi, n, p copied to host buffers
    e_pts = 0
    e_wall = 0.0
    for i in range(0 if a.no_e2e else a.steps):
        npts, conv, dev_s, wall = step(workers, fields=True)
        e_pts += npts; e_wall += wall
    if a.no_e2e:
        e_pts, e_wall = tot_pts, tot_wall
    # roofline: one more step with every launch timed by CUDA events on the solver stream
    prof = None
    if not a.no_profile and workers:          # event timing is per thread: one sweep alone,
        s0 = max(workers, key=lambda s: s.gummel)   # the step's longest (with its grid share)
        s0.prepare()
        nk = lib.b200x_prof(1)
        s0.run(False)
        lib.b200x_prof(0)
        rows = []
        for k in range(nk):
            ms, cnt, by = (np.zeros(1) for _ in range(3))
            lib.b200x_prof_read(k, abi.dptr(ms), abi.dptr(cnt), abi.dptr(by))
            rows.append((lib.b200x_prof_name(k).decode(), float(ms[0]), int(cnt[0]), float(by[0])))
        prof = rows
    gummel = sum(s.gummel for s in workers)
    # the FP64 GPU path on the same steps (own instances, one warm-up step): batched (both
    # sweeps at once, as above) and plain (one sweep after the other, one instance at a time)
    f64 = None
    if prec == 1 and not a.no_fp64:
        w64 = make(0)
        step(w64)
        balance_shares(lib, w64, nsm, on=a.share == "gummel")
        f_pts = s_pts = 0
        f_dev = s_dev = 0.0
        for i in range(a.steps):
            npts, conv, dev_s, wall = step(w64)
            f_pts += npts; f_dev += dev_s
        cur64 = {s.si: list(s.cur) for s in w64}
        per_rank = len(sweep_order(nsw, 0, dist.world, replicate))   # the most sweeps a rank holds
        balance_shares(lib, w64, nsm, on=False)                      # one at a time: the whole GPU
        lib.api3b_set_pred_order(1)                                  # and the reference's secant step
        for i in range(a.steps):
            for q in range(per_rank):
                if q < len(w64):
                    w64[q].prepare()
                dist.barrier()
                if q < len(w64):
                    w64[q].run(False)
                    s_pts += w64[q].npts; s_dev += w64[q].dev_s
        f64 = (dist.sum(f_pts), dist.max(f_dev), dist.max(max([rel_dI(cur[k], cur64[k]) for k in cur] or [0.0])),
               dist.sum(s_pts), dist.max(s_dev),
               dist.max(max([rel_dI(cur[k], cur64[k], on=1e-9) for k in cur] or [0.0])))
        for s in w64:
            s.free()
        lib.api3b_set_pred_order(order)
    # the other sweep predictor on one more step of the same instances (same grid shares)
    other = None
    if not graph:                             # every rank takes the step's collectives
        lib.api3b_set_pred_order(3 - order)
        npts, conv, dev_s, wall = step(workers)
        lib.api3b_set_pred_order(order)
        curo = {s.si: list(s.cur) for s in workers}
        band = worst_terminal(curo, cur)[1] if workers else 0.0
        other = {"predictor": "secant" if order == 2 else "quadratic",
                 "points_per_s": round(dist.sum(npts) / max(dist.max(dev_s), 1e-9), 4), "unit": UNIT,
                 "gummel_iterations_per_step": sum(s.gummel for s in workers),
                 "max_rel_dI_vs_headline": {
                     "all_points": dist.max(max([rel_dI(curo[k], cur[k]) for k in cur] or [0.0])),
                     "on_state_Id_gt_1nA": dist.max(max([rel_dI(curo[k], cur[k], on=1e-9) for k in cur] or [0.0])),
                     "max_dI_over_band": dist.max(band)}}
    # the learned predictor: trained (untimed) on this device's own solutions at gate
    # voltages half a step off the workload's, then one step of the workload seeded by it
    learned = None
    if not a.no_learned and not graph:
        learned = learned_step(a, lib, workers, step, cur, gummel, dist,
                               other["gummel_iterations_per_step"] if other else None, order)
    tight = None
    if prec == 1 and not a.no_fp64 and not a.no_tight and workers:
        tight = tight_check(lib, workers, mesh)
    # the batching configuration (64 pn-diode variants), measured in the same run
    batch = run_batch(a, dist) if WL == "nmosfet" and not a.no_batch else None
    T = dist.max(tot_dev)
    pts_all = dist.sum(tot_pts)
    e_T = dist.max(e_wall)
    e_all = dist.sum(e_pts)
    out = None
    if dist.rank == 0:
        hbm, pk_kind = peaks()
        roof = None
        kernels = None
        if prof and graph:                    # per-class byte counts are the tensor stencil's
            tot_ms = sum(r[1] for r in prof) or 1.0
            kernels = {r[0]: {"ms": round(r[1], 2), "share": round(r[1] / tot_ms, 4), "launches": r[2]}
                       for r in sorted(prof, key=lambda r: -r[1]) if r[2] > 0}
        elif prof:
            tot_ms = sum(r[1] for r in prof) or 1.0
            top = max(prof, key=lambda r: r[1])
            ach = top[3] / (top[1] / 1e3) / 1e9 if top[1] > 0 else 0.0
            ratio = NCU_DRAM_PER_ALG.get(top[0]) if (WL, mesh) == ("nmosfet", (120, 80, 60)) else None
            traffic = round(ratio * top[3] / max(top[2], 1)) if ratio else None
            roof = {"bound": "hbm", "kernel": top[0], "achieved": round(ach, 1), "peak": hbm,
                    "peak_kind": pk_kind, "unit": "GB/s", "frac": round(ach / hbm, 4), "traffic": traffic,
                    "launches": top[2], "avg_launch_us": round(1e3 * top[1] / max(top[2], 1), 2),
                    "bytes_per_launch": round(top[3] / max(top[2], 1)),
                    "traffic_source": ("ncu DRAM bytes per algorithmic byte of this class on the probe case, "
                                       "times this run's algorithmic bytes per launch") if traffic else None,
                    "note": ("one cooperative launch per linear solve: its multigrid hierarchy and Krylov vectors "
                             "stay in the 126 MB L2 (DRAM traffic about a tenth of the algorithmic bytes); "
                             "the time goes to the grid barriers between dependent passes")
                            if top[0].startswith("persistent") else None}
            kernels = {r[0]: {"ms": round(r[1], 2), "share": round(r[1] / tot_ms, 4), "launches": r[2],
                              "GBps": round(r[3] / (r[1] / 1e3) / 1e9, 1) if r[1] > 0 else 0.0}
                       for r in sorted(prof, key=lambda r: -r[1]) if r[2] > 0}
        h2d = 8 * 4 * len(w.contacts)                              # contact voltages per point
        d2h = 3 * 8 * w.N + 16 * len(w.contacts)                   # psi, n, p + currents per point
        npts_step = int(pts_all) // max(a.steps, 1)
        value = pts_all / T
        out = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": dist.world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * T / a.steps, 2),
            "higher_is_better": True, "scaling": "weak" if replicate else "strong", "vs_baseline": None,
            "dtype": "f32 inner solves refined in f64 (f64 residuals, physics, currents)" if prec else "f64",
            "data": "synthetic (device built from the workload definition)",
            "config": dict({"workload": workload_name(mesh),
                            "nodes": w.N, "points_per_step": npts_step}, **workload_config(w),
                           **{"solver": list(D.GUI_SOLVER), "precision": "fp64" if graph else a.precision,
                              "launch_shapes": tune,
                              "sweep_predictor": ("quadratic through the last three points"
                                                  if order == 2 else "secant (the reference's)"),
                              "linear_solves": ("persistent (one cooperative launch per solve)"
                                                if lib.api3b_set_persist(-1, -1) else "per-pass graphs"),
                              "grid_shares": shares or None,
                              "parallelism": (f"replicas{dist.world}, {nsw} concurrent sweeps per GPU "
                                              "(instance + stream each)") if replicate else
                                             (f"sweeps split over {dist.world} GPU(s) by node count, concurrent "
                                              "sweeps per GPU (instance + stream each)"),
                              "point_set": f"every point of the {nsw} sweeps after their first, each step",
                              "l2": f"state of {w.N} nodes (~{w.N * 760 / 1e9:.2f} GB) exceeds the 126 MB L2; "
                                    "no flush"}),
            "converged_points": tot_conv, "wall_s": round(tot_wall, 3),
            "e2e": {"value": round(e_all / e_T, 4), "unit": UNIT, "h2d_bytes_per_step": h2d * npts_step,
                    "d2h_bytes_per_step": d2h * npts_step},
            "gpu_launches": launches,
            "roofline": roof,
            "kernels": kernels,
            "clocks": clk,
        }
        if f64:
            out["plain_fp64"] = {"value": round(f64[3] / f64[4], 4), "unit": UNIT,
                                 "what": "FP64 solves, one sweep at a time (no concurrent instances), linear guess",
                                 "speedup": round(value / (f64[3] / f64[4]), 3)}
            out["fp64_batched"] = {"value": round(f64[0] / f64[1], 4), "unit": UNIT,
                                   "speedup": round(value / (f64[0] / f64[1]), 3)}
            out["max_rel_dI_vs_fp64"] = {"all_points": f64[2], "on_state_Id_gt_1nA": f64[5],
                                         "note": "both at the workload's default tolerances; terminals above "
                                                 "their round-off floor"}
        if iv is not None:
            arr, seen = iv
            out["iv_gather"] = {"shape": list(arr.shape), "layout": "sweeps x points x contacts x (I, Iflr)",
                                "solved_per_sweep": seen, "complete": bool(np.isfinite(arr).all())}
        if tight:
            out["max_rel_dI_vs_fp64_tight"] = tight
        if batch:
            out["diodes64"] = batch
        if other:
            out["other_predictor"] = other
        if learned:
            out["learned_seed"] = learned
        if dist.world == 1 and not a.no_cpu_baseline and WL != "power_cell":   # 8.4M nodes: hours on the host
            cb = cpu_baseline(mesh, a.cpu_seconds)
            if cb:
                cb, rcur = cb
                out["cpu_baseline"] = cb
                last = [(list(p[:, 0]), list(p[:, 1])) for p in iv[0][nsw - 1]]     # the gathered last sweep
                out["max_rel_dI_vs_reference"] = {
                    "all_points": rel_dI(last, rcur), "on_state_Id_gt_1nA": rel_dI(last, rcur, on=1e-9),
                    "note": "the reference core's sampled points; off-state currents converge to ~1e-3 in either "
                            "code at the workload's default tolerances"}
    return out


def run_reference(a, dist):
    """The reference's own CPU core on the same workload, all host threads.  The workload's
    step is every point of its sweeps after the first (48 for the n-MOSFET); a reference
    step times a window of 3 consecutive points of that sequence, and the windows slide
    through it from step to step, so that over the timed steps every point of the GPU arm's
    step is timed (the windows cycle; catching up to a window's start - a new sweep's
    api3_solve and any points before it - is untimed).  Each window continues from the
    previous point exactly as the GPU arm's sweep does."""
    if dist.rank != 0:
        return None
    mesh = mesh_of(a)
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_ref.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "reference core not built (make -C oracle)"}
    ref = abi.bind(ctypes.CDLL(path))
    cores = os.cpu_count() or 1
    ref.api3_set_threads(cores)
    w = build(ref, mesh)
    npts = 3
    seq = [(si, q) for si in range(len(w.sweeps)) for q in range(1, len(w.sweeps[si]["V"]))]
    nwin = len(seq) // npts
    cur_si, next_q = None, None
    tot = 0.0
    pts = 0
    timed = set()

    def resolve(s, q):
        for cid, vv in D.bias_vector(w, s, s["V"][q]).items():
            ref.api3_set_contact_V(cid, vv)
        return ref.api3_resolve()

    for i in range(a.warmup + a.steps):
        win = seq[(i % nwin) * npts:(i % nwin + 1) * npts]
        si, q0 = win[0]
        s = w.sweeps[si]
        if cur_si != si or next_q is None or next_q > q0:
            D.start_sweep(ref, w, s)                  # untimed: equilibrium + ramp to the sweep's start
            cur_si, next_q = si, 1
        while next_q < q0:                            # untimed: up to the window's first point
            resolve(s, next_q)
            next_q += 1
        t0 = time.perf_counter()
        for _, q in win:
            resolve(s, q)
        dt = time.perf_counter() - t0
        next_q = q0 + npts
        if i >= a.warmup:
            tot += dt
            pts += npts
            timed.update(win)
    v = pts / tot
    cfg = dict({"workload": workload_name(mesh), "nodes": w.N, "points_per_step": npts}, **workload_config(w),
               **{"solver": list(D.GUI_SOLVER), "precision": "fp64", "parallelism": f"cpu, {cores} threads",
                  "point_set": f"windows of {npts} consecutive points sliding through the {len(seq)} points of "
                               f"the workload step ({len(timed)} of them timed over the run)"})
    return {"metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * tot / a.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic (device built from the workload definition)",
            "config": cfg,
            "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{npts} consecutive points per step, windows sliding through all "
                                       f"{len(seq)} points of the workload step; {len(timed)} distinct points "
                                       "timed"},
            "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_batch(a, dist):
    """The batching workload: the 64 pn-diode variants (node counts 32^3..72^3, doping
    log-uniform in 1e15..1e18 cm^-3, junction depth 0.2..0.8 um, recorded seed), each swept
    0..0.7 V in 25 mV steps, one solver instance (own CUDA stream) per variant and
    `workers` host threads driving them at once (0: one per variant).  Untimed: device
    set-up, equilibrium and the first point of every sweep; timed (wall clock, max over
    ranks): the remaining 28 points of every sweep.  Ranks take every world-th variant
    (a fixed batch split across GPUs: strong scaling, no data-path collective)."""
    import queue
    import semiconductor_devices_simulator_b200 as S
    lib = S.load()
    lib.b200x_set_device(dist.local)
    prec = 1 if a.precision == "refined" else 0
    allv = D.diode_variants(64)[:a.variants or None]
    var = shard(allv, dist.rank, dist.world, weights=[int(np.prod(v["n"])) for v in allv])
    hs = [lib.api3b_new() for _ in var]
    ws = [None] * len(var)
    W = a.workers or len(var)
    persist_old = lib.api3b_set_persist(1 if a.batch_solves == "persistent" else 0, -1)
    # grid shares of the persistent solves: the SMs split in proportion to node counts when
    # every variant runs at once (cooperative grids that together exceed the SMs take turns)
    vn = [int(np.prod(v["n"])) for v in var]
    nsm = sm_count(dist.local)
    shares = [max(1, int(nsm * x / sum(vn))) for x in vn] if a.share == "gummel" and W >= len(var) else None

    def setup(q):
        lib.api3b_use(hs[q])
        lib.b200x_set_device(dist.local)
        lib.api3b_set_precision(prec)
        lib.api3b_set_share(shares[q] if shares else 0)
        ws[q] = D.diode_variant(lib, var[q])
        ok = D.start_sweep(lib, ws[q], ws[q].sweeps[0])
        lib.api3b_use(0)
        return ok

    def pool(fn, n, W):
        jobs = queue.Queue()
        for q in range(n):
            jobs.put(q)
        res = [None] * n

        def loop():
            while True:
                try:
                    q = jobs.get_nowait()
                except queue.Empty:
                    return
                res[q] = fn(q)
        th = [threading.Thread(target=loop) for _ in range(W)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        return res

    pool(setup, len(var), W)

    def run(q):
        lib.api3b_use(hs[q])
        n, c = sweep_points(lib, ws[q], ws[q].sweeps[0])
        lib.api3b_use(0)
        return n, c
    dist.barrier()
    t0 = time.perf_counter()
    res = pool(run, len(var), W)
    wall = time.perf_counter() - t0
    pts = sum(r[0] for r in res)
    conv = sum(r[1] for r in res)
    T = dist.max(wall)
    pts_all = dist.sum(pts)
    nodes = [int(np.prod(v["n"])) for v in var]
    for h in hs:
        lib.api3b_free(h)
    lib.api3b_set_persist(persist_old, -1)
    if dist.rank != 0:
        return None
    return {"metric": "I-V bias points/s (64 pn-diode variants, one instance and stream each)",
            "value": round(pts_all / T, 3), "unit": UNIT, "n_gpus": dist.world, "higher_is_better": True,
            "scaling": "strong", "wall_s": round(T, 3), "points": int(pts_all),
            "converged_points": conv, "dtype": "f32 inner solves refined in f64" if prec else "f64",
            "config": {"workload": "pn_diode_variants_64", "variants": len(var), "workers": W,
                       "nodes_min": min(nodes), "nodes_max": max(nodes), "nodes_total": sum(nodes),
                       "sweep_V": [0.0, 0.7, 0.025], "precision": a.precision,
                       "linear_solves": ("persistent (one cooperative launch per solve)"
                                         if a.batch_solves == "persistent" else "per-pass graphs"),
                       "grid_shares": "by node count" if shares and a.batch_solves == "persistent" else None,
                       "timing": "wall clock around all sweeps (host control included)"}}


def main():
    global WL
    a = parse()
    if a.workload in WORKLOADS:
        WL = a.workload
    if a.probe:
        return run_probe(a)
    dist = Dist()
    if a.workload == "diodes64" and a.impl != "reference":
        out = run_batch(a, dist)
    else:
        out = run_reference(a, dist) if a.impl == "reference" else run_b200(a, dist)
    if dist.rank == 0 and out is not None:
        print(json.dumps(out))
    dist.close()


if __name__ == "__main__":
    main()
