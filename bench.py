"""Throughput of the B200 SCN TLM step (node-updates/s and % of HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload heterogeneous|plain|precision|energy|batched|served|fdtd]
                    [--storage f32|bf16|f16|f64|bfp16] [--near-field R]

A "step" is one TLM time step (inject, monitors, scatter, connect) of the
whole grid. Default workload: 192^3 heterogeneous grid (16 lossy dielectric
boxes, differentiated-Gaussian source, 8 probes), FP32, synthetic and seeded.
Under torchrun every rank advances its own replica (weak scaling; the
instances are independent, so no collective is on the data path); times are
CUDA-event times on the solver's stream, max over ranks.

`--impl reference` times the reference's own CPU TLM step (compiled headless
under oracle/_ref from its sources) on the host cores for the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TLM node-updates/s"
UNIT = "node-updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="heterogeneous",
                   choices=["heterogeneous", "plain", "precision", "energy", "batched", "served", "fdtd", "slab"])
    p.add_argument("--instances", type=int, default=256, help="batched: number of instances")
    p.add_argument("--requests", type=int, default=200, help="served: number of requests")
    p.add_argument("--rate", type=float, default=200.0, help="served: mean arrivals per second")
    p.add_argument("--edge-max", type=int, default=128,
                   help="served: largest cubic edge (the full stream goes to 256)")
    p.add_argument("--steps-max", type=int, default=2000,
                   help="served: most steps per request (the full stream goes to 8000)")
    p.add_argument("--no-autotune", action="store_true",
                   help="batched: skip the autotuner (default tuning, windows of --window steps)")
    p.add_argument("--window", type=int, default=100, help="batched: steps per CUDA-graph window")
    p.add_argument("--profile-steps", type=int, default=0,
                   help="batched: only attach the instances and step them this many steps without "
                        "graphs (a small case for ncu); prints no bench line")
    p.add_argument("--near-field", type=int, default=None,
                   help="16-bit storage: radius of the FP32-residual box around PEC and ports "
                        "(default 6 for f16/bf16)")
    p.add_argument("--precision-steps", type=int, default=8000, help="precision: steps per mode")
    p.add_argument("--slab-edge", type=int, default=384,
                   help="slab: edge of the heterogeneous grid split into z-slabs over the ranks")
    p.add_argument("--order", default="least-work", choices=["least-work", "arrival"],
                   help="served: admission order")
    p.add_argument("--max-running-cells", type=int, default=8 << 20,
                   help="served: cap on the running requests' padded cells (0: none)")
    p.add_argument("--solo-cells", type=int, default=1 << 20,
                   help="served: requests this large run on their own beside the batch (0: never)")
    p.add_argument("--served-16bit", default="f16nf", choices=["f16nf", "bf16"],
                   help="served: storage of the stream's 16-bit half")
    p.add_argument("--energy-steps", type=int, default=3000, help="energy: steps per mode")
    p.add_argument("--chunk", type=int, default=32, help="batched: instances set up per window")
    p.add_argument("--host-threads", type=int, default=8,
                   help="batched: host threads that set up, read back and free the instances")
    p.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16", "f64", "bfp16"])
    p.add_argument("--steps-per-launch", type=int, default=0)
    p.add_argument("--kernel-variant", type=int, default=0,
                   help="tile shape of the step kernel (tlm_kernel_variants lists them)")
    p.add_argument("--no-staging", action="store_true",
                   help="one step kernel for all tiles (no staged FP32 / interior-only 16-bit kernel)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def make_workload(name, steps):
    from emsolver_b200 import workloads
    if name == "plain":
        return workloads.plain_free_space(steps=steps)
    if name == "precision":
        return workloads.precision_dipole(steps=steps)
    return workloads.heterogeneous(steps=2000)


STORAGE = {"f32": (0, 4, 4), "bf16": (1, 2, 4), "f16": (2, 2, 4), "f64": (3, 8, 8), "bfp16": (4, 2, 4)}


def near_of(args):
    """The near-field radius for the storage mode (default 6 for FP16/BF16)."""
    if args.storage not in ("f16", "bf16"):
        return 0
    return 6 if args.near_field is None else args.near_field


def box_nodes(s):
    b = s.nearFieldBox()
    return 0 if b is None else b[1][0] * b[1][1] * b[1][2]


def check_world(args):
    """--gpus N must match the launcher's WORLD_SIZE (torchrun starts the
    ranks; this script does not)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        sys.stderr.write(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch N ranks with "
                         f"python -m torch.distributed.run --nproc-per-node {args.gpus} bench.py --gpus "
                         f"{args.gpus} ...\n")
        sys.exit(2)
    return world
DTYPE = {"f32": "f32", "bf16": "bf16 storage / f32 arithmetic",
         "f16": "f16 storage / f32 arithmetic", "f64": "f64",
         "bfp16": "16-bit block floating point storage / f32 arithmetic"}


# ---------------------------------------------------------------- distributed
class Dist:
    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device="cuda")
            self.pg.all_reduce(t)
            torch.cuda.synchronize()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([float(v)], device="cuda", dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.path = None
        self.gpu = gpu_index

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- helpers
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload, storage):
    """DRAM bytes per step-kernel launch from the committed ncu capture."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    return d.get(f"{workload}_{storage}")


def reference_rate(w, steps_budget, seconds_budget, warm=2):
    """The reference's own CPU step on this host: node-updates/s over a
    bounded number of full-grid steps."""
    from oracle import RefSolver, Oracle, drive, ref_available
    if ref_available():
        S, kind = RefSolver(), "reference"
    else:
        S, kind = Oracle(False), "port"
    drive.setup(S, w)
    drive.advance(S, w, warm)
    t0 = time.perf_counter()
    done = 0
    while done < steps_budget:
        chunk = min(5, steps_budget - done)
        drive.advance(S, w, chunk)
        done += chunk
        if time.perf_counter() - t0 > seconds_budget:
            break
    dt = time.perf_counter() - t0
    cores = S.threads if kind == "reference" else 1
    return w.ncells * done / dt, cores, kind, done, dt


def run_reference_arm(args):
    world = check_world(args)
    d = Dist(args.gpus) if world > 1 else None
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from emsolver_b200 import workloads  # noqa: F401
    w = make_workload(args.workload, args.warmup + args.steps)
    rate, cores, kind, done, dt = reference_rate(w, args.steps, 120.0, warm=min(args.warmup, 3))
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dt / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "impl": "reference",
        "config": {"workload": f"{args.workload} {w.nx}x{w.ny}x{w.nz}", "steps_timed": done},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{done} full-grid steps of {w.nx}x{w.ny}x{w.nz} "
                                   f"({os.cpu_count()} host cores, {cores} solver threads)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if d:
        d.close()


def accuracy_vs_reference(s, w, steps_done):
    """Port and probe records of the timed solve against the reference's own
    CPU step on the same grid (tests/golden/heterogeneous.npz, written by the
    reference compiled headless): the largest |difference| over the peak of
    each series, over the steps both runs cover."""
    path = os.path.join(ROOT, "tests", "golden", "heterogeneous.npz")
    if w.name != "heterogeneous" or (w.nx, w.ny, w.nz) != (192, 192, 192) or not os.path.exists(path):
        return None
    g = np.load(path)
    n = min(steps_done, g["port0_v"].shape[0])
    ours = {}
    p = s.port(0)
    ours["port0_v"], ours["port0_i"] = p.vRec, p.iRec
    for q in range(len(w.probes_cell)):
        r = s.probe(q)
        ours[f"probe{q}_ex"], ours[f"probe{q}_ey"], ours[f"probe{q}_ez"] = r.ex, r.ey, r.ez
    worst, exact = 0.0, True
    for k, a in ours.items():
        a = np.asarray(a[:n], np.float64)
        b = g[k][:n].astype(np.float64)
        d = float(np.abs(a - b).max()) if n else 0.0
        peak = float(np.abs(b).max()) if n else 0.0
        exact = exact and d == 0.0
        if peak > 0:
            worst = max(worst, d / peak)
    return {"vs": "the reference's CPU step on the same grid (its records in tests/golden/heterogeneous.npz)",
            "steps_compared": n, "series": len(ours), "max_abs_diff_over_peak": worst,
            "bitwise": bool(exact), "tolerance": 1e-5}


def run_ours(args):
    from emsolver_b200.runner import build_solver
    import torch

    check_world(args)
    dist = Dist(args.gpus)
    dev = dist.local if dist.world > 1 else 0
    code, sbytes, rbytes = STORAGE[args.storage]
    nf = near_of(args)
    w = make_workload(args.workload, args.warmup + args.steps)
    w.steps = args.warmup + args.steps
    s = build_solver(w, device=dev, storage=code, steps_per_launch=args.steps_per_launch, near_field=nf,
                     no_staging=args.no_staging, kernel_variant=args.kernel_variant)
    torch.cuda.set_device(dev)
    ext = torch.cuda.ExternalStream(s.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the clock sampler's first samples come from an idle GPU: the warm-up
    # steps follow them, right before the timed steps (after an idle pause
    # the first steps measured about 1 % slower)
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    s.step(args.warmup)
    dist.barrier()
    torch.cuda.synchronize(dev)
    s.sync()
    s.setKernelTiming(True)
    e0.record(ext)
    s.stepAsync(args.steps)
    e1.record(ext)
    s.sync()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    kern_ms, launches = s.kernelTime()
    s.setKernelTiming(False)
    per_step_kernels = s.stepLaunches()
    ms_max = dist.max(ms)
    kern_max = dist.max(kern_ms)
    accuracy = accuracy_vs_reference(s, w, args.warmup + args.steps) if args.storage == "f32" else None
    nbox = box_nodes(s)
    s.close()

    n = w.ncells
    value = dist.world * n * args.steps / (ms_max / 1000.0)
    # 16-bit storage with a near-field box: its cells also read and write
    # the 12 FP32 residuals
    bytes_step = w.bytes_per_step(sbytes, rbytes) + 96 * nbox
    per_launch_ms = kern_max / max(launches, 1)
    achieved = bytes_step / (per_launch_ms / 1000.0) / 1e9
    peak, peak_kind = peaks()
    window = args.steps_per_launch or 64
    epilogues = -(-args.steps // window)

    # end to end through the public API: host material map in, setup,
    # K steps, probe and port records back to the host.
    e2e = None
    if not args.no_e2e:
        # one untimed solve through the same calls first (W steps): the
        # process's first set-ups pay one-time host costs (the allocator's
        # first pass over a fresh heap measured 3 ms of a 5 ms solve)
        s2 = build_solver(w, device=dev, storage=code, steps_per_launch=args.steps_per_launch, near_field=nf,
                          no_staging=args.no_staging, kernel_variant=args.kernel_variant)
        s2.step(max(args.warmup, 1))
        [s2.probe(q) for q in range(len(w.probes_cell))]
        s2.close()
        dist.barrier()
        t0 = time.perf_counter()
        s2 = build_solver(w, device=dev, storage=code, steps_per_launch=args.steps_per_launch, near_field=nf,
                          no_staging=args.no_staging, kernel_variant=args.kernel_variant)
        s2.step(args.steps)
        recs = [s2.probe(q) for q in range(len(w.probes_cell))]
        ports = [s2.port(p) for p in range(len(w.ports))]
        t1 = time.perf_counter()
        s2.close()
        dt = dist.max(t1 - t0)
        h2d = w.mat.nbytes + 8 * len(w.table) + (w.sv.nbytes if w.sv is not None else 0)
        d2h = sum(3 * 4 * r.ez.size for r in recs) + sum(2 * 4 * p.vRec.size for p in ports)
        e2e = {"value": dist.world * n * args.steps / dt, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "seconds": dt, "includes": "setup (H2D of the material map, tables, sources), "
                                          "all steps, D2H of probe and port records (after one untimed "
                                          "warm-up solve of W steps through the same calls)"}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        rate, cores, kind, done, dt = reference_rate(w, 400, 20.0)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{done} full-grid steps of {w.nx}x{w.ny}x{w.nz} in {dt:.1f}s "
                         f"({os.cpu_count()} host cores)"}

    if dist.rank == 0:
        tr = ncu_traffic(args.workload, args.storage)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[args.storage], "data": "synthetic (seeded)",
            "config": {"workload": f"{args.workload} {w.nx}x{w.ny}x{w.nz}, {len(w.table)} lossy "
                                   f"dielectric boxes, {len(w.probes_cell)} probes",
                       "nodes": n, "dielectric_nodes": w.n_diel(),
                       "storage": args.storage, "near_field": nf, "near_field_cells": nbox,
                       "steps_per_launch": window,
                       "parallelism": f"replicas x{dist.world}",
                       "l2": f"state {2 * 12 * sbytes * n / 1e6:.0f} MB > L2 (126 MB); no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": tr, "algorithmic_bytes_per_step": bytes_step,
                         "kernel_ms_per_step": per_launch_ms, "kernels_per_step": per_step_kernels},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "accuracy": accuracy,
            "gpu_launches": launches * per_step_kernels + epilogues,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    dist.close()


def run_fdtd(args):
    """The Yee FDTD solver on the 192^3 heterogeneous grid (same materials,
    source and probes as the TLM default): cell-updates/s of the whole step
    (sources, monitors, H and E updates, Mur boundary), against the
    reference's own FdtdSolver on the host cores."""
    import torch
    from emsolver_b200 import workloads
    from emsolver_b200.fdtd import build_fdtd
    from oracle import RefFdtd, drive
    w = workloads.heterogeneous(steps=args.warmup + args.steps)
    s = build_fdtd(w)
    s.step(args.warmup)
    ext = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    e0.record(ext)
    s.step(args.steps)
    e1.record(ext)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    s.close()
    n = w.ncells
    bytes_step = n * (75 + 24)   # H: E read + H read/write; E: H read + E read/write + masks + lossy coefficients
    achieved = bytes_step / (ms / args.steps / 1000.0) / 1e9
    peak, kind = peaks()
    t0 = time.perf_counter()
    s2 = build_fdtd(w)
    s2.step(args.steps)
    recs = [s2.probe(q) for q in range(len(w.probes_cell))]
    t1 = time.perf_counter()
    s2.close()
    cpu = None
    if not args.no_cpu_baseline:
        R = RefFdtd()
        drive.setup(R, w)
        if w.waveform == 3:
            R.steps(2, sv=w.sv[:2])
        done, tc = 0, time.perf_counter()
        while done < 200 and time.perf_counter() - tc < 20.0:
            drive.advance(R, w, 5)
            done += 5
        dtc = time.perf_counter() - tc
        cpu = {"value": n * done / dtc, "unit": "cell-updates/s", "cores": max(1, min(16, (os.cpu_count() or 2) - 1)),
               "kind": "reference", "sample": f"{done} full-grid FDTD steps of {w.nx}x{w.ny}x{w.nz} in {dtc:.1f}s"}
    line = {"metric": "FDTD cell-updates/s", "value": n * args.steps / (ms / 1000.0), "unit": "cell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"fdtd heterogeneous {w.nx}x{w.ny}x{w.nz}, {len(w.table)} lossy dielectric boxes",
                       "cells": n},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": kind, "traffic": None, "algorithmic_bytes_per_step": bytes_step},
            "cpu_baseline": cpu,
            "e2e": {"value": n * args.steps / (t1 - t0), "unit": "cell-updates/s",
                    "h2d_bytes_per_step": w.mat.nbytes / args.steps,
                    "d2h_bytes_per_step": sum(12 * r[0].size for r in recs) / args.steps, "seconds": t1 - t0},
            "clocks": clk}
    print(json.dumps(line), flush=True)


PRECISION_MODES = [("f64", 3, 0), ("f32", 0, 0), ("f16", 2, 0), ("f16_near6", 2, 6), ("bf16", 1, 0),
                   ("bf16_near6", 1, 6), ("bfp16", 4, 0)]


def timed_solve(w, storage, near):
    """Set up, step the whole run with CUDA events on the solver's stream,
    return (solver, ms)."""
    import torch
    from emsolver_b200.runner import build_solver
    s = build_solver(w, storage=storage, near_field=near)
    s.step(1)
    ext = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    s.stepAsync(w.steps - 1)
    e1.record(ext)
    s.sync()
    torch.cuda.synchronize()
    return s, e0.elapsed_time(e1)


def run_precision(args):
    """The precision configuration: 384x384x256 grid, half-wave dipole of 60
    PEC cells with a 1-cell feed gap, Gaussian voltage source across the gap,
    outer reflection 0, port DFT at 64 frequencies over 0.5-1.5 of resonance,
    --precision-steps steps (8000 by default), in every storage mode. Input
    impedance and S11 of each mode against the FP64 storage mode (bitwise
    the FP64 oracle on the grids the tests cover), largest relative error
    over the 64 frequencies; node-updates/s and the fraction of the measured
    HBM bandwidth at each mode's algorithmic bytes."""
    from emsolver_b200 import workloads
    from emsolver_b200.solver import s11_from_dft
    w = workloads.precision_dipole(steps=args.precision_steps)
    peak, kind = peaks()
    res = {}
    for name, code, near in PRECISION_MODES:
        s, ms = timed_solve(w, code, near)
        v, i = s.portDft(0)
        z, g = s11_from_dft(v, i)
        sb, rb = {0: (4, 4), 1: (2, 4), 2: (2, 4), 3: (8, 8), 4: (2, 4)}[code]
        nbox = box_nodes(s)
        s.close()
        per_step = ms / (w.steps - 1)
        bytes_step = w.bytes_per_step(sb, rb) + 96 * nbox
        res[name] = {"z": z, "s11": g, "ms_per_step": per_step, "near_field_cells": nbox,
                     "node_updates_per_s": w.ncells / (per_step / 1e3),
                     "hbm_frac": bytes_step / (per_step / 1e3) / 1e9 / peak}
    zr, gr = res["f64"]["z"], res["f64"]["s11"]
    modes = {}
    for name, r in res.items():
        modes[name] = {"s11_rel_err_vs_fp64": float(np.max(np.abs(r["s11"] - gr) / np.abs(gr))),
                       "zin_rel_err_vs_fp64": float(np.max(np.abs(r["z"] - zr) / np.abs(zr))),
                       "ms_per_step": r["ms_per_step"], "node_updates_per_s": r["node_updates_per_s"],
                       "hbm_frac": r["hbm_frac"], "near_field_cells": r["near_field_cells"]}
    head = modes["f16_near6"]
    line = {"metric": "S11 relative error vs FP64 storage", "value": head["s11_rel_err_vs_fp64"],
            "unit": "relative (max over 64 frequencies)", "n_gpus": 1, "steps": w.steps, "warmup": 1,
            "ms_per_step": head["ms_per_step"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 storage + FP32 residuals in the near-field box / f32 arithmetic",
            "data": "synthetic (seeded)",
            "config": {"workload": f"precision dipole {w.nx}x{w.ny}x{w.nz}, {w.meta['length'] - 1} PEC cells "
                                   f"+ 1-cell gap, {len(w.dft_freqs)} DFT frequencies, {w.steps} steps",
                       "headline_mode": "f16_near6", "peak_kind": kind},
            "zin_rel_err_vs_fp64": head["zin_rel_err_vs_fp64"],
            "s11_rel_err_vs_fp64": {k: m["s11_rel_err_vs_fp64"] for k, m in modes.items()},
            "modes": modes}
    print(json.dumps(line), flush=True)


def run_energy(args):
    """Energy drift of a closed lossless grid: 128^3 cells, outer reflection
    1, no loss, a PEC dipole of 31 cells fed by a Gaussian pulse that has
    died out by step 512. The FP64 energy history (every 16 steps, the
    reference's cadence) from step 512 to the last step stays constant in
    exact arithmetic; reported per storage mode: the relative change from
    step 512 to the end and the largest relative excursion."""
    from emsolver_b200 import workloads
    w = workloads.dipole(128, 128, 128, 31, None, steps=args.energy_steps, nfreq=8, name="closed_cavity")
    w.rho = 1.0
    modes = {}
    for name, code, near in PRECISION_MODES:
        s, ms = timed_solve(w, code, near)
        st, ev = s.getEnergyHistory(f64=True)
        s.close()
        st, ev = np.asarray(st), np.asarray(ev, np.float64)
        k0 = int(np.searchsorted(st, 512))
        e0 = ev[k0]
        modes[name] = {"drift": float((ev[-1] - e0) / e0),
                       "max_excursion": float(np.max(np.abs(ev[k0:] - e0)) / e0),
                       "from_step": int(st[k0]), "to_step": int(st[-1]), "ms_per_step": ms / (w.steps - 1)}
    line = {"metric": "relative energy drift, closed lossless grid", "value": modes["f32"]["drift"],
            "unit": "relative", "n_gpus": 1, "steps": w.steps, "warmup": 1,
            "ms_per_step": modes["f32"]["ms_per_step"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (per-mode results in `modes`)", "data": "synthetic",
            "config": {"workload": f"closed cavity {w.nx}x{w.ny}x{w.nz}, rho 1, lossless, 31-cell PEC dipole, "
                                   f"Gaussian pulse source, {w.steps} steps"},
            "modes": modes}
    print(json.dumps(line), flush=True)


def run_slab(args):
    """One grid split into z-slabs over the ranks of the launch (torchrun,
    NCCL between GPUs): the heterogeneous grid of --slab-edge cells per axis
    (16 lossy dielectric boxes, a source, 8 probes), every rank stepping its
    own planes with the halo exchange overlapped (tlm_slab_step_begin/_end),
    device-timed on each rank's stream, max over ranks. Strong scaling: the
    grid is the same at every rank count; value = the grid's node-updates
    per second."""
    import datetime
    import torch
    import torch.distributed as tdist
    from emsolver_b200 import workloads
    from emsolver_b200.slab import SlabSolver
    world = check_world(args)
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not tdist.is_initialized():
        if world > 1:
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        else:
            tdist.init_process_group("gloo", init_method="tcp://127.0.0.1:0", rank=0, world_size=1)
    w = workloads.heterogeneous(n=args.slab_edge, steps=args.warmup + args.steps)
    s = SlabSolver(w, device=local)
    s.step(args.warmup)
    ext = torch.cuda.ExternalStream(s.slab.solver.stream(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        tdist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0.record(ext)
    s.step(args.steps)
    e1.record(ext)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
    halo = s.slab.nbytes * ((s.send_lo is not None) + (s.send_hi is not None))
    s.close()
    if rank == 0:
        line = {"metric": "TLM node-updates/s (one grid in z-slabs)", "value": w.ncells * args.steps / (ms / 1e3),
                "unit": "node-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": {"workload": f"heterogeneous {w.nx}x{w.ny}x{w.nz} split into {world} z-slabs",
                           "nodes": w.ncells, "slab_planes": [list(r) for r in s.ranges],
                           "halo_bytes_per_step_rank0": halo, "parallelism": f"z-slabs x{world}"},
                "clocks": clk}
        print(json.dumps(line), flush=True)
    tdist.destroy_process_group()


def sequential_solves(ws):
    """Each instance alone through the plain API, one after the other:
    setup, all steps, port DFT back to the host, free. Returns per-solve
    seconds."""
    from emsolver_b200.runner import build_solver
    times = []
    for w in ws:
        t0 = time.perf_counter()
        s = build_solver(w)
        s.step(w.steps)
        s.portDft(0)
        s.close()
        times.append(time.perf_counter() - t0)
    return times


def batch_dfts(ws, storage, near, tuning=None):
    """Every instance attached to one batch and run to its end; returns the
    port DFTs (untimed helper for the accuracy check)."""
    from emsolver_b200 import Batch
    from emsolver_b200.runner import build_solver
    solvers = [build_solver(w, storage=storage, near_field=near) for w in ws]
    with Batch() as b:
        for s in solvers:
            b.attach(s)
        if tuning is not None:
            b.set_tuning(tuning)
        b.run()
    out = [s.portDft(0) for s in solvers]
    for s in solvers:
        s.close()
    return out


def run_batched(args):
    """256 independent dipole instances (edges U{24..96} per axis, wire of
    U[0.3,0.9] of the z extent with a 1-cell gap port, dielectric slab eps_r
    U[1,6]), 1000 steps each, FP32 storage unless --storage says otherwise;
    CUDA-graph windows of 100 steps, tile shape and window chosen by the
    autotuner (--no-autotune: defaults). Against the same instances solved
    one after the other through the plain API; every instance's S11 against
    an FP64-storage batch of the same instances."""
    import torch
    from emsolver_b200 import Batch, BatchTuning, workloads
    from emsolver_b200.runner import build_solver
    from emsolver_b200.solver import s11_from_dft
    code, sbytes, rbytes = STORAGE[args.storage]
    nf = near_of(args)
    ws = workloads.batched_instances(count=args.instances, steps=1000)
    for w in ws:
        w.storage = code
        w.meta["near_field"] = nf
    if args.profile_steps > 0:
        solvers = [build_solver(w) for w in ws]
        with Batch() as b:
            for s in solvers:
                b.attach(s)
            b.set_tuning(BatchTuning(steps_per_launch=16, use_graphs=False))
            b.step(args.profile_steps)
        for s in solvers:
            s.close()
        return
    nodes = sum(w.ncells for w in ws)
    work = sum(w.ncells * w.steps for w in ws)
    sequential_solves(ws[:4])                        # warm-up (context, kernels)
    # Python's cyclic garbage collector is paused in both timed regions, as
    # timeit does, so that a collection pass over the thousands of workload
    # objects alive here lands in neither
    import gc
    gc.collect()
    gc.disable()
    seq = sequential_solves(ws)
    gc.enable()
    # the solves through Batch.solve: set-up of the next instances overlaps
    # the device's windows, finished members leave at once
    tp = time.perf_counter()
    with Batch() as bp:
        bp.set_tuning(BatchTuning(steps_per_launch=args.window))
        dfts = bp.solve(ws, build_solver, lambda s, w: s.portDft(0), chunk=args.chunk)
    pipelined_s = time.perf_counter() - tp
    assert len(dfts) == len(ws)
    # the tuning: the autotuner on these instances (untimed; cached by
    # workload signature), or the defaults
    if args.no_autotune:
        tuning = BatchTuning(steps_per_launch=args.window)
    else:
        tsolvers = [build_solver(w) for w in ws]
        with Batch() as bt:
            for s in tsolvers:
                bt.attach(s)
            tuning = bt.autotune(trial_windows=2)
        for s in tsolvers:
            s.close()
    # all instances attached at once: set-up, the device time of the whole
    # run, read-back; handles are independent (a stream each, a thread-safe
    # device pool), so the host work is spread over --host-threads threads
    from concurrent.futures import ThreadPoolExecutor
    pool = ThreadPoolExecutor(max_workers=max(1, args.host_threads))
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    solvers = list(pool.map(build_solver, ws))
    tb = time.perf_counter()
    b = Batch()
    for s in solvers:
        b.attach(s)
    b.set_tuning(tuning)
    ta = time.perf_counter()
    t1 = time.perf_counter()
    ext = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    b.run()
    e1.record(ext)
    torch.cuda.synchronize()
    gpu_ms = e0.elapsed_time(e1)
    got = list(pool.map(lambda s: s.portDft(0), solvers))
    t2 = time.perf_counter()
    b.close()
    tc = time.perf_counter()
    nbox = sum(box_nodes(s) for s in solvers)
    list(pool.map(lambda s: s.close(), solvers))
    t3 = time.perf_counter()
    pool.shutdown()
    gc.enable()
    batched_s = t3 - t0
    # accuracy: S11 of every instance against the FP64 storage mode
    ref = batch_dfts(ws, 3, 0)
    errs = []
    for (v, i), (rv, ri) in zip(got, ref):
        a, r = s11_from_dft(v, i)[1], s11_from_dft(rv, ri)[1]
        errs.append(float(np.max(np.abs(a - r) / np.abs(r))))
    peak, kind = peaks()
    bytes_all = sum(w.bytes_per_step(sbytes, rbytes) * w.steps for w in ws) + 96 * nbox * 1000
    line = {
        "metric": "batched solves/s", "value": len(ws) / batched_s, "unit": "solves/s",
        "n_gpus": 1, "steps": 1000, "warmup": 4, "ms_per_step": gpu_ms / 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE[args.storage] + (f", near-field box r={nf}" if nf else ""),
        "data": "synthetic (seeded)",
        "config": {"workload": f"batched: {len(ws)} dipole instances, edges U{{24..96}}, 1000 steps",
                   "nodes": nodes, "storage": args.storage, "near_field": nf,
                   "tuning": tuning.__dict__, "autotuned": not args.no_autotune,
                   "host_threads": args.host_threads, "python_gc": "paused in the timed regions",
                   "includes": "setup of every instance, all steps, port DFT read-back, free"},
        "sequential_plain_gpu": {"value": len(ws) / sum(seq), "unit": "solves/s",
                                 "seconds": sum(seq), "p50_s": float(np.percentile(seq, 50)),
                                 "p99_s": float(np.percentile(seq, 99))},
        "speedup_vs_sequential": sum(seq) / batched_s,
        "seconds": batched_s,
        "s11_rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs)), "instances": len(errs),
                                "within_1e-3": int(sum(e <= 1e-3 for e in errs))},
        "pipelined": {"value": len(ws) / pipelined_s, "unit": "solves/s", "seconds": pipelined_s,
                      "chunk": args.chunk, "speedup_vs_sequential": sum(seq) / pipelined_s,
                      "api": "Batch.solve: host set-up of the next chunk overlaps each window"},
        "batched_gpu": {"node_updates_per_s": work / (gpu_ms / 1e3), "seconds": gpu_ms / 1e3,
                        "setup_s": t1 - t0, "setup_build_s": tb - t0, "setup_attach_s": ta - tb,
                        "readback_s": t2 - t1 - gpu_ms / 1e3, "batch_close_s": tc - t2,
                        "free_s": t3 - tc,
                        "hbm_frac": bytes_all / (gpu_ms / 1e3) / 1e9 / peak, "peak_kind": kind},
    }
    print(json.dumps(line), flush=True)


def run_served(args):
    """Poisson arrivals of dipole solves (cubic edge log-uniform, steps
    uniform, FP32 or 16-bit storage with probability 0.5), scaled by
    --edge-max and --steps-max; latency percentiles beside solves/s, against
    the same stream served one solve at a time by the plain API (a FIFO
    replay of each request's measured plain solve time). The stream's 16-bit
    half is stored as FP16 with the near-field box (--served-16bit f16nf,
    the default: BF16 misses the 1e-3 S11 bar even with the box) or as BF16
    (--served-16bit bf16). Every request's S11 is checked against an FP64
    storage run of the same solve."""
    import threading
    from emsolver_b200 import Server, workloads
    from emsolver_b200.solver import s11_from_dft
    stream = workloads.request_stream(count=args.requests, rate=args.rate, edge_hi=args.edge_max,
                                      steps_hi=args.steps_max)
    arrivals = [t for t, _ in stream]
    ws = [w for _, w in stream]
    for w in ws:
        w.dft_freqs = w.dft_freqs[:16]
        if w.storage == 1:                        # the stream's 16-bit half
            if args.served_16bit == "f16nf":
                w.storage, w.meta["near_field"] = 2, 6
            else:
                w.meta["near_field"] = 0
    sequential_solves([ws[0]])
    seq = sequential_solves(ws)
    # plain FIFO single-solve server on the same arrival stream
    done = 0.0
    plain_lat = []
    for a, svc in zip(arrivals, seq):
        done = max(done, a) + svc
        plain_lat.append(done - a)
    plain_span = done - arrivals[0]
    srv = Server(steps_per_launch=64)
    srv.set_policy(Server.ARRIVAL if args.order == "arrival" else Server.LEAST_WORK, args.max_running_cells,
                   args.solo_cells)
    ids = [None] * len(ws)
    t0 = time.perf_counter()

    def feeder():
        for k, (a, w) in enumerate(zip(arrivals, ws)):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            ids[k] = srv.submit(w)

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    for rid in ids:
        srv.wait(rid, -1.0)
    t1 = time.perf_counter()
    lat, got = [], []
    for rid in ids:
        v, i, l = srv.result(rid)
        lat.append(l)
        got.append((v, i))
    st = srv.stats()
    srv.close()
    span = t1 - t0
    # every request's S11 against the FP64 storage mode (one FP64 batch)
    ref = batch_dfts(ws, 3, 0)
    errs = {"f32": [], "16-bit": []}
    for w, (v, i), (rv, ri) in zip(ws, got, ref):
        a, r = s11_from_dft(v, i)[1], s11_from_dft(rv, ri)[1]
        errs["f32" if w.storage == 0 else "16-bit"].append(float(np.max(np.abs(a - r) / np.abs(r))))
    work = sum(w.ncells * w.steps for w in ws)
    line = {
        "metric": "served solves/s", "value": len(ws) / span, "unit": "solves/s", "n_gpus": 1,
        "steps": len(ws), "warmup": 1, "ms_per_step": 1000.0 * span / len(ws),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 or 16-bit storage per request (" +
                 ("FP16 + near-field box r=6" if args.served_16bit == "f16nf" else "BF16") + ")",
        "data": "synthetic (seeded Poisson stream)",
        "config": {"workload": f"served: {len(ws)} requests, Poisson {args.rate}/s, cubic edge "
                               f"log-U[32,{args.edge_max}], steps U[500,{args.steps_max}]",
                   "node_updates": work, "order": args.order, "max_running_cells": args.max_running_cells,
                   "solo_cells": args.solo_cells,
                   "served_16bit": args.served_16bit},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "mean": float(np.mean(lat))},
        "plain_sequential": {"solves_per_s": len(ws) / plain_span,
                             "latency_p50_s": float(np.percentile(plain_lat, 50)),
                             "latency_p99_s": float(np.percentile(plain_lat, 99)),
                             "busy_s": sum(seq)},
        "speedup_vs_plain": plain_span / span,
        "node_updates_per_s": work / span,
        "s11_rel_err_vs_fp64": {k: {"max": max(v), "median": float(np.median(v)), "requests": len(v),
                                    "within_1e-3": int(sum(e <= 1e-3 for e in v))}
                                for k, v in errs.items() if v},
        "server": st,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "fdtd":
        run_fdtd(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload == "energy":
        run_energy(args)
    elif args.workload == "slab":
        run_slab(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
