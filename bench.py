"""Benchmark of the B200 multi-fluid Hall-MHD step (one JSON line on stdout).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (synthetic inputs generated here):
  cube32   config 1: one periodic curvilinear 32^3 block, Orszag-Tang vortex on
           two ion fluids (H+, Na+ mass 1:23), Hall + electron pressure on,
           resistivity off, CFL 0.4, FP64.

Metric: Mcell-updates/s = owned cells x steps / time (ghost cells are never
counted; "per fluid" is the same count with n_fluids = 2).  ``value`` times K
steps with the state resident in HBM (CUDA events on the solve's stream, L2
flushed between steps because the 32^3 working set fits in L2); ``e2e`` is a
full solve through the C ABI with host buffers: pinned-host uploads of every
input field, mhd_prepare, K synchronous mhd_step calls each returning dt to the
host, and the download of the final state.

With --gpus N > 1 (torchrun), each rank runs an independent replica of the
workload (the single-block step has no data-path exchange); ``value`` is the
sum of all replicas' cell updates over the max-over-ranks device time.

``--impl reference`` times the reference's own CPU implementation (the
reference solver compiled from its sources, oracle/_ref/mercury_ref) on a
bounded sample of the same workload on this host; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s batched vs plain on 1 B200 at stated error; p50/p99 latency"
UNIT = "Mcell-updates/s"
L2_BYTES = 126 * 1024 * 1024

# Algorithmic HBM bytes per owned cell of each FP64 kernel: the distinct field
# components it must read and write once per DOF (8 B each), as listed in
# mpcns_mercury_b200/csrc/mhd_kernels.cu.  Kernels over the allocated cell
# range count the allocated cells.
KERNEL_BYTES_PER_CELL = {
    "k_face_emf": 8 * (3 + 3 + 3 + 9),                      # B, Badd, UCON -> Eface
    "k_edge_emf": 8 * (9 + 3 + 3 + 2 + 2 + 3),              # Eface, UCON, B, p_e x2, rho x2 -> E
    "k_hall_cell": 8 * (2 + 3 + 3 + 3 + 1),                 # rho x2, J_cell, B_cell -> EHC, beta
    "k_hall_edge": 8 * (3 + 1 + 9 + 3 + 3 + 3 + 3 + 3),     # EHC, beta, dr, dl, Area, B, taper -> Ehall
    "k_add_hall": 8 * (3 + 3 + 3),                          # E += Ehall
    "k_fluid": 8 * (10 + 10 + 9 + 1 + 3 + 3 + 3 + 1 + 3 + 10),  # U, PV, JD, Jac, U+, B_cell, J_cell, Photo, xyz -> U'
    "k_bface": 8 * (3 + 3 + 3),                             # B += dt curl E
    "k_bcell_jedge": 8 * (3 + 3 + 18 + 3 + 3 + 3 + 3 + 3),  # B, Badd, W_B, beta, alpha -> B_cell, Bind, J edges
    "k_jcell": 8 * (3 + 36 + 3),                            # J edges, W_J -> J_cell
    "k_pv_uplus": 8 * (10 + 1 + 9 + 3 + 10 + 3 + 3),        # U, Jac, JD, B_cell -> PV, U+, UCON (+ dt)
}
ALLOCATED_RANGE_KERNELS = {"k_hall_cell", "k_pv_uplus"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int = 0):
        self.index = index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
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
        self.out.seek(0)
        rows = [r.strip() for r in self.out.read().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            f = [x.strip() for x in r.split(",")]
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ workloads
def build_workload(name: str):
    """(cells per block, static+state fields {ref name: Arr}, topology kind)"""
    from mpcns_mercury_b200 import setup as S

    if name == "cube32":
        geom, f = S.cube_case(32)
        return [(32, 32, 32)], [f], "config 1: periodic curvilinear 32^3 cube, Orszag-Tang, 2 ion fluids, Hall+p_e, FP64"
    if name.startswith("cube"):
        n = int(name[4:])
        geom, f = S.cube_case(n)
        return [(n, n, n)], [f], f"config-1 physics on a periodic curvilinear {n}^3 cube (size study), FP64"
    raise SystemExit(f"unknown workload {name}")


from mpcns_mercury_b200.workloads import UPLOAD_FIELDS, capi_field  # noqa: E402


def make_context(cells, fields, pinned=None):
    """Create a context and upload every input field (optionally from pinned copies)."""
    from mpcns_mercury_b200 import Context, reference_constants

    ctx = Context(cells, 4, reference_constants(cfl=0.4))
    h2d = 0
    for b, f in enumerate(fields):
        for name in UPLOAD_FIELDS:
            a = f[name]
            data = pinned[b][name] if pinned is not None else a.data
            ctx.upload(capi_field(name), data, a.lo, a.hi, block=b)
            h2d += data.nbytes
    ctx.sync("UCELL")
    ctx.sync("BFACE")
    ctx.prepare()
    return ctx, h2d


def owned_cells(cells):
    return sum(a * b * c for a, b, c in cells)


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world, device):
    import torch

    cells, fields, desc = build_workload(args.workload)
    ncell = owned_cells(cells)
    ctx, _ = make_context(cells, fields)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)

    ctx.step(args.warmup)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(device.index if device.index is not None else 0)
    if rank == 0:
        sampler.start()
    total_ms = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.fill_(1.0)  # evict L2 between timed steps (32^3 working set < L2)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.step_async(1)
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
    ctx.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop() if rank == 0 else None
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        torch.distributed.barrier()
    info = ctx.info()
    value = world * ncell * args.steps / (total_ms * 1e-3) / 1e6

    # per-kernel profile (eager, events between kernels) for the roofline
    nprof = max(3, min(20, args.steps))
    prof = profile_kernels(ctx, nprof)
    launches_per_step = ctx.kernels_per_step()
    peak, peak_kind = load_peaks()
    roof = roofline(prof, cells, peak, peak_kind)

    # e2e through the C ABI with host buffers
    e2e = run_e2e(args, cells, fields, device)
    ctx.close()

    cpu = cpu_baseline_sample(args) if (rank == 0 and not args.no_cpu_baseline) else None
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "cells_per_replica": ncell,
                   "blocks": [list(c) for c in cells], "nghost": 4, "precision": "fp64",
                   "l2": "flushed between timed steps (2x L2 write)", "graph": "one CUDA graph per step",
                   "parallelism": f"replicas x{world}", "final_dt": info.dt, "final_time": info.time},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
        "kernel_ms": {k: round(v, 5) for k, v in prof.items()},
    }
    return line


def profile_kernels(ctx, nsteps):
    import ctypes
    from mpcns_mercury_b200.capi import check, lib

    L = lib()
    L.mhd_step_profiled.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int)]
    ms = (ctypes.c_float * 256)()
    names = (ctypes.c_char_p * 256)()
    n = ctypes.c_int()
    check(L.mhd_step_profiled(ctx.ctx, nsteps, 256, ms, names, ctypes.byref(n)), "mhd_step_profiled")
    out = {}
    for q in range(n.value):
        key = names[q].decode()
        out[key] = out.get(key, 0.0) + ms[q]
    return out


def roofline(prof, cells, peak, peak_kind):
    kernels = {k: v for k, v in prof.items() if k in KERNEL_BYTES_PER_CELL}
    if not kernels:
        return None
    top = max(kernels, key=kernels.get)
    g = 4
    ncell = sum((a + 2 * g) * (b + 2 * g) * (c + 2 * g) if top in ALLOCATED_RANGE_KERNELS else a * b * c
                for a, b, c in cells)
    algo_bytes = KERNEL_BYTES_PER_CELL[top] * ncell
    ms = kernels[top]
    achieved = algo_bytes / (ms * 1e-3) / 1e9
    traffic = load_traffic(top)
    return {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind,
            "algo_bytes_per_launch": int(algo_bytes), "launch_ms": round(ms, 5),
            "traffic": traffic, "share_of_step": round(ms / sum(prof.values()), 4)}


def load_traffic(kernel):
    """dram bytes per launch of ``kernel`` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "dram_bytes.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


def run_e2e(args, cells, fields, device):
    import torch

    pinned = []
    h2d_bytes = 0
    for f in fields:
        pf = {}
        for name in UPLOAD_FIELDS:
            a = f[name].data
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            pf[name] = t.numpy()
            h2d_bytes += a.nbytes
        pinned.append(pf)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx, _ = make_context(cells, fields, pinned=pinned)
    for _ in range(args.steps):
        ctx.step(1)  # synchronous: returns the step's dt to the host
    d2h = 0
    for b, f in enumerate(fields):
        for name, cname in (("U_H", "U_H"), ("U_Na", "U_NA"), ("B_xi", "B_XI"), ("B_eta", "B_ETA"),
                            ("B_zeta", "B_ZETA")):
            a = f[name]
            out = ctx.download(cname, a.lo, a.hi, block=b)
            d2h += out.nbytes
    t1 = time.perf_counter()
    ctx.close()
    ncell = owned_cells(cells)
    d2h += args.steps * 8
    return {"value": round(ncell * args.steps / (t1 - t0) / 1e6, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d_bytes / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
            "wall_s": round(t1 - t0, 4)}


# ------------------------------------------------------------------ reference arm
def reference_workload_job(workload):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    if workload == "cube32":
        job = dict(mo.CUBE_JOB)
        job.update(n=32)
        return job, 32 ** 3
    raise SystemExit(f"unknown workload {workload}")


def run_reference_steps(workload, steps):
    """Run the reference build for ``steps`` steps; returns (seconds in StepOnce, cells)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    job, cells = reference_workload_job(workload)
    job.update(steps=steps, dump_fields="U_H", dump_at=str(steps))
    d = mo.run_job(job, timeout=1800)
    secs, nsteps, ncell = d[("timing", -1)].data.ravel()
    return float(secs), int(ncell)


def cpu_baseline_sample(args):
    """The reference (built from its sources) on the host: a bounded sample of
    the same workload, single core (the reference has one thread per rank)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    if not mo.available():
        return None
    steps = args.cpu_sample_steps
    secs, ncell = run_reference_steps(args.workload, steps)
    return {"value": round(ncell * steps / secs / 1e6, 4), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{args.workload}: {steps} StepOnce calls of the reference build (oracle/_ref), "
                      f"setup excluded, 1 core"}


def run_reference(args, rank, world):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    if rank != 0:
        return None
    if not mo.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/mercury_ref is not built on this host"}
    total, cells = 0.0, 0
    steps = args.cpu_sample_steps
    for _ in range(max(1, args.warmup // 3)):
        run_reference_steps(args.workload, 1)
    times = []
    for _ in range(args.steps):
        secs, cells = run_reference_steps(args.workload, steps)
        times.append(secs)
        total += secs
    value = cells * steps * args.steps / total / 1e6
    desc = {"workload": args.workload, "steps_per_sample": steps,
            "implementation": "reference solver compiled from its own sources, single rank, 1 thread"}
    return {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / (args.steps * steps), 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": desc,
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{args.steps} x {steps} StepOnce calls"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="cube32")
    ap.add_argument("--cpu-sample-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_ours(args, rank, world, device)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
