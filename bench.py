"""Benchmark of the B200 multi-fluid Hall-MHD step (one JSON line on stdout).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (synthetic inputs generated here, seeded):
  ensemble (default)  64 independent periodic curvilinear boxes, cells per axis
           log-uniform (x, y in [24, 64], z in [24, 128]), Orszag-Tang vortex on
           two ion fluids (H+, Na+ mass 1:23), Hall + electron pressure on,
           resistivity off, CFL 0.4.  ``value``: one mixed-precision batch (one
           CUDA graph launch advances every solve by a step), K timed steps with
           the state resident in HBM (inputs larger than L2).  Beside it: the
           same solves one by one through the plain FP64 single-solve path, the
           FP64 batch, and the mixed batch's relative L2 error against FP64.
  serve    a seeded Poisson stream of requests (sizes from a pool of shapes of
           the ensemble's distribution, 50-500 steps each) served by the
           continuous-batching request loop (mixed precision) and one by one
           through the plain FP64 path: throughput and p50/p99 latency.
  cube32   one periodic curvilinear 32^3 block (the same physics), FP64 — the
           reference's own single-block test case; cubeN: N^3.

Metric: Mcell-updates/s = owned cells x steps / time (ghost cells are never
counted; "per fluid" is the same count with n_fluids = 2).  ``e2e`` is the
same metric through the C ABI from host buffers, uploads and downloads
included.

With --gpus N > 1 (torchrun), each rank runs an independent replica of the
workload (solves have no data-path exchange); ``value`` is the sum of all
replicas' cell updates over the max-over-ranks device time.

``--impl reference`` times the reference's own CPU implementation (the
reference solver compiled from its sources, oracle/_ref/mercury_ref) on a
bounded sample of the same workload on this host's cores; rank 0 only.
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

# Algorithmic HBM traffic per owned cell of each step kernel: the distinct
# field components it must read and write once per DOF, as (real-valued
# components, metric components) — mpcns_mercury_b200/csrc/mhd_kernels.cu.
# A real component is 8 B in FP64 and 4 B in mixed precision; the metric
# (Jac, JD) is 8 B in both.  Kernels over the allocated cell range count the
# allocated cells.
KERNEL_COMPS = {
    "k_face_emf": (3 + 3 + 3 + 9 + 2 + 1 + 9 + 3, 0),        # B, Badd, UCON, p x2, grad coef -> Eface, node p_e, grad p_e
    "k_edge_emf": (9 + 3 + 3 + 1 + 2 + 3, 0),                # Eface, UCON, B, node p_e, rho x2 -> E
    "k_hall_edge": (3 + 1 + 9 + 6 + 3 + 3 + 3, 0),           # EHC, beta, dr, Hall ratios, B, taper -> Ehall
    "k_add_hall": (3 + 3 + 3, 0),                            # E += Ehall
    "k_fluid": (10 + 10 + 3 + 10 + 3 + 3 + 3 + 3 + 1 + 3 + 10, 0),  # U, PV, |JD|, JD + 1/Jac, grad p_e, U+, B_cell, J_cell, Photo, xyz -> U'
    "k_bface": (3 + 3 + 3, 0),                               # B += dt curl E
    "k_bcell_jedge": (3 + 3 + 18 + 3 + 3 + 3 + 3 + 3, 0),    # B, Badd, W_B, beta, alpha -> B_cell, Bind, J edges
    "k_jcell": (3 + 36 + 3, 0),                              # J edges, W_J -> J_cell
    "k_pv_uplus": (10 + 3 + 3 + 12 + 10 + 10 + 3 + 3 + 3 + 1, 1),  # U, B_cell, J_cell, face normals, UCON coef -> PV, U+, UCON, Hall EHC, beta (+ dt); Jac
}
ALLOCATED_RANGE_KERNELS = {"k_pv_uplus"}


def kernel_bytes_per_cell(name, precision):
    real, metric = KERNEL_COMPS[name]
    return real * (4 if precision == 1 else 8) + metric * 8


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


# ------------------------------------------------------------------ ranks
def max_over_ranks(vals, device=None):
    """Element-wise maximum of ``vals`` over all ranks (identity on one rank)."""
    import torch

    dist = torch.distributed
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in vals]
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replicas_value(world, cells_per_replica, steps, max_ms):
    """Whole-job Mcell-updates/s of `world` replicas timed by the slowest rank."""
    return world * cells_per_replica * steps / (max_ms * 1e-3) / 1e6


# ------------------------------------------------------------------ workloads
def build_workload(name: str):
    """(cells per block, static+state fields {ref name: Arr}, topology kind)"""
    from mpcns_mercury_b200 import setup as S

    if name.startswith("cube"):
        n = int(name[4:])
        geom, f = S.cube_case(n)
        return [(n, n, n)], [f], (f"periodic curvilinear {n}^3 cube, Orszag-Tang on 2 ion fluids, Hall + p_e, "
                                  "CFL 0.4, FP64")
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


# Members of the magnetosphere ensemble in the default shells workload: the
# first 32 of its seeded draws (19.7 M owned cells).  A mixed-precision solve
# with the implicit resistive substep holds its FP32 fields and an FP64
# companion for the substep, about 7 KB per owned cell with the ghost layers
# (139 GB for these 32); all 64 draws (40.2 M cells) would need 283 GB.
SHELL_SOLVES = 32


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
        (total_ms,) = max_over_ranks([total_ms], device)
        torch.distributed.barrier()
    info = ctx.info()
    value = replicas_value(world, ncell, args.steps, total_ms)

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


def roofline(prof, cells, peak, peak_kind, precision=0, traffic_key=None):
    kernels = {k: v for k, v in prof.items() if k in KERNEL_COMPS}
    if not kernels:
        return None
    top = max(kernels, key=kernels.get)
    g = 4
    ncell = sum((a + 2 * g) * (b + 2 * g) * (c + 2 * g) if top in ALLOCATED_RANGE_KERNELS else a * b * c
                for a, b, c in cells)
    algo_bytes = kernel_bytes_per_cell(top, precision) * ncell
    ms = kernels[top]
    achieved = algo_bytes / (ms * 1e-3) / 1e9
    per_cell = load_traffic(traffic_key) if traffic_key and traffic_key.startswith(top + "_") else None
    traffic = int(per_cell * sum(a * b * c for a, b, c in cells)) if per_cell else None
    return {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind,
            "algo_bytes_per_launch": int(algo_bytes), "launch_ms": round(ms, 5),
            "traffic": traffic, "traffic_note": ("ncu DRAM bytes per owned cell of a captured launch (8-solve "
                                                 "ensemble) x this launch's owned cells") if per_cell else None,
            "share_of_step": round(ms / sum(prof.values()), 4)}


def load_traffic(key):
    """DRAM bytes per owned cell of a kernel from the committed ncu summary
    (profiles/dram_bytes.json), if any."""
    p = os.path.join(ROOT, "profiles", "dram_bytes.json")
    try:
        with open(p) as f:
            return float(json.load(f)[key]["bytes_per_owned_cell"])
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


# ------------------------------------------------------------------ ensemble (batched vs plain)
class _PinnedInputs:
    """One page-locked host buffer, reused for every solve's input fields."""

    def __init__(self):
        self.buf = None

    def copy(self, fields, names=UPLOAD_FIELDS):
        """Page-locked copies of fields[name] for `names` (Arr, or a plain
        array such as "nodes")."""
        import torch
        from mpcns_mercury_b200.setup import Arr

        arr = {n: (fields[n].data if isinstance(fields[n], Arr) else fields[n]) for n in names}
        need = sum(a.nbytes for a in arr.values())
        if self.buf is None or self.buf.numel() < need:
            self.buf = None
            self.buf = torch.empty(need, dtype=torch.uint8, pin_memory=True)
        raw = self.buf.numpy()
        out, off = {}, 0
        for n in names:
            a = arr[n]
            v = raw[off:off + a.nbytes].view(np.float64).reshape(a.shape)
            v[...] = a
            out[n] = Arr(fields[n].lo, fields[n].hi, v) if isinstance(fields[n], Arr) else v
            off += a.nbytes
        return out


def _owned_state(get, fields):
    """Owned DOFs of the state fields, from get(name, lo, hi)."""
    from mpcns_mercury_b200.workloads import STATE_FIELDS

    out = {}
    for name in STATE_FIELDS:
        a = fields[name]
        d = get(name, a.lo, a.hi)
        g = [-v for v in a.lo]
        out[name] = d[g[0]:a.hi[0], g[1]:a.hi[1], g[2]:a.hi[2]].copy()
    return out


def _rel_l2(a, b):
    den = float(np.sqrt(np.sum(b * b)))
    return float(np.sqrt(np.sum((a - b) ** 2))) / (den if den > 0 else 1.0)


def _batch_step_profile(batch, nsteps):
    import ctypes
    from mpcns_mercury_b200.capi import check, lib

    ms = (ctypes.c_float * 256)()
    names = (ctypes.c_char_p * 256)()
    n = ctypes.c_int()
    check(lib().mhd_batch_step_profiled(batch.b, nsteps, 256, ms, names, ctypes.byref(n)), "mhd_batch_step_profiled")
    out = {}
    for q in range(n.value):
        key = names[q].decode()
        out[key] = out.get(key, 0.0) + ms[q]
    return out


def _timed_batch_steps(batch, steps, device):
    """Device time (ms) of ``steps`` graph launches on the batch's stream."""
    import torch

    stream = torch.cuda.ExternalStream(batch.stream(), device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ensemble(args, rank, world, device):
    """64 independent periodic-box solves of uneven sizes, advanced together by
    one batch in mixed precision, against the same solves run one by one through
    the plain FP64 single-solve path."""
    import torch
    from mpcns_mercury_b200 import Context, reference_constants
    from mpcns_mercury_b200 import setup as S
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    nsol = args.solves
    sizes = W.ensemble_sizes(nsol)
    base_id = rank * nsol
    cells = [tuple(c) for c in sizes]
    ncell = owned_cells(cells)
    W_, K = args.warmup, args.steps
    total_steps = W_ + K
    err_steps = max(total_steps, args.error_steps)  # the mixed error is stated after this many steps
    k0 = reference_constants(cfl=0.4)
    batches = {1: Batch(nsol, 1), 0: Batch(nsol, 0)}
    slots = {1: [], 0: []}
    plain_ms = 0.0
    plain_state = []
    only = getattr(args, "batched_only", False)
    if only:
        batches[0].close()
        del batches[0]
    # setup outside every timed region: device memory for all solves reserved
    # in each batch's pool (the reference likewise allocates at setup)
    for prec, b in batches.items():
        need = 0
        for n in cells:
            d = SolveDesc([n], 4, k0, precision=prec)
            need += d.device_bytes()
            d.close()
        b.reserve(need)
    pin, pin_nodes = _PinnedInputs(), _PinnedInputs()
    for sid, fields in enumerate(W.generate_cases([(c, base_id + s) for s, c in enumerate(cells)])):
        n = cells[sid]
        # the inputs in page-locked host memory (not timed): every field for
        # the FP64 batch (bitwise against the plain path); the block's nodes
        # and the state for the mixed batch, whose static fields are computed
        # on the device (mhd_batch_setup_geometry) inside the timed region
        pinned = pin.copy(fields)
        _, nx, ny, nz = S.cube_nodes(n)
        node_inputs = pin_nodes.copy({"nodes": np.stack([nx, ny, nz], axis=-1), **{k: fields[k] for k in W.STATE_FIELDS}},
                                     names=["nodes"] + W.STATE_FIELDS)
        for prec, b in batches.items():
            # FP64: host topology as explicit copy lists (setup, not timed), the
            # reference-format path; mixed: the periodic tables compiled directly
            d = SolveDesc([n], 4, k0, precision=prec) if prec == 0 else None
            slot = b.add(d) if prec == 0 else b.add_periodic(n, 4, k0)
            if prec == 1:
                nb = W.upload_request(lambda f, a, lo, hi, blk: b.upload(slot, f, a, lo, hi, block=blk),
                                      lambda nodes: b.setup_geometry(slot, nodes), node_inputs)
            else:
                nb = W.upload_case(lambda f, a, lo, hi, blk: b.upload(slot, f, a, lo, hi, block=blk), pinned)
            b.sync(slot, "UCELL")
            b.sync(slot, "BFACE")
            b.prepare(slot)
            b.request(slot, err_steps)
            slots[prec].append(slot)
            if d is not None:
                d.close()
        if only:
            continue
        # plain FP64, this solve alone
        ctx = Context([n], 4, k0)
        W.upload_case(lambda f, a, lo, hi, blk: ctx.upload(f, a, lo, hi, block=blk), fields)
        ctx.sync("UCELL")
        ctx.sync("BFACE")
        ctx.prepare()
        ctx.step(W_)
        stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step_async(K)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
        if err_steps > total_steps:
            ctx.step_async(err_steps - total_steps)  # untimed: on to the error check's step count
        ctx.synchronize()
        plain_state.append((fields, _owned_state(lambda nm, lo, hi: ctx.download(W.capi_field(nm), lo, hi), fields)))
        ctx.close()
        del fields

    # batched runs: W untimed launches, then K timed (inputs >> L2)
    for prec, b in batches.items():
        b.run(W_)
        b.poll()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(device.index if device.index is not None else 0)
    if rank == 0:
        sampler.start()
    mixed_ms = _timed_batch_steps(batches[1], K, device)
    clocks = sampler.stop() if rank == 0 else None
    if only:
        ms = mixed_ms
        batches[1].close()
        return {"metric": METRIC, "value": round(world * ncell * K / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
                "n_gpus": world, "steps": K, "warmup": W_, "ms_per_step": round(ms / K, 5),
                "config": {"workload": "ensemble", "solves": nsol, "batched_only": True}}
    fp64_ms = _timed_batch_steps(batches[0], K, device)
    for b in batches.values():  # untimed: on to the error check's step count
        if err_steps > total_steps:
            b.run(err_steps - total_steps)
    infos = {p: b.poll() for p, b in batches.items()}
    for p in batches:
        for s in slots[p]:
            if infos[p][s].status != 0 or infos[p][s].step != err_steps:
                raise RuntimeError(f"batch precision {p} slot {s}: status {infos[p][s].status} step {infos[p][s].step}")
    if world > 1:
        mixed_ms, fp64_ms, plain_ms = max_over_ranks([mixed_ms, fp64_ms, plain_ms], device)

    # errors: mixed batch vs plain FP64 (the FP64 path equals the reference bitwise),
    # and FP64 batch vs plain FP64 (must be identical)
    worst = {}
    fp64_identical = True
    for sid, (fields, ref) in enumerate(plain_state):
        got = _owned_state(lambda nm, lo, hi: batches[1].download(slots[1][sid], W.capi_field(nm), lo, hi), fields)
        for name in ref:
            worst[name] = max(worst.get(name, 0.0), _rel_l2(got[name], ref[name]))
        if sid < 8:  # the FP64 batch on a sample of solves
            got64 = _owned_state(lambda nm, lo, hi: batches[0].download(slots[0][sid], W.capi_field(nm), lo, hi),
                                 fields)
            fp64_identical = fp64_identical and all(np.array_equal(got64[k], ref[k]) for k in ref)

    value = replicas_value(world, ncell, K, mixed_ms)
    plain = replicas_value(world, ncell, K, plain_ms)
    batched64 = replicas_value(world, ncell, K, fp64_ms)
    for s_ in slots[1]:
        batches[1].request(s_, 3)  # every solve active for the profiled steps
    prof = _batch_step_profile(batches[1], 3)
    peak, peak_kind = load_peaks()
    roof = roofline(prof, cells, peak, peak_kind, precision=1, traffic_key="k_fluid_mixed_ensemble")
    launches = batches[1].kernels_per_step()
    for b in batches.values():
        b.close()
    e2e = run_e2e_batch(cells, base_id, W_, K, world)
    cpu = cpu_baseline_sample(args, cells) if (rank == 0 and not args.no_cpu_baseline) else None
    return {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W_,
        "ms_per_step": round(mixed_ms / K, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (metric f64)", "data": "synthetic",
        "config": {"workload": "ensemble", "solves": nsol, "description":
                   f"{nsol} independent periodic curvilinear boxes (Orszag-Tang, 2 ion fluids, Hall + p_e), "
                   "cells per axis log-uniform x,y in [24,64], z in [24,128], one block each, seeded noise per "
                   "solve; one batch, one CUDA graph launch per step advancing every solve",
                   "cells_per_replica": ncell, "precision": "mixed: FP32 state/work/flux/EMF/update, FP64 Jac/JD",
                   "l2": "inputs larger than L2 (not flushed)", "parallelism": f"replicas x{world}",
                   "plain_fp64_one_by_one_mcells": round(plain, 3),
                   "batched_fp64_mcells": round(batched64, 3),
                   "batched_mixed_vs_plain_fp64": round(value / plain, 3),
                   "batched_fp64_vs_plain_fp64": round(batched64 / plain, 3),
                   "error_vs_fp64_rel_l2_max_over_solves": {k: float(f"{v:.3e}") for k, v in worst.items()},
                   "error_steps": err_steps, "fp64_batch_bitwise_equal_plain": bool(fp64_identical)},
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches * K, "clocks": clocks,
        "kernel_ms": {k: round(v, 5) for k, v in prof.items()},
    }


def run_e2e_batch(cells, base_id, W_, K, world):
    """The mixed batch end to end through the C ABI, timed as one wall-clock
    region: from page-locked host inputs (each solve's block nodes and initial
    state), add every solve (sync tables compiled from the periodic
    connectivity), compute its static fields on the device from the nodes,
    upload the state, prepare, run W + K steps, and download every solve's
    final state to host memory.  The device memory reservation of the batch
    happens before the timed region (the reference arm times StepOnce only)."""
    import torch
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.capi import Batch, SolveDesc

    k0 = reference_constants(cfl=0.4)
    inputs = W.state_cases([(c, base_id + s) for s, c in enumerate(cells)])
    pinned = []
    for inp in inputs:  # page-locked copies of the host inputs (not timed)
        pf = {}
        for name, a in inp.items():
            arr = a.data if hasattr(a, "data") and not isinstance(a, np.ndarray) else a
            t = torch.empty(arr.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = arr
            pf[name] = t.numpy() if isinstance(a, np.ndarray) else type(a)(a.lo, a.hi, t.numpy())
        pinned.append(pf)
    del inputs
    batch = Batch(len(cells), 1)
    need = 0
    for n in cells:
        d = SolveDesc([n], 4, k0, precision=1)
        need += d.device_bytes()
        d.close()
    batch.reserve(need)
    torch.cuda.synchronize()
    h2d = d2h = 0
    t0 = time.perf_counter()
    slots = []
    for n, pf in zip(cells, pinned):
        slot = batch.add_periodic(n, 4, k0)
        h2d += W.upload_request(lambda f, a, lo, hi, blk: batch.upload(slot, f, a, lo, hi, block=blk),
                                lambda nodes: batch.setup_geometry(slot, nodes), pf)
        batch.sync(slot, "UCELL")
        batch.sync(slot, "BFACE")
        batch.prepare(slot)
        batch.request(slot, W_ + K)
        slots.append(slot)
    batch.run(W_ + K)
    info = batch.poll()
    for slot, pf in zip(slots, pinned):
        for name in W.STATE_FIELDS:
            a = pf[name]
            d2h += batch.download(slot, W.capi_field(name), a.lo, a.hi).nbytes
    t1 = time.perf_counter()
    ok = all(info[s].status == 0 and info[s].step == W_ + K for s in slots)
    batch.close()
    if not ok:
        raise RuntimeError("e2e batch: a solve did not finish its steps")
    ncell = owned_cells(cells)
    return {"value": round(world * ncell * (W_ + K) / (t1 - t0) / 1e6, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / (W_ + K)), "d2h_bytes_per_step": int(d2h / (W_ + K)),
            "wall_s": round(t1 - t0, 4), "steps": W_ + K,
            "what": "one wall-clock region: add of every solve (mhd_batch_add_periodic), its static fields "
                    "computed on the device from the uploaded nodes (mhd_batch_setup_geometry), upload of the "
                    "initial state, prepare, W+K steps, download of every final state, all through the C ABI "
                    "from page-locked host arrays"}


# ------------------------------------------------------------------ magnetosphere shells (batched vs plain)
SHELL_STATE = (("U_H", (0, 0, 0)), ("U_NA", (0, 0, 0)), ("B_XI", (1, 0, 0)), ("B_ETA", (0, 1, 0)),
               ("B_ZETA", (0, 0, 1)))


def _shell_state(get, case, dtype=np.float64):
    """Owned DOFs of the state fields of every panel, from get(field, lo, hi, block)."""
    n = (case.na, case.na, case.nr)
    out = {}
    for name, st in SHELL_STATE:
        hi = tuple(n[a] + st[a] for a in range(3))
        out[name] = np.concatenate([get(name, (0, 0, 0), hi, b).astype(dtype).ravel() for b in range(6)])
    return out


def _flux_divergence(ctx, case):
    """max over the owned cells of |sum of the induced field's outward face
    fluxes|, over the largest face flux of the total field (induced + dipole
    + IMF background): the constrained transport's div B in units of the
    field it transports."""
    n0, n1, n2 = case.na, case.na, case.nr
    worst, big = 0.0, 0.0
    for blk in range(6):
        f = {}
        for ax, name in enumerate(("B_XI", "B_ETA", "B_ZETA")):
            hi = [n0, n1, n2]
            hi[ax] += 1
            f[ax] = ctx.download(name, (0, 0, 0), tuple(hi), block=blk)[..., 0]
            tot = f[ax] + ctx.download("BADD" + name[1:], (0, 0, 0), tuple(hi), block=blk)[..., 0]
            big = max(big, float(np.abs(tot).max()))
        div = (f[0][1:] - f[0][:-1]) + (f[1][:, 1:] - f[1][:, :-1]) + (f[2][:, :, 1:] - f[2][:, :, :-1])
        worst = max(worst, float(np.abs(div).max()))
    return worst / max(big, 1e-300)


def _shell_descs(cases, ks, topo, precision):
    from mpcns_mercury_b200.capi import SolveDesc

    return [SolveDesc(c.cells, 4, k, precision=precision, topology=topo.get(c)) for c, k in zip(cases, ks)]


def _shell_batch(cases, ks, topo, precision, steps):
    """A batch holding the cases, set up on the device, prepared, each with
    ``steps`` steps requested.  Returns (batch, slots)."""
    from mpcns_mercury_b200 import magnetosphere as M
    from mpcns_mercury_b200.capi import Batch

    b = Batch(len(cases), precision)
    descs = _shell_descs(cases, ks, topo, precision)
    b.reserve(sum(d.device_bytes() for d in descs))
    slots = []
    for c, k, d in zip(cases, ks, descs):
        s = b.add(d)
        d.close()
        M.set_up(b, c, slot=s, k=k)
        b.prepare(s)
        b.request(s, steps)
        slots.append(s)
    return b, slots


def _check_batch(b, slots, steps, what):
    info = b.poll()
    for s in slots:
        if info[s].status != 0 or info[s].step != steps:
            raise RuntimeError(f"{what} slot {s}: status {info[s].status} step {info[s].step}")


def run_shells(args, rank, world, device):
    """The magnetosphere ensemble (64 cubed-sphere shells of uneven sizes and
    seeded upstream conditions) advanced together by one mixed-precision
    batch, against the same solves one by one through the plain FP64 path."""
    import torch
    from mpcns_mercury_b200 import magnetosphere as M

    nsol = args.solves
    cases = M.ensemble(nsol, stream=300000 + 1000 * rank)
    ks = [M.constants(c) for c in cases]
    cells = [n for c in cases for n in c.cells]
    ncell = owned_cells(cells)
    W_, K = args.warmup, args.steps
    total = W_ + K
    # the mixed error is stated after the configuration's step count (not
    # needed when only the batch is profiled)
    err_steps = total if getattr(args, "batched_only", False) else max(total, args.error_steps)
    topo = M.TopologyCache()
    t0 = time.perf_counter()
    for c in cases:  # the grids' sync tables (host, shared by every solve of one grid; not timed)
        topo.get(c)
    topo_s = time.perf_counter() - t0

    # 1) the mixed-precision batch: its fluid tile picked by the autotuner on
    # the batch itself, W untimed steps, K timed (state >> L2), on to err_steps
    from mpcns_mercury_b200 import autotune

    mixed, slots = _shell_batch(cases, ks, topo, 1, err_steps)
    if getattr(args, "cg_host_loop", False):  # profiling: the CG iterations as plain launches
        mixed.cg_host_loop(True)
    tune_mixed = autotune.tune(mixed, 1, cells, reps=3, cache=None)
    mixed.run(W_)
    mixed.poll()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(device.index if device.index is not None else 0)
    if rank == 0:
        sampler.start()
    mixed.substep_ms()  # restart the substep's count
    mixed_ms = _timed_batch_steps(mixed, K, device)
    mixed_substep = mixed.substep_ms()
    clocks = sampler.stop() if rank == 0 else None
    if err_steps > total:
        mixed.run(err_steps - total)
    _check_batch(mixed, slots, err_steps, "mixed batch")
    # the mixed state is FP32 on the device: kept as float32 on the host, exactly
    mixed_state = [_shell_state(lambda f, lo, hi, blk: mixed.download(s, f, lo, hi, block=blk), c, np.float32)
                   for s, c in zip(slots, cases)]
    for s in slots:
        mixed.request(s, 3)  # every solve active for the profiled steps
    prof = _batch_step_profile(mixed, 3)
    launches = mixed.kernels_per_step()
    mixed.close()
    if getattr(args, "batched_only", False):
        topo.close()
        return {"metric": METRIC, "value": round(replicas_value(world, ncell, K, mixed_ms), 3), "unit": UNIT,
                "n_gpus": world, "steps": K, "warmup": W_, "ms_per_step": round(mixed_ms / K, 5),
                "config": {"workload": "shells", "solves": nsol, "batched_only": True,
                           "implicit_substep_ms_per_step": round(mixed_substep, 4),
                           "autotune_fluid_tile": {"mixed": _tune_summary(tune_mixed)}},
                "kernel_ms": {k: round(v, 5) for k, v in prof.items()}}

    # 2) plain FP64, one solve at a time: W untimed, K timed, on to err_steps
    plain_ms = []
    worst = {}
    worst_tot = {}
    sub_bytes, nsub = 0, 0
    for c, k in zip(cases, ks):  # the FP64 batch's subset: the first solves within 40 GB
        d = _shell_descs([c], [k], topo, 0)[0]
        if sub_bytes + d.device_bytes() > 40e9 and nsub > 0:
            d.close()
            break
        sub_bytes += d.device_bytes()
        nsub += 1
        d.close()
    plain_sub = []
    # the FP64 fluid tile, picked by the autotuner on the subset's FP64 batch
    # (used by the plain path and the FP64 batch alike)
    tb, _ = _shell_batch(cases[:nsub], ks[:nsub], topo, 0, 1)
    tune64 = autotune.tune(tb, 0, cells, reps=3, cache=None)
    tb.close()
    tile64 = tune64["variant"]
    for i, (c, k) in enumerate(zip(cases, ks)):
        ctx = M.context(c, precision=0, k=k, topologies=topo)
        ctx.fluid_tile(tile64)
        ctx.step(W_)
        stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step_async(K)
        e1.record(stream)
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
        if err_steps > total:
            ctx.step_async(err_steps - total)
        ctx.synchronize()
        info = ctx.info()
        if info.status != 0 or info.step != err_steps:
            raise RuntimeError(f"plain FP64 solve {i}: status {info.status} step {info.step}")
        st = _shell_state(lambda f, lo, hi, blk: ctx.download(f, lo, hi, block=blk), c)
        for name in st:
            worst[name] = max(worst.get(name, 0.0), _rel_l2(mixed_state[i][name].astype(np.float64), st[name]))
        # the induced field's error against the total field (induced + dipole + IMF background)
        badd = _shell_state(lambda f, lo, hi, blk: ctx.download(f.replace("B_", "BADD_"), lo, hi, block=blk)
                            if f.startswith("B_") else np.zeros(1), c)
        for name in ("B_XI", "B_ETA", "B_ZETA"):
            tot = st[name] + badd[name]
            e = float(np.linalg.norm(mixed_state[i][name].astype(np.float64) - st[name])) / max(
                float(np.linalg.norm(tot)), 1e-300)
            worst_tot[name] = max(worst_tot.get(name, 0.0), e)
        if i < nsub:
            plain_sub.append(st)
        ctx.close()
    del mixed_state

    # 3) the FP64 batch on the subset: its rate, and bitwise equality with the plain path
    fp64, fslots = _shell_batch(cases[:nsub], ks[:nsub], topo, 0, err_steps)
    fp64.fluid_tile(tile64)
    fp64.run(W_)
    fp64.poll()
    fp64_ms = _timed_batch_steps(fp64, K, device)
    if err_steps > total:
        fp64.run(err_steps - total)
    _check_batch(fp64, fslots, err_steps, "FP64 batch")
    fp64_identical = True
    for i, (s, c) in enumerate(zip(fslots, cases[:nsub])):
        got = _shell_state(lambda f, lo, hi, blk: fp64.download(s, f, lo, hi, block=blk), c)
        fp64_identical = fp64_identical and all(np.array_equal(got[n], plain_sub[i][n]) for n in got)
    fp64.close()
    del plain_sub
    sub_cells = sum(c.cell_count() for c in cases[:nsub])
    if world > 1:
        mixed_ms, plain_total, fp64_ms, plain_sub_ms = max_over_ranks(
            [mixed_ms, sum(plain_ms), fp64_ms, sum(plain_ms[:nsub])], device)
    else:
        plain_total, plain_sub_ms = sum(plain_ms), sum(plain_ms[:nsub])

    value = replicas_value(world, ncell, K, mixed_ms)
    plain = replicas_value(world, ncell, K, plain_total)
    batched64 = replicas_value(world, sub_cells, K, fp64_ms)
    plain_sub_rate = replicas_value(world, sub_cells, K, plain_sub_ms)
    peak, peak_kind = load_peaks()
    roof = roofline(prof, cells, peak, peak_kind, precision=1, traffic_key="k_fluid_mixed_shells")
    e2e = run_e2e_shells(cases, ks, topo, err_steps, world, tune_mixed["variant"])
    topo.close()
    serving = None
    if args.serve_requests > 0:  # a short request stream of the same physics: p50/p99 beside the throughput
        items = M.request_stream(args.serve_requests, args.serve_rate, 8, 48, 96, 50, 100,
                                 stream=500000 + 1000 * rank)
        sb, sp, _ = serve_shells(items, args.serve_requests, args.hbm_budget,
                                 fluid_tiles=(tune_mixed["variant"], tile64), shapes=8)
        sb.pop("latencies")
        sp.pop("latencies")
        serving = {"requests": args.serve_requests, "arrival_rate_per_s": args.serve_rate,
                   "grids": "8 shell sizes, na log-uniform in [24,48], nr in [24,96]; 50-100 steps per request; "
                            "upstream conditions per request as the ensemble's",
                   "batched_mixed": _round_stats(sb), "plain_fp64_one_by_one": _round_stats(sp),
                   "latency_p50_s": round(sb["latency_p50_s"], 4), "latency_p99_s": round(sb["latency_p99_s"], 4),
                   "throughput_batched_vs_one_by_one": round(sb["mcell_updates_per_s"] / sp["mcell_updates_per_s"],
                                                             3)}
    cpu = cpu_baseline_sample(args) if (rank == 0 and not args.no_cpu_baseline) else None
    return {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W_,
        "ms_per_step": round(mixed_ms / K, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (metric f64)", "data": "synthetic",
        "config": {"workload": "shells", "solves": nsol, "description":
                   f"{nsol} magnetosphere solves: 6-panel cubed-sphere shells r in [1, 8] (r geometric), cells per "
                   "panel axis log-uniform (na in [24,64], nr in [24,128]), H+ and Na+ (mass 1:23) with Na+ "
                   "fraction U[1e-4,1e-2], centred dipole, upstream |v| U[2,6], n U[0.5,3], IMF Bz U[-0.4,0.4], "
                   "Hall (radial taper 1.1-1.2) + electron pressure, solid inner wall, farfield outer sphere, "
                   "implicit resistivity eta = 1e-3 exp(-(r - 1) / 0.2) (the reference's tanh window, outer edge 1, "
                   "width 0.4), CG to 1e-10, CFL 0.4; set up on the device from these parameters; one batch: per "
                   "step one CUDA graph for the explicit part of every solve, the implicit substep of every solve "
                   "at once (one device CG loop; in the mixed batch FP64 CG on the solves' FP64 companions), one "
                   "graph for the rest",
                   "cells_per_replica": ncell, "blocks_per_replica": len(cells),
                   "precision": "mixed: FP32 state/work/flux/EMF/update, FP64 Jac/JD",
                   "l2": "inputs larger than L2 (not flushed)", "parallelism": f"replicas x{world}",
                   "plain_fp64_one_by_one_mcells": round(plain, 3),
                   "batched_mixed_vs_plain_fp64": round(value / plain, 3),
                   "batched_fp64_subset": {"solves": nsub, "cells": sub_cells, "mcells": round(batched64, 3),
                                           "plain_fp64_same_solves_mcells": round(plain_sub_rate, 3),
                                           "bitwise_equal_plain": bool(fp64_identical)},
                   "error_vs_fp64_rel_l2_max_over_solves": {k: float(f"{v:.3e}") for k, v in worst.items()},
                   "error_vs_fp64_of_B_relative_to_total_field": {k: float(f"{v:.3e}") for k, v in worst_tot.items()},
                   "implicit_substep_ms_per_step": {"mixed_batch": round(mixed_substep, 4)},
                   "error_steps": err_steps, "host_topology_build_s": round(topo_s, 2),
                   "autotune_fluid_tile": {"mixed": _tune_summary(tune_mixed), "fp64": _tune_summary(tune64)}},
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": e2e, "serving": serving,
        "latency_p50_s": serving["latency_p50_s"] if serving else None,
        "latency_p99_s": serving["latency_p99_s"] if serving else None,
        "gpu_launches": launches * K, "clocks": clocks,
        "kernel_ms": {k: round(v, 5) for k, v in prof.items()},
    }


def _tune_summary(t):
    from mpcns_mercury_b200.capi import fluid_tile_shape

    return {"pick": t["variant"], "shape_k_j_i_ctas": list(t["shape"]),
            "ms_per_fluid_pass": [round(v, 4) for v in t["ms"]] if t["ms"] else None,
            "variants": [list(fluid_tile_shape(v)) for v in range(len(t["ms"] or []))],
            "gain_over_default": round(t["ms"][0] / t["ms"][t["variant"]], 4) if t["ms"] else None}


def run_config2(args, rank, world, device):
    """The magnetosphere configuration itself: one 6 x 48x48x96 shell with the
    implicit resistive substep, 200 steps in plain FP64 (the reference's
    arithmetic, bit for bit in its explicit part), then its mixed-precision
    form with the error against the FP64 run after the same steps and div B
    of both."""
    import torch
    from mpcns_mercury_b200 import magnetosphere as M

    steps = args.config_steps
    # eta = 1e-3 exp(-(r - 1) / 0.2) (units of mu0 U_ref L_ref) as the
    # reference's tanh window (magnetosphere.ETA_CONFIG)
    case = M.ShellCase(na=48, nr=96, resistive=True, **M.ETA_CONFIG)
    out = {}
    states = {}
    # FP64; mixed with the substep's policy (FP64 CG on the companion while
    # solves are short); mixed with iterative refinement throughout (FP32 CG
    # corrections of FP64 residuals, the configuration's stated method)
    for prec in (0, 1, "refined"):
        k = M.constants(case)
        if prec == "refined":
            k.res_direct_iters = -1
        ctx = M.context(case, precision=0 if prec == 0 else 1, k=k)
        ctx.step(args.warmup)
        stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        ctx.step(steps)  # the implicit substep's CG synchronises with the host once per step
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        info = ctx.info()
        if info.status != 0:
            raise RuntimeError(f"config2 precision {prec}: status {info.status}")
        states[prec] = _shell_state(lambda f, lo, hi, blk: ctx.download(f, lo, hi, block=blk), case)
        out[prec] = {"mcells": round(case.cell_count() * steps / (ms * 1e-3) / 1e6, 3), "ms_per_step": round(ms / steps, 4),
                     "div_b_max": ctx.div_b(), "div_b_flux_sum_over_max_face_flux": _flux_divergence(ctx, case),
                     "last_substep_cg_iterations": int(info.res_iters),
                     "last_substep_refinements": int(info.res_refinements),
                     "last_substep_relative_residual": float(info.res_relres)}
        ctx.close()
    err = {n: float(f"{_rel_l2(states[1][n], states[0][n]):.3e}") for n in states[0]}
    err_ref = {n: float(f"{_rel_l2(states['refined'][n], states[0][n]):.3e}") for n in states[0]}
    return {
        "metric": METRIC, "value": out[0]["mcells"], "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": out[0]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "config2", "description":
                   "one magnetosphere shell, 6 panels of 48x48x96 cells (r in [1, 8], geometric), H+ and Na+ (1e-3), "
                   "centred dipole, upstream |v| 4, n 1, p 0.1, IMF Bz -0.2, Hall + p_e, implicit resistivity "
                   "eta = 1e-3 exp(-(r - 1) / 0.2) as the reference's tanh window (outer edge 1, width 0.4, inner 0: "
                   "equal for r - 1 >> 0.2, half at the surface), CG to 1e-10, CFL 0.4; set up on the device",
                   "cells": case.cell_count(), "fp64": out[0], "mixed": out[1],
                   "mixed_vs_fp64_rel_l2_after_steps": err,
                   "mixed_refined": out["refined"], "mixed_refined_vs_fp64_rel_l2_after_steps": err_ref},
    }


def run_e2e_shells(cases, ks, topo, steps, world, fluid_tile=0):
    """The mixed batch end to end through the C ABI, one wall-clock region:
    add every solve (its grid's sync tables, built ahead like a grid file),
    its static fields and background computed on the device from the
    page-locked node coordinates, the initial state filled on the device,
    prepare, ``steps`` steps (the configuration's per-solve count), download
    of every solve's final state."""
    import torch
    from mpcns_mercury_b200 import magnetosphere as M
    from mpcns_mercury_b200.capi import Batch, shell_grid

    pinned = []
    for c in cases:
        g = shell_grid(c.na, c.nr, c.r_out, M.NGHOST + 1)
        t = torch.empty(g.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = g
        pinned.append(t.numpy())
    descs = _shell_descs(cases, ks, topo, 1)
    b = Batch(len(cases), 1)
    b.reserve(sum(d.device_bytes() for d in descs))
    b.fluid_tile(fluid_tile)  # the autotuner's pick for this workload
    torch.cuda.synchronize()
    h2d = d2h = 0
    t0 = time.perf_counter()
    slots = []
    for c, k, d, nodes in zip(cases, ks, descs, pinned):
        s = b.add(d)
        h2d += M.set_up(b, c, slot=s, k=k, nodes=nodes)
        b.prepare(s)
        b.request(s, steps)
        slots.append(s)
    b.run(steps)
    info = b.poll()
    for s, c in zip(slots, cases):
        st = _shell_state(lambda f, lo, hi, blk: b.download(s, f, lo, hi, block=blk), c)
        d2h += sum(v.nbytes for v in st.values())
    t1 = time.perf_counter()
    for d in descs:
        d.close()
    ok = all(info[s].status == 0 and info[s].step == steps for s in slots)
    b.close()
    if not ok:
        raise RuntimeError("e2e batch: a solve did not finish its steps")
    ncell = sum(c.cell_count() for c in cases)
    return {"value": round(world * ncell * steps / (t1 - t0) / 1e6, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": int(d2h / steps),
            "wall_s": round(t1 - t0, 4), "steps": steps,
            "what": "one wall-clock region: add of every solve (its grid's sync tables, built on the host ahead "
                    "like a grid file), static fields and background computed on the device from page-locked "
                    "node coordinates (mhd_batch_setup_geometry_bg, Sync(Badd)), initial state filled on the "
                    "device, Sync(U), Sync(B), prepare, the configuration's steps per solve, download of every "
                    "final state, all through the C ABI"}


# ------------------------------------------------------------------ serving
def run_serving(args, rank, world, device):
    """Poisson request stream served by the continuous-batching server
    (mixed precision) and, for comparison, one by one through the plain FP64
    path."""
    from mpcns_mercury_b200 import serving as SV
    from mpcns_mercury_b200 import workloads as W
    from mpcns_mercury_b200.setup import Uniform

    nreq = args.requests
    shapes = W.ensemble_sizes(args.shapes, stream=200000 + rank)
    # each shape's request carries its nodes and initial state; the server
    # computes the static fields on the device when the shape first arrives
    pool = W.state_cases([(c, 300000 + rank * 1000 + i) for i, c in enumerate(shapes)])
    u = Uniform(400000 + rank).sym(0.5, 3 * nreq) + 0.5
    t = 0.0
    reqs = []
    for q in range(nreq):
        t += -np.log(1.0 - u[3 * q]) / args.rate           # exponential inter-arrival times
        shape = min(int(u[3 * q + 1] * args.shapes), args.shapes - 1)
        steps = 50 + min(int(u[3 * q + 2] * 451), 450)      # 50 .. 500
        reqs.append(SV.Request(rid=q, arrival_s=t, cells=tuple(shapes[shape]), steps=steps, fields=pool[shape]))
    srv = SV.Server(capacity=args.capacity, precision=1, hbm_budget=args.hbm_budget)
    batched = srv.serve(reqs)
    srv.close()
    for r in reqs:
        r.done_s = float("nan")
    plain = SV.serve_one_by_one(reqs, precision=0)
    line = {
        "metric": METRIC, "value": round(batched["mcell_updates_per_s"] * world, 3), "unit": UNIT, "n_gpus": world,
        "steps": int(sum(r.steps for r in reqs)), "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (metric f64)", "data": "synthetic",
        "config": {"workload": "serve", "requests": nreq, "arrival_rate_per_s": args.rate, "shapes": args.shapes,
                   "capacity": args.capacity, "hbm_budget_bytes": args.hbm_budget,
                   "batched_mixed": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in batched.items()},
                   "plain_fp64_one_by_one": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in plain.items()},
                   "latency_p50_s": round(batched["latency_p50_s"], 4),
                   "latency_p99_s": round(batched["latency_p99_s"], 4)},
        "roofline": None, "cpu_baseline": None,
        "e2e": {"value": round(batched["mcell_updates_per_s"] * world, 3), "unit": UNIT,
                "what": "wall clock of the whole request loop, uploads and downloads included"},
    }
    return line


def serve_shells(items, capacity, hbm_budget, fluid_tiles=(0, 0), shapes=16):
    """Magnetosphere requests [(arrival_s, ShellCase, steps)] served by the
    continuous-batching server (mixed precision) and one by one through the
    plain FP64 path (one context per grid, each request's fields set up on
    the device).  Returns (batched stats, plain stats, requests)."""
    import torch
    from mpcns_mercury_b200 import capi
    from mpcns_mercury_b200 import magnetosphere as M
    from mpcns_mercury_b200 import serving as SV

    reqs = [SV.Request(rid=q, arrival_s=t, cells=None, steps=st, fields={}, case=c)
            for q, (t, c, st) in enumerate(items)]
    # the grids' tables and nodes, prepared ahead for both (host setup, like grid files read ahead)
    topo, nodes = M.TopologyCache(), {}
    for r in reqs:
        topo.get(r.case)
        key = ("shell", r.case.na, r.case.nr, bool(r.case.resistive))
        if key not in nodes:
            nodes[key] = capi.shell_grid(r.case.na, r.case.nr, r.case.r_out, M.NGHOST + 1)
    srv = SV.Server(capacity=capacity, precision=1, hbm_budget=hbm_budget, max_grids=max(shapes, len(nodes)),
                    topologies=topo, nodes=nodes)
    srv.batch.fluid_tile(fluid_tiles[0])
    dist = torch.distributed
    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    if multi:
        dist.barrier()  # the ranks' request clocks start together
    batched = srv.serve(reqs)
    srv.close()
    batched["latencies"] = [r.done_s - r.arrival_s for r in reqs]
    for r in reqs:
        r.done_s = float("nan")
    if multi:
        dist.barrier()
    plain = SV.serve_one_by_one(reqs, precision=0, topologies=topo, nodes=nodes, fluid_tile=fluid_tiles[1])
    plain["latencies"] = [r.done_s - r.arrival_s for r in reqs]
    topo.close()
    return batched, plain, reqs


def run_serving_shells(args, rank, world, device):
    """The serving configuration on magnetosphere requests: a seeded Poisson
    stream (``--requests``, ``--rate``), sizes log-uniform up to
    6 x 96 x 96 x 192 from ``--shapes`` grids, 50-500 steps each, served by the
    continuous-batching server (mixed) and one by one (plain FP64)."""
    from mpcns_mercury_b200 import magnetosphere as M
    from mpcns_mercury_b200.distributed import aggregate, partition

    # one stream for the whole job, each rank serving its own partition
    stream = M.request_stream(args.requests, args.rate, args.shapes, 96, 192, 50, 500, stream=500000)
    mine = partition([c.cell_count() * st for _, c, st in stream], world)[rank]
    sb, sp, reqs = serve_shells([stream[q] for q in mine], args.capacity, args.hbm_budget, shapes=args.shapes)
    sb = aggregate(sb, sb.pop("latencies"))
    sp = aggregate(sp, sp.pop("latencies"))
    return {
        "metric": METRIC, "value": round(sb["mcell_updates_per_s"], 3), "unit": UNIT, "n_gpus": world,
        "steps": int(sum(r.steps for r in reqs)), "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (metric f64)", "data": "synthetic",
        "config": {"workload": "serve-shells", "requests": args.requests, "arrival_rate_per_s": args.rate,
                   "grids": args.shapes, "capacity": args.capacity, "hbm_budget_bytes": args.hbm_budget,
                   "parallelism": f"request stream partitioned over {world} rank(s) (longest first)",
                   "batched_mixed": _round_stats(sb), "plain_fp64_one_by_one": _round_stats(sp)},
        "latency_p50_s": round(sb["latency_p50_s"], 4), "latency_p99_s": round(sb["latency_p99_s"], 4),
        "roofline": None, "cpu_baseline": None,
        "e2e": {"value": round(sb["mcell_updates_per_s"], 3), "unit": UNIT,
                "what": "wall clock of the whole request loop: per request its fields set up on the device from "
                        "its parameters, its steps, its slot freed"},
    }


def _round_stats(d):
    return {k: (round(v, 4) if isinstance(v, float) else v) for k, v in d.items()}


# ------------------------------------------------------------------ implicit substep
# Algorithmic bytes of one CG iteration per unknown: about 21 words touched
# per edge unknown (the operator's E from p, dB = -dt curl E, dJ = alpha
# C^T beta dB, q = E - eta dJ, and the vector updates and dot products), in
# the substep's real type.
RES_WORDS_PER_DOF_ITER = 21


def run_implicit(args, rank, world, device):
    """The implicit resistive substep on the periodic curvilinear n^3 cube
    (Orszag-Tang, eta from the reference's radial window 0.84 < r < 1.04 with
    eta_max_mercury 1.25e7), FP64 (CG) and mixed precision (FP32 CG inside
    FP64 refinement), both to a relative residual of 1e-10.  The substep's
    time is the step's time with it minus the step's time without it (same
    inputs); value: CG unknown-iterations per second of the FP64 solve."""
    import numpy as np
    import torch

    from mpcns_mercury_b200 import Context, reference_constants
    from mpcns_mercury_b200 import setup as S

    n = args.implicit_n
    geom, f = S.cube_case(n)
    eta = S.resistivity_eta(geom, reference_constants())
    peak, peak_kind = load_peaks()
    sampler = ClockSampler(device.index if device.index is not None else 0)

    def timed(precision, resistive):
        k = reference_constants(cfl=0.4, resistive=resistive, res_rtol=1e-10, res_max_it=2000)
        ctx = Context([(n, n, n)], 4, k, precision=precision)
        for name in UPLOAD_FIELDS:
            a = f[name]
            ctx.upload(capi_field(name), a.data, a.lo, a.hi)
        if resistive:
            for name, a in eta.items():
                ctx.upload(name.upper(), a.data, a.lo, a.hi)
        ctx.sync("UCELL")
        ctx.sync("BFACE")
        ctx.prepare()
        dofs = 0
        if resistive:
            w = ctx.download("RES_W", (0, 0, 0), (n + 1, n + 1, n + 1))
            dofs = int(np.count_nonzero(w > 0.0))
        stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
        for _ in range(args.warmup):
            ctx.step(1)
        torch.cuda.synchronize()
        ms, iters, refinements, relres = 0.0, 0, 0, 0.0
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.step(1)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            info = ctx.info()
            iters += info.res_iters
            refinements += info.res_refinements
            relres = max(relres, info.res_relres)
            assert info.status == 0, info.status
        ctx.close()
        return ms / args.steps, dofs, iters / args.steps, refinements / args.steps, relres

    out = {}
    if rank == 0:
        sampler.start()
    for prec, label in ((0, "fp64"), (1, "mixed")):
        ms_res, dofs, it, ref, relres = timed(prec, True)
        ms_plain, _, _, _, _ = timed(prec, False)
        sub_ms = ms_res - ms_plain
        dof_iters = dofs * it
        word = 8 if prec == 0 else 4
        gbs = RES_WORDS_PER_DOF_ITER * word * dof_iters / (sub_ms * 1e-3) / 1e9
        out[label] = {"step_ms_with_substep": round(ms_res, 4), "step_ms_without": round(ms_plain, 4),
                      "substep_ms": round(sub_ms, 4), "unknowns": dofs, "cg_iterations_per_step": round(it, 2),
                      "refinements_per_step": round(ref, 2), "max_relres": relres,
                      "us_per_cg_iteration": round(1e3 * sub_ms / max(it, 1e-9), 3),
                      "dof_iterations_per_s": round(dof_iters / (sub_ms * 1e-3), 1),
                      "achieved_gbs": round(gbs, 2), "frac_of_peak": round(gbs / peak, 4)}
    clocks = sampler.stop() if rank == 0 else None
    f64 = out["fp64"]
    return {
        "metric": "implicit resistive CG unknown-iterations/s", "value": f64["dof_iterations_per_s"],
        "unit": "dof-iterations/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": f64["step_ms_with_substep"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "implicit", "cells": [n, n, n], "nghost": 4, "res_rtol": 1e-10,
                   "eta": "reference window 0.84 < r < 1.04, eta_max_mercury 1.25e7", "l2": "not flushed",
                   "bytes_per_dof_iteration": f"{RES_WORDS_PER_DOF_ITER} words of the real type",
                   "peak_gbs": peak, "peak_source": peak_kind, **out},
        "clocks": clocks,
    }


# ------------------------------------------------------------------ reference arm
def reference_members(args):
    """Every member of ``args.workload`` as the reference harness job that
    sets it up exactly as our arm runs it, with its owned cells: [(job, cells)].
    Sizes and upstream conditions are drawn without loading the CUDA library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo
    from mpcns_mercury_b200 import workloads as W

    def cube(n, sid):
        job = dict(mo.CUBE_JOB)
        job.update(n=" ".join(str(int(v)) for v in n), solve_id=sid)
        return job, int(n[0]) * int(n[1]) * int(n[2])

    if args.workload.startswith("cube"):
        n = int(args.workload[4:])
        return [cube((n, n, n), 0)]
    if args.workload == "ensemble":
        return [cube(c, s) for s, c in enumerate(W.ensemble_sizes(args.solves))]
    if args.workload == "serve":
        return [cube(c, s) for s, c in enumerate(W.ensemble_sizes(args.shapes, stream=200000))]
    if args.workload == "shells":
        from mpcns_mercury_b200 import magnetosphere as M

        out = []
        for c in M.ensemble(args.solves, stream=300000):
            up = [float(v) for v in c.upstream]
            job = dict(mo.SHELL_JOB)
            job.update(na=c.na, nr=c.nr, na_fraction=float(c.na_fraction),
                       initial_line=" ".join(repr(v) for v in up),
                       farfield_line=" ".join(repr(v) for v in (up[0], up[1], up[2], up[4], up[5])))
            if c.resistive:  # the implicit substep, solved by the reference's GMRES to the same tolerance
                job.update(resistive=1, eta_max=float(c.eta_max), eta_r_inner=float(c.eta_r_inner),
                           eta_r_outer=float(c.eta_r_outer), eta_width=float(c.eta_width),
                           ksp_rtol=float(c.res_rtol), ksp_atol=1e-300, ksp_max_it=int(c.res_max_it))
            out.append((job, c.cell_count()))
        return out
    raise SystemExit(f"unknown workload {args.workload}")


def run_reference_member(job, warm, steps):
    """One member on the reference build (one single-rank process): ``warm``
    untimed StepOnce calls, then ``steps`` timed ones.  Returns (seconds per
    timed step, owned cells)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    job = dict(job)
    job.update(steps=warm + steps, time_from=warm, dump_fields="U_H", dump_at=str(warm + steps), dump_grid=0,
               dump_taper=0, dump_static="")
    d = mo.run_job(job, timeout=3600)
    secs, nsteps, ncell = d[("timing", -1)].data.ravel()
    return float(secs) / max(1.0, float(nsteps)), int(ncell)


# Host memory of one reference process per owned cell, an upper estimate
# (its fields with four ghost layers, the implicit solve's matrix and Krylov
# vectors): concurrent members are capped so that the largest ones fit.
REF_BYTES_PER_CELL = 16384


def _ref_procs_in_memory(members):
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError, AttributeError):
        return len(members)
    biggest = max(m[1] for m in members) * REF_BYTES_PER_CELL
    return max(1, int(0.8 * avail // max(biggest, 1)))


def reference_sample(members, warm, steps, procs):
    """Every member on the reference build, the members partitioned over
    ``procs`` host cores (longest first onto the least loaded core), each core
    running its members one after another as single-rank processes.  A step
    of the whole workload advances every member once, so it takes as long as
    the busiest core's members take per step.  Returns (Mcell-updates/s,
    seconds per workload step, cores used)."""
    from concurrent.futures import ThreadPoolExecutor

    procs = max(1, min(procs, len(members), _ref_procs_in_memory(members)))
    load = [0] * procs
    parts = [[] for _ in range(procs)]
    for sid in sorted(range(len(members)), key=lambda q: -members[q][1]):
        w = load.index(min(load))
        parts[w].append(sid)
        load[w] += members[sid][1]

    def core(part):
        return sum(run_reference_member(members[sid][0], warm, steps)[0] for sid in part)

    with ThreadPoolExecutor(max_workers=procs) as ex:
        per_core = list(ex.map(core, parts))
    step_s = max(per_core)
    cells = sum(m[1] for m in members)
    return cells / step_s / 1e6, step_s, procs


def cpu_baseline_sample(args, cells=None):
    """The reference (built from its sources) on this host: a bounded sample
    of the same workload (its first members, a few steps each, on every
    core), and the 32^3 cube on one core (the single-block case, one solve)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    if not mo.available():
        return None
    members = reference_members(args)
    cores = os.cpu_count() or 1
    sample = members[:min(len(members), cores)]
    rate, step_s, procs = reference_sample(sample, 1, 2, cores)
    cube = dict(mo.CUBE_JOB)
    cube.update(n="32 32 32", solve_id=0)
    one_step_s, one_cells = run_reference_member(cube, 1, 5)
    return {"value": round(rate, 4), "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{args.workload}: the first {len(sample)} members at their own shapes and conditions, one "
                      f"single-rank reference process per member (oracle/_ref, built from the reference sources) "
                      f"spread over {procs} cores, 1 untimed + 2 timed StepOnce calls each, setup excluded",
            "one_core_cube32": {"value": round(one_cells / one_step_s / 1e6, 4), "unit": UNIT, "cores": 1,
                                "ms_per_step": round(1e3 * one_step_s, 3),
                                "sample": "periodic curvilinear 32^3 cube (Orszag-Tang, 2 ion fluids, Hall + p_e), "
                                          "one process on one core, 1 untimed + 5 timed StepOnce calls"}}


def run_reference(args, rank, world):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mercury_oracle as mo

    if rank != 0:
        return None
    if not mo.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/mercury_ref is not built on this host"}
    members = reference_members(args)
    cores = os.cpu_count() or 1
    # every member once: one untimed step, then a bounded number of timed
    # steps (the reference's per-member setup takes seconds, so the whole
    # run stays within minutes)
    steps = max(1, min(args.steps, args.ref_steps))
    t0 = time.perf_counter()
    value, step_s, procs = reference_sample(members, 1, steps, cores)
    wall = time.perf_counter() - t0
    cells = sum(m[1] for m in members)
    return {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": round(1e3 * step_s, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "members": len(members), "cells_per_replica": cells,
                       "wall_s": round(wall, 2),
                       "implementation": "reference solver compiled from its own sources (oracle/_ref), one "
                                         f"single-rank process per member, members spread over {procs} cores",
                       "timing": "per member: 1 untimed StepOnce, then the timed ones (setup excluded); a workload "
                                 "step takes as long as the busiest core's members take per step"},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": procs, "kind": "reference",
                             "sample": f"all {len(members)} members at their own shapes, {steps} timed steps each"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="shells",
                    help="shells (default), ensemble, serve, implicit, cube32, cubeN")
    ap.add_argument("--solves", type=int, default=None,
                    help="ensemble / shells: solves per GPU (default: 64 periodic boxes; the first "
                         f"{SHELL_SOLVES} magnetosphere shells, which fit in HBM with their FP64 companions)")
    ap.add_argument("--cg-host-loop", action="store_true",
                    help="shells: launch the implicit substep's CG iterations from the host (for profilers that do "
                         "not follow conditional graph nodes)")
    ap.add_argument("--batched-only", action="store_true",
                    help="ensemble: run only the mixed batch (profiling; no plain/FP64 legs, no error check)")
    ap.add_argument("--requests", type=int, default=400, help="serve: requests")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: mean arrivals per second")
    ap.add_argument("--shapes", type=int, default=16, help="serve: distinct request shapes")
    ap.add_argument("--capacity", type=int, default=64, help="serve: batch slots")
    ap.add_argument("--hbm-budget", type=float, default=100e9, help="serve: device bytes for admitted solves")
    ap.add_argument("--implicit-n", type=int, default=64, help="implicit: cells per axis of the cube")
    ap.add_argument("--error-steps", type=int, default=100,
                    help="ensemble: steps after which the mixed batch's error against FP64 is stated")
    ap.add_argument("--ref-steps", type=int, default=5, help="reference arm: timed steps per member (at most --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="shells: requests of the serving leg (p50/p99; 0 leaves it out)")
    ap.add_argument("--serve-rate", type=float, default=40.0, help="shells: their mean arrivals per second")
    ap.add_argument("--config-steps", type=int, default=200, help="config2: timed steps")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.solves is None:
        args.solves = SHELL_SOLVES if args.workload == "shells" else 64

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
        if args.workload == "shells":
            line = run_shells(args, rank, world, device)
        elif args.workload == "ensemble":
            line = run_ensemble(args, rank, world, device)
        elif args.workload == "serve":
            line = run_serving(args, rank, world, device)
        elif args.workload == "serve-shells":
            line = run_serving_shells(args, rank, world, device)
        elif args.workload == "config2":
            line = run_config2(args, rank, world, device)
        elif args.workload == "implicit":
            line = run_implicit(args, rank, world, device)
        else:
            line = run_ours(args, rank, world, device)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
