"""Request loop over a batch (mhd_batch): independent solves arrive over time,
are admitted while a slot and device memory are free, run together on one
CUDA graph per step (continuous batching: a solve joins or leaves between
graph launches while the others keep running), and leave when their steps
are done.  The reference runs one solve per MPI job and has no counterpart;
this is the serving layer around the step.

    server = Server(capacity=64, precision=1, hbm_budget=100e9)
    stats = server.serve(requests)      # requests: arrival times, sizes, steps
    stats["latency_p50_s"], stats["latency_p99_s"], stats["mcell_updates_per_s"]
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .constants import reference_constants
from .workloads import NGHOST, STATE_FIELDS, capi_field, upload_request


@dataclass
class Request:
    rid: int
    arrival_s: float          # seconds after the start of serving
    cells: tuple              # cells per axis of the (single, periodic) block
    steps: int
    fields: dict              # {reference field name: Arr} inputs: static + initial state, or the
                              # block's "nodes" (statics computed on the device) + initial state
    keep_result: bool = False
    geometry: object = None   # requests with equal keys share their grid and static fields (default: cells)
    case: object = None       # a magnetosphere.ShellCase: the solve is that shell, set up on the device
                              # from its parameters (cells and fields unused)
    # filled in by the server
    admitted_s: float = float("nan")
    done_s: float = float("nan")
    result: dict = field(default_factory=dict)
    slot: int = -1


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else float("nan")


def _geometry_key(req: Request):
    if req.case is not None:
        return ("shell", req.case.na, req.case.nr, bool(req.case.resistive))
    return req.geometry if req.geometry is not None else tuple(req.cells)


def _cell_count(req: Request) -> int:
    return req.case.cell_count() if req.case is not None else int(np.prod(req.cells))


def _shell_result(get, case):
    """Owned state of every panel of a shell, from get(field, lo, hi, block)."""
    n = (case.na, case.na, case.nr)
    out = {}
    for name, st in (("U_H", (0, 0, 0)), ("U_NA", (0, 0, 0)), ("B_XI", (1, 0, 0)), ("B_ETA", (0, 1, 0)),
                     ("B_ZETA", (0, 0, 1))):
        hi = tuple(n[a] + st[a] for a in range(3))
        out[name] = [get(name, (0, 0, 0), hi, b) for b in range(6)]
    return out


def _upload_state(upload, fields):
    for name in STATE_FIELDS:
        a = fields[name]
        upload(capi_field(name), a.data, a.lo, a.hi, 0)


class Server:
    """Continuous-batching server of independent solves on one GPU.

    The first request of a grid makes a template solve holding the grid's
    topology tables and static fields (never stepped); every request is then
    admitted with mhd_batch_add_like from its grid's template (shared tables,
    static fields copied on the device) and uploads only its state."""

    def __init__(self, capacity: int = 64, precision: int = 1, hbm_budget: float = 100e9, chunk_steps: int = 8,
                 cfl: float = 0.4, max_grids: int = 16, topologies=None, nodes=None):
        """topologies, nodes: a magnetosphere.TopologyCache and a dict of grid
        nodes to take shell grids from (the caller's, kept open)."""
        self.batch = capi.Batch(capacity + max_grids, precision)
        self.capacity = capacity
        self.max_grids = max_grids
        self.precision = precision
        self.hbm_budget = float(hbm_budget)
        self.chunk = int(chunk_steps)
        self.constants = reference_constants(cfl=cfl)
        self.templates = {}     # geometry key -> template slot
        self.grid_bytes = {}    # geometry key -> device bytes of one solve
        self.topologies = topologies  # shells: their grids' sync tables
        self._own_topologies = topologies is None
        self.nodes = nodes if nodes is not None else {}  # shells: their grids' node coordinates

    def close(self):
        self.batch.close()
        if self.topologies is not None and self._own_topologies:
            self.topologies.close()

    def _shell_grid(self, case):
        from . import magnetosphere as M

        if self.topologies is None:
            self.topologies = M.TopologyCache()
        key = ("shell", case.na, case.nr, bool(case.resistive))
        if key not in self.nodes:
            self.nodes[key] = capi.shell_grid(case.na, case.nr, case.r_out, NGHOST + 1)
        return self.topologies.get(case), self.nodes[key]

    # ------------------------------------------------------------------ one solve
    def _template(self, req: Request) -> int:
        key = _geometry_key(req)
        if key not in self.templates:
            if len(self.templates) >= self.max_grids:
                raise RuntimeError(f"more than {self.max_grids} distinct grids")
            if req.case is not None:  # a shell grid: its tables (every request sets its own fields up)
                from . import magnetosphere as M

                topo, _ = self._shell_grid(req.case)
                d = capi.SolveDesc(req.case.cells, NGHOST, M.constants(req.case), precision=self.precision,
                                   topology=topo)
                self.templates[key] = self.batch.add(d)
                d.close()
                return self.templates[key]
            slot = self.batch.add_periodic(req.cells, NGHOST, self.constants)
            upload_request(lambda f, a, lo, hi, b: self.batch.upload(slot, f, a, lo, hi, block=b),
                           lambda nodes: self.batch.setup_geometry(slot, nodes), req.fields)
            self.templates[key] = slot
        return self.templates[key]

    def _admit(self, req: Request) -> int:
        if req.case is not None:
            from . import magnetosphere as M

            k = M.constants(req.case)
            slot = self.batch.add_like(self._template(req), constants=k, copy_static=False)
            _, nodes = self._shell_grid(req.case)
            M.set_up(self.batch, req.case, slot=slot, k=k, nodes=nodes)
            self.batch.prepare(slot)
            self.batch.request(slot, req.steps)
            req.slot = slot
            return slot
        slot = self.batch.add_like(self._template(req), copy_static=True)
        _upload_state(lambda f, a, lo, hi, b: self.batch.upload(slot, f, a, lo, hi, block=b), req.fields)
        self.batch.sync(slot, "UCELL")
        self.batch.sync(slot, "BFACE")
        self.batch.prepare(slot)
        self.batch.request(slot, req.steps)
        req.slot = slot
        return slot

    def _retire(self, req: Request):
        if req.keep_result and req.case is not None:
            req.result = _shell_result(lambda f, lo, hi, b: self.batch.download(req.slot, f, lo, hi, block=b),
                                       req.case)
        elif req.keep_result:
            req.result = {name: self.batch.download(req.slot, capi_field(name), req.fields[name].lo,
                                                    req.fields[name].hi) for name in STATE_FIELDS}
        self.batch.remove(req.slot)

    @staticmethod
    def _bytes(req: Request, precision: int, topology=None) -> int:
        """Device bytes of the request's solve (a shell's from its grid's
        topology: the given handle, else one built and freed here)."""
        if req.case is not None:
            from . import magnetosphere as M

            own = topology is None
            topo = M.topology(req.case) if own else topology
            d = capi.SolveDesc(req.case.cells, NGHOST, M.constants(req.case), precision=precision, topology=topo)
            b = d.device_bytes()
            d.close()
            if own:
                capi.lib().mhd_topology_destroy(topo)
            return b
        d = capi.SolveDesc([req.cells], NGHOST, reference_constants(), precision=precision)
        b = d.device_bytes()
        d.close()
        return b

    def _need(self, req: Request) -> int:
        key = _geometry_key(req)
        if key not in self.grid_bytes:
            topo = self._shell_grid(req.case)[0] if req.case is not None else None
            self.grid_bytes[key] = self._bytes(req, self.precision, topo)
        return self.grid_bytes[key]

    # ------------------------------------------------------------------ the loop
    def serve(self, requests, clock=time.perf_counter):
        """Serve ``requests`` (sorted by arrival) in real time; returns statistics.

        Each pass admits the requests that have arrived (asynchronous calls,
        ordered on the batch's stream), enqueues `chunk` graph launches and a
        state snapshot, then waits for the previous pass's snapshot only: the
        host retires finished solves and admits new ones while the GPU runs
        the next chunk.  A solve that finishes inside a chunk idles for the
        rest of it."""
        pending = sorted(requests, key=lambda r: r.arrival_s)
        need = {r.rid: self._need(r) for r in pending}
        running: dict[int, Request] = {}
        epoch: dict[int, int] = {}   # slot -> snapshots enqueued before its request
        used = 0
        t0 = clock()
        nxt = 0
        graph_steps = 0
        snaps = 0
        ticket = None                # (ticket, snapshot number) of the last enqueued snapshot
        while nxt < len(pending) or running:
            now = clock() - t0
            # admission: arrived requests, in arrival order, while a slot and memory are
            # free (a grid's template, made on first use, is charged once)
            while (nxt < len(pending) and pending[nxt].arrival_s <= now and len(running) < self.capacity
                   and used + need[pending[nxt].rid] * (1 if _geometry_key(pending[nxt]) in self.templates else 2)
                   <= self.hbm_budget):
                r = pending[nxt]
                if _geometry_key(r) not in self.templates:
                    used += need[r.rid]
                r.admitted_s = clock() - t0
                self._admit(r)
                running[r.slot] = r
                epoch[r.slot] = snaps
                used += need[r.rid]
                nxt += 1
            if not running:
                if pending[nxt].arrival_s <= clock() - t0:
                    raise RuntimeError(f"request {pending[nxt].rid} does not fit the device budget "
                                       f"({need[pending[nxt].rid]} bytes, {used} held by grid templates)")
                # idle until the next arrival
                wait = pending[nxt].arrival_s - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.05))
                continue
            self.batch.run(self.chunk)
            graph_steps += self.chunk
            new = (self.batch.poll_async(), snaps + 1)
            snaps += 1
            if ticket is not None:
                infos = self.batch.poll_wait(ticket[0])
                now = clock() - t0
                for slot in list(running):
                    if epoch[slot] >= ticket[1]:
                        continue  # admitted after that snapshot was taken
                    inf = infos[slot]
                    if inf.status != 0:
                        raise capi.MhdError(inf.status, f"request {running[slot].rid} (slot {slot})")
                    if inf.remaining == 0:
                        r = running.pop(slot)
                        del epoch[slot]
                        r.done_s = now
                        self._retire(r)
                        used -= need[r.rid]
            ticket = new
        self.batch.poll()
        makespan = clock() - t0
        lat = [r.done_s - r.arrival_s for r in pending]
        work = sum(_cell_count(r) * r.steps for r in pending)
        return {"requests": len(pending), "makespan_s": makespan, "graph_steps": graph_steps,
                "cell_updates": work, "mcell_updates_per_s": work / makespan / 1e6,
                "latency_p50_s": percentile(lat, 50), "latency_p99_s": percentile(lat, 99),
                "latency_mean_s": float(np.mean(lat)) if lat else float("nan")}


def serve_one_by_one(requests, precision: int = 0, clock=time.perf_counter, cfl: float = 0.4, topologies=None,
                     nodes=None, fluid_tile: int = 0):
    """The same requests served first-come first-served through the plain
    single-solve path (mhd_ctx, one solve on the GPU at a time).  Like the
    server, it keeps one context per grid (tables and static fields uploaded
    once) and uploads each request's state; a shell request sets its fields
    up on its grid's context (topologies / nodes: shell grids prepared
    ahead, as for the server)."""
    pending = sorted(requests, key=lambda r: r.arrival_s)
    ctxs = {}
    shells = dict(nodes or {})  # shell grids: nodes per grid, and "topo": the topology cache
    own_topo = topologies is None
    if topologies is not None:
        shells["topo"] = topologies
    t0 = clock()
    for r in pending:
        now = clock() - t0
        if r.arrival_s > now:
            time.sleep(r.arrival_s - now)
        r.admitted_s = clock() - t0
        key = _geometry_key(r)
        ctx = ctxs.get(key)
        if r.case is not None:  # a shell: one context per grid, every request sets its own fields up
            from . import magnetosphere as M

            if "topo" not in shells:
                shells["topo"] = M.TopologyCache()
            k = M.constants(r.case)
            if key not in shells:
                shells[key] = capi.shell_grid(r.case.na, r.case.nr, r.case.r_out, NGHOST + 1)
            if ctx is not None and ctx.info().status != 0:
                ctx.close()
                ctx = None
            if ctx is None:
                ctx = capi.Context(r.case.cells, NGHOST, k, topology=shells["topo"].get(r.case), precision=precision,
                                   keep_topology=True)
                ctx.fluid_tile(fluid_tile)
                ctxs[key] = ctx
            ctx.set_constants(k)
            M.set_up(ctx, r.case, k=k, nodes=shells[key])
            ctx.prepare()
            ctx.step(r.steps)
            if r.keep_result:
                r.result = _shell_result(lambda f, lo, hi, b: ctx.download(f, lo, hi, block=b), r.case)
            r.done_s = clock() - t0
            continue
        if ctx is None:
            ctx = capi.Context([r.cells], NGHOST, reference_constants(cfl=cfl), precision=precision)
            upload_request(lambda f, a, lo, hi, b: ctx.upload(f, a, lo, hi, block=b), ctx.setup_geometry, r.fields)
            ctxs[key] = ctx
        else:
            _upload_state(lambda f, a, lo, hi, b: ctx.upload(f, a, lo, hi, block=b), r.fields)
        ctx.sync("UCELL")
        ctx.sync("BFACE")
        ctx.prepare()
        ctx.step(r.steps)
        if r.keep_result:
            r.result = {name: ctx.download(capi_field(name), r.fields[name].lo, r.fields[name].hi)
                        for name in STATE_FIELDS}
        r.done_s = clock() - t0
    makespan = clock() - t0
    for ctx in ctxs.values():
        ctx.close()
    if "topo" in shells and own_topo:
        shells["topo"].close()
    lat = [r.done_s - r.arrival_s for r in pending]
    work = sum(_cell_count(r) * r.steps for r in pending)
    return {"requests": len(pending), "makespan_s": makespan, "cell_updates": work,
            "mcell_updates_per_s": work / makespan / 1e6, "latency_p50_s": percentile(lat, 50),
            "latency_p99_s": percentile(lat, 99), "latency_mean_s": float(np.mean(lat)) if lat else float("nan")}
