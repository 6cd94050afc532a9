"""Synthetic workloads of the step and the upload of their fields.

cube      one periodic curvilinear block, Orszag-Tang vortex on two ion
          fluids (the single-block case of the reference's test setup).
ensemble  independent periodic-box solves of uneven sizes: per block, cells
          per axis drawn log-uniform (x, y in [24, 64], z in [24, 128]), each
          solve with its own seeded noise (solve_id), all advanced together
          by one batch.

Inputs are generated on the host in the reference's FieldBlock index space
and uploaded through the C ABI (mhd_upload_field / mhd_batch_upload_field).
"""
from __future__ import annotations

import math

import numpy as np

from . import setup as S
from .capi import REF_FIELD

NGHOST = 4

# Every field the step reads: static geometry, sources and the state.
UPLOAD_FIELDS = ["Jac", "JDxi", "JDet", "JDze", "Area_xi", "Area_eta", "Area_zeta", "dl_xi", "dl_eta", "dl_zeta",
                 "dr_xi", "dr_eta", "dr_zeta", "beta_xi", "beta_eta", "beta_zeta", "alpha_xi", "alpha_eta",
                 "alpha_zeta", "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Badd_xi", "Badd_eta", "Badd_zeta",
                 "Photo_rate", "cell_x", "cell_y", "cell_z", "taper_xi", "taper_eta", "taper_zeta",
                 "U_H", "U_Na", "B_xi", "B_eta", "B_zeta"]
STATE_FIELDS = ["U_H", "U_Na", "B_xi", "B_eta", "B_zeta"]
CAPI_NAME = {"beta_xi": "HODGE_FACE_XI", "beta_eta": "HODGE_FACE_ETA", "beta_zeta": "HODGE_FACE_ZETA",
             "alpha_xi": "HODGE_EDGE_XI", "alpha_eta": "HODGE_EDGE_ETA", "alpha_zeta": "HODGE_EDGE_ZETA",
             "cell_x": "CELL_X", "cell_y": "CELL_Y", "cell_z": "CELL_Z"}


def capi_field(name: str) -> str:
    return CAPI_NAME.get(name) or REF_FIELD[name]


def case_fields(cells, solve_id: int = 0) -> dict:
    """{reference field name: Arr} of one periodic box (cells per axis)."""
    _, f = S.cube_case(tuple(int(v) for v in cells), solve_id=solve_id)
    return {k: f[k] for k in UPLOAD_FIELDS}


def upload_case(upload, fields: dict, block: int = 0) -> int:
    """Calls upload(capi name, array, lo, hi, block) for every input field;
    returns the bytes uploaded."""
    nbytes = 0
    for name in UPLOAD_FIELDS:
        a = fields[name]
        upload(capi_field(name), a.data, a.lo, a.hi, block)
        nbytes += a.data.nbytes
    return nbytes


def upload_request(upload, setup_geometry, fields: dict, block: int = 0) -> int:
    """Inputs of one solve: with a "nodes" entry (the block's node
    coordinates, AoS) the static fields are computed on the device
    (setup_geometry(nodes)) and only the state is uploaded; otherwise every
    input field is uploaded.  Returns the bytes sent to the device."""
    if "nodes" not in fields:
        return upload_case(upload, fields, block)
    setup_geometry(fields["nodes"])
    nbytes = fields["nodes"].nbytes
    for name in STATE_FIELDS:
        a = fields[name]
        upload(capi_field(name), a.data, a.lo, a.hi, block)
        nbytes += a.data.nbytes
    return nbytes


def state_cases(cases):
    """[(cells, solve_id)] -> [{"nodes": ..., state fields}]: the requests of
    device-side setup (host work: nodes and the seeded initial state only)."""
    out = []
    for cells, sid in cases:
        nodes, state = S.cube_state(tuple(int(v) for v in cells), solve_id=sid)
        out.append({"nodes": nodes, **state})
    return out


def setup_case_on_device(setup_geometry, upload, cells, solve_id: int = 0) -> int:
    """One periodic box set up with its static fields computed on the device:
    setup_geometry(nodes) (mhd_setup_geometry) then upload(capi name, array,
    lo, hi, block) of the initial state only; returns the bytes uploaded."""
    nodes, state = S.cube_state(tuple(int(v) for v in cells), solve_id=solve_id)
    setup_geometry(nodes)
    nbytes = nodes.nbytes
    for name in STATE_FIELDS:
        a = state[name]
        upload(capi_field(name), a.data, a.lo, a.hi, 0)
        nbytes += a.data.nbytes
    return nbytes


def ensemble_sizes(nsolves: int, stream: int = 100000):
    """Per-solve block sizes of the ensemble: cells per axis log-uniform,
    x and y in [24, 64], z in [24, 128] (the per-block range 24^3 .. 64x64x128),
    drawn from the seeded generator with solve_id = ``stream`` (a stream no
    solve's own noise uses).  Computed without the CUDA library, so that the
    CPU reference arm can size the same workload."""
    u = S.host_uniform_sym(stream, 0.5, 3 * nsolves) + 0.5
    lo, hx, hz = math.log(24.0), math.log(64.0), math.log(128.0)
    sizes = []
    for s in range(nsolves):
        a, b, c = u[3 * s:3 * s + 3]
        sizes.append((int(round(math.exp(lo + a * (hx - lo)))), int(round(math.exp(lo + b * (hx - lo)))),
                      int(round(math.exp(lo + c * (hz - lo))))))
    return sizes


def _case_worker(spec):
    cells, solve_id = spec
    return case_fields(cells, solve_id=solve_id)


def generate_cases(specs, workers: int | None = None):
    """Yields case_fields(cells, solve_id) for every (cells, solve_id) in
    ``specs``, in order, computed by a pool of spawned host processes (safe to
    start after CUDA is initialised in this process)."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor

    specs = list(specs)
    workers = workers or min(len(specs), max(1, (os.cpu_count() or 2) - 1), 32)
    if workers <= 1 or len(specs) <= 1:
        for sp in specs:
            yield _case_worker(sp)
        return
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        yield from ex.map(_case_worker, specs)
