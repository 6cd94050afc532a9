"""The reference's output step (MercurySolver::UpdateControlAndOutput,
Z4_Mercury/src/MercurySolver_Driver.cpp:74-88) for a solve on the GPU: the
checkpoint (MPCNSRST, IOModule::WriteRestartBinFile), the plot file
(Tecplot binary, IOModule::WriteTecplotBinFile in the AllNode mode) and the
run-data file (IOModule::WriteRunDataFile), under the reference's names in
one directory: flow_field<rank>.bin, flow_field<rank>.plt, RunData.bin.

The solve is anything with the Context interface used here: sync(group),
save_restart(path), download(field, lo, hi, block) and info()."""
from __future__ import annotations

import os

from . import capi

# download names of the plot file's cell fields, in capi.TECPLOT_FIELDS order
_CELL_FIELDS = {"PV_H": "PV_H", "PV_Na": "PV_NA", "B_cell": "B_CELL", "Bind_cell": "BIND_CELL", "J_cell": "J_CELL"}


def write_output_step(solve, directory: str, cells, nghost: int, nodes, na, block_names=None, monitors_d=None,
                      monitors_i=None, rank: int = 0) -> dict:
    """Write the three files of an output step; returns their paths.

    cells: cells per block; nghost: ghost layers of the cell fields written
    to the plot file's inputs (the reference's ngg); nodes: per block the
    node coordinates (n+1, n+1, n+1, 3); na: per block the Na density cell
    field over [-nghost, n + nghost) (a static input the solve does not
    hold); monitors: the run's performance monitors for the run-data file
    (the reference's are RuntimeMonitor's wall-clock figures)."""
    os.makedirs(directory, exist_ok=True)
    tag = f"{rank:04d}"
    paths = {"restart": os.path.join(directory, f"flow_field{tag}.bin"),
             "plot": os.path.join(directory, f"flow_field{tag}.plt"),
             "rundata": os.path.join(directory, "RunData.bin")}
    nb = len(cells)
    names = list(block_names) if block_names is not None else ["Fluid"] * nb

    # the checkpoint: every ghost layer of the state, as the reference holds it
    solve.save_restart(paths["restart"])

    # the plot file: the derived cell fields with their ghost layers filled
    solve.sync("B_CELL")
    solve.sync("J_CELL")
    lo = (-nghost,) * 3
    fields = {f: [] for f in capi.TECPLOT_FIELDS}
    jac = []
    for b, n in enumerate(cells):
        hi = tuple(int(v) + nghost for v in n)
        for ref, name in _CELL_FIELDS.items():
            fields[ref].append(solve.download(name, lo, hi, block=b))
        fields["Na"].append(na[b])
        jac.append(solve.download("JAC", (-1, -1, -1), tuple(int(v) + 1 for v in n), block=b))
    info = solve.info()
    capi.tecplot_write(paths["plot"], [tuple(c) for c in cells], names, info.time, nodes, jac, 1, fields, nghost)

    capi.rundata_write(paths["rundata"], info.step, info.time, info.dt, monitors_d=monitors_d, monitors_i=monitors_i)
    return paths
