"""The output step (mpcns_mercury_b200.output.write_output_step) against the
three files the reference writes at an output step (restart, plot file,
run-data file), byte for byte.  The solve is a stand-in serving the
reference's own dumped state through the Context interface (download, sync,
save_restart, info), so the files check the output step's glue and writers
on the host; the run-data monitors (wall-clock figures) are the reference's."""
import os
import struct
import types

import numpy as np
import pytest

STEPS = 2
FIELDS = "U_H U_Na B_xi B_eta B_zeta PV_H PV_Na B_cell Bind_cell Na J_cell"


def _monitors(path):
    raw = open(path, "rb").read()
    p = 8 + 4 + 4 + 8 + 8
    nref = struct.unpack_from("<i", raw, p)[0]
    p += 4 + 8 * nref + 8
    out = []
    for fmt, size in (("<d", 8), ("<i", 4)):
        n = struct.unpack_from("<i", raw, p)[0]
        p += 4
        m = {}
        for _ in range(n):
            ln = struct.unpack_from("<i", raw, p)[0]
            m[raw[p + 4:p + 4 + ln].decode()] = struct.unpack_from(fmt, raw, p + 4 + ln)[0]
            p += 4 + ln + size
        out.append(m)
    return out


class DumpSolve:
    """The Context interface over a reference dump (state after STEPS steps)."""

    def __init__(self, dump, cells, nghost):
        from mpcns_mercury_b200 import capi

        self.d, self.cells, self.nghost = dump, cells, nghost
        self.name = {v: k for k, v in capi.REF_FIELD.items()}
        dt, time = dump[(f"step{STEPS}:dt_time", -1)].data.ravel()
        self.meta = types.SimpleNamespace(step=STEPS, time=float(time), dt=float(dt))
        self.synced = []

    def _rec(self, field, block):
        ref = self.name[field]
        key = (f"step{STEPS}:{ref}", block)
        return self.d[key] if key in self.d else self.d[("static:" + ref, block)]

    def download(self, field, lo, hi, block=0):
        r = self._rec(field, block)
        sl = tuple(slice(lo[a] - r.lo[a], hi[a] - r.lo[a]) for a in range(3))
        return r.data[sl]

    def sync(self, group):
        self.synced.append(group)

    def save_restart(self, path):
        from mpcns_mercury_b200 import capi

        fields = {f: [self._rec(c, b).data for b in range(len(self.cells))]
                  for f, c in zip(capi.RESTART_FIELDS, capi.RESTART_CAPI)}
        capi.restart_write(path, self.meta.step, self.meta.time, self.cells, self.nghost, fields)

    def info(self):
        return self.meta


@pytest.mark.parametrize("extra,n,nblock", [({}, 6, 1), ({"case": "lattice", "nb": "2 1 2"}, 4, 4)])
def test_output_step_matches_reference(ref_oracle, tmp_path, extra, n, nblock):
    from mpcns_mercury_b200.output import write_output_step

    ref = {k: str(tmp_path / f"ref.{k}") for k in ("bin", "plt", "run")}
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=n, steps=STEPS, dump_at=str(STEPS), dump_fields=FIELDS, dump_static="Jac", dump_grid=1,
               write_restart=ref["bin"], write_tecplot=ref["plt"], write_rundata=ref["run"], **extra)
    d = ref_oracle.run_job(job, workdir=str(tmp_path / "job"))
    cells = [(n, n, n)] * nblock
    nghost = -d[(f"step{STEPS}:PV_H", 0)].lo[0]
    nodes = []
    for b in range(nblock):
        rec = d[("node_x", b)]
        sl = tuple(slice(-lo, -lo + n + 1) for lo in rec.lo)
        nodes.append(np.stack([d[("node_" + a, b)].data[..., 0][sl] for a in "xyz"], axis=-1))
    na = [d[(f"step{STEPS}:Na", b)].data for b in range(nblock)]
    mon_d, mon_i = _monitors(ref["run"])
    solve = DumpSolve(d, cells, nghost)
    paths = write_output_step(solve, str(tmp_path / "out"), cells, nghost, nodes, na, monitors_d=mon_d,
                              monitors_i=mon_i)
    assert solve.synced == ["B_CELL", "J_CELL"]
    assert os.path.basename(paths["restart"]) == "flow_field0000.bin"
    for key, ours in (("bin", "restart"), ("plt", "plot"), ("run", "rundata")):
        with open(ref[key], "rb") as a, open(paths[ours], "rb") as c:
            assert a.read() == c.read(), key
